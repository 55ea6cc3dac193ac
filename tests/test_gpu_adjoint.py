"""The hand-written adjoint (bdb_adjoint), wrapped in a torch.autograd.Function
in this test harness only, against central finite differences of the FP64
forward pass (itself pinned to the oracle and to BD_BOX by the parity tests).

The loss is the mean squared deviation of final pairwise distances of seeded
bead pairs from seeded targets in [10, 60] A; gradients are taken with
respect to the initial positions and to scale factors on every bead's LJ
epsilon and sigma, every bond's H and the Debye length. The decks use cutoffs
beyond the chain's extent, so no pair crosses a cutoff under the finite
differences."""
import copy

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

from bd_box_b200 import decks, engine  # noqa: E402

K, CKPT, SEED = 12, 5, 4242


def scaled(deck, x0=None, s=(1.0, 1.0, 1.0, 1.0)):
    d = copy.deepcopy(deck)
    if x0 is not None:
        d.coord = d.coord.copy()
        d.coord[:, :3] = x0
    d.LJ = d.LJ.copy()
    d.LJ[:, 1] *= s[0]
    d.LJ[:, 0] *= s[1]
    d.bond_parms = d.bond_parms.copy()
    d.bond_parms[:, 2] *= s[2]
    d.prm = dict(d.prm)
    d.prm["kappa_c"] = d.prm["kappa_c"] / s[3]
    return d


def loss_only(deck, pairs, targets):
    sysm = engine.System(deck, precision=engine.PREC_FP64, refresh=1, noise=engine.NOISE_PHILOX, seed=SEED)
    sysm.step(K)
    x = sysm.get_coord()[:, :3]
    sysm.close()
    r = np.linalg.norm(x[pairs[:, 1]] - x[pairs[:, 0]], axis=1)
    return float(np.mean((r - targets) ** 2))


@pytest.fixture(scope="module")
def case(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("adj"))
    deck = decks.read_deck(decks.write_chain_deck(d, "adj", 48, seed=17, hydro="cholesky",
                                                  extra={"cutoff_c": 1000, "cutoff_lj": 1000, "nb_list": "brute"}))
    rng = np.random.default_rng(3)
    pairs = np.array([rng.choice(deck.n, 2, replace=False) for _ in range(16)], dtype=np.int32)
    targets = rng.uniform(10, 60, size=len(pairs))
    return deck, pairs, targets


def test_adjoint_matches_finite_differences(case):
    deck, pairs, targets = case
    sysm = engine.System(deck, precision=engine.PREC_FP64, refresh=1, noise=engine.NOISE_PHILOX, seed=SEED)
    loss, gx, gp = sysm.adjoint(K, CKPT, pairs, targets)
    sysm.close()
    assert abs(loss - loss_only(deck, pairs, targets)) <= 1e-12 * loss
    rng = np.random.default_rng(8)
    h = 1e-4
    x0 = deck.coord[:, :3]
    for _ in range(3):
        v = rng.standard_normal(x0.shape)
        v /= np.linalg.norm(v)
        fd = (loss_only(scaled(deck, x0 + h * v), pairs, targets) -
              loss_only(scaled(deck, x0 - h * v), pairs, targets)) / (2 * h)
        an = float(np.sum(gx * v))
        assert abs(fd - an) <= 1e-4 * max(abs(fd), 1e-3 * np.abs(gx).sum()), (fd, an)
    for k in range(4):
        sp, sm = [1.0] * 4, [1.0] * 4
        sp[k] += h
        sm[k] -= h
        fd = (loss_only(scaled(deck, s=sp), pairs, targets) - loss_only(scaled(deck, s=sm), pairs, targets)) / (2 * h)
        assert abs(fd - gp[k]) <= 1e-4 * max(abs(fd), 1e-6), (k, fd, gp[k])


def test_adjoint_through_torch_autograd(case):
    torch = pytest.importorskip("torch")
    deck, pairs, targets = case

    class Trajectory(torch.autograd.Function):
        """loss(x0, scale factors) with the engine's adjoint as backward"""

        @staticmethod
        def forward(ctx, x0, s):
            d = scaled(deck, x0.detach().cpu().numpy(), tuple(s.detach().cpu().numpy()))
            sysm = engine.System(d, precision=engine.PREC_FP64, refresh=1, noise=engine.NOISE_PHILOX, seed=SEED)
            loss, gx, gp = sysm.adjoint(K, CKPT, pairs, targets)
            sysm.close()
            # the engine's parameter gradient is taken at scale 1 of the scaled
            # deck: d loss / d s = (d loss / d s') / s
            ctx.save_for_backward(torch.from_numpy(gx), torch.from_numpy(gp) / s.detach())
            return torch.tensor(loss, dtype=torch.float64)

        @staticmethod
        def backward(ctx, g):
            gx, gp = ctx.saved_tensors
            return g * gx, g * gp

    x0 = torch.tensor(deck.coord[:, :3], dtype=torch.float64, requires_grad=True)
    s = torch.ones(4, dtype=torch.float64, requires_grad=True)
    loss = Trajectory.apply(x0, s)
    loss.backward()
    assert x0.grad is not None and s.grad is not None
    # a few components of the Jacobian by torch's own central differences
    sel = torch.zeros_like(x0)
    sel[5, 1] = 1.0
    sel[30, 2] = 1.0
    h = 1e-4
    for idx in [(5, 1), (30, 2)]:
        xp = x0.detach().clone()
        xm = x0.detach().clone()
        xp[idx] += h
        xm[idx] -= h
        fd = (Trajectory.apply(xp, s.detach()) - Trajectory.apply(xm, s.detach())).item() / (2 * h)
        assert abs(fd - x0.grad[idx].item()) <= 1e-4 * max(abs(fd), 1e-3 * x0.grad.abs().sum().item()), (idx, fd)
    s2 = torch.tensor([1.2, 1.0, 0.9, 1.1], dtype=torch.float64, requires_grad=True)
    Trajectory.apply(x0.detach(), s2).backward()
    for k in range(4):
        sp = s2.detach().clone()
        sm = s2.detach().clone()
        sp[k] += h
        sm[k] -= h
        fd = (Trajectory.apply(x0.detach(), sp) - Trajectory.apply(x0.detach(), sm)).item() / (2 * h)
        assert abs(fd - s2.grad[k].item()) <= 1e-4 * max(abs(fd), 1e-6), (k, fd, s2.grad[k].item())


# ---------------------------------------------------------------------------
# An FP64 reference gradient independent of the GPU: central differences of
# the oracle's forward pass (CPU, FP64), Richardson-extrapolated, fed the
# device noise stream restated below.

def philox_gauss(seed, stream, n3):
    """The engine's device Gaussians for one Philox stream index: Philox-
    4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) keyed by the seed on the
    counter (pair index, stream, 0x42444242), two 53-bit uniforms per call
    and the Box-Muller transform, as the engine's noise kernel defines them
    (numpy's log and trigonometric functions may differ from CUDA's in the
    last bit)."""
    m32 = np.uint64(0xFFFFFFFF)
    t = np.arange((n3 + 1) // 2, dtype=np.uint64)
    c0, c1 = t, np.full_like(t, np.uint64(stream) & m32)
    c2, c3 = np.full_like(t, np.uint64(stream) >> np.uint64(32)), np.full_like(t, np.uint64(0x42444242))
    k0, k1 = np.uint64(seed) & m32, (np.uint64(seed) >> np.uint64(32)) & m32
    for _ in range(10):
        p0, p1 = np.uint64(0xD2511F53) * c0, np.uint64(0xCD9E8D57) * c2
        c0, c1, c2, c3 = ((p1 >> np.uint64(32)) ^ c1 ^ k0, p1 & m32, (p0 >> np.uint64(32)) ^ c3 ^ k1, p0 & m32)
        k0, k1 = (k0 + np.uint64(0x9E3779B9)) & m32, (k1 + np.uint64(0xBB67AE85)) & m32
    two53 = 9007199254740992.0
    u0 = ((c0 >> np.uint64(5)).astype(np.float64) * 67108864.0 + (c1 >> np.uint64(6)).astype(np.float64) + 0.5) / two53
    u1 = ((c2 >> np.uint64(5)).astype(np.float64) * 67108864.0 + (c3 >> np.uint64(6)).astype(np.float64)) / two53
    r = np.sqrt(-2.0 * np.log(u0))
    g = np.empty(2 * len(t))
    g[0::2] = r * np.cos(2 * np.pi * u1)
    g[1::2] = r * np.sin(2 * np.pi * u1)
    return g[:n3]


def oracle_loss(deck, pairs, targets, gauss):
    import pyoracle
    traj, _, _ = pyoracle.Oracle(deck).run_steps(K, gauss)
    x = traj[-1][:, :3]
    r = np.linalg.norm(x[pairs[:, 1]] - x[pairs[:, 0]], axis=1)
    return float(np.mean((r - targets) ** 2))


def reference_gradient(deck, pairs, targets, gauss, h=2e-3):
    """d loss / d (x0, s) by central differences of the oracle at h and h/2,
    Richardson-extrapolated (truncation O(h^4))."""
    x0 = deck.coord[:, :3]

    def dd(f, h):
        return (f(h) - f(-h)) / (2 * h)

    gx = np.zeros(x0.shape)
    for i in range(deck.n):
        for a in range(3):
            def f(e, i=i, a=a):
                x = x0.copy()
                x[i, a] += e
                return oracle_loss(scaled(deck, x), pairs, targets, gauss)
            gx[i, a] = (4 * dd(f, h / 2) - dd(f, h)) / 3
    gp = np.zeros(4)
    for k in range(4):
        def f(e, k=k):
            s = [1.0] * 4
            s[k] += e
            return oracle_loss(scaled(deck, s=s), pairs, targets, gauss)
        gp[k] = (4 * dd(f, h / 2) - dd(f, h)) / 3
    return gx, gp


def test_philox_restatement_reproduces_device_noise(case):
    deck = case[0]
    n3 = 3 * deck.n
    s = engine.System(deck, precision=engine.PREC_FP64, refresh=1, noise=engine.NOISE_PHILOX, seed=SEED)
    s.step(2)
    xd = s.get_coord()
    s.close()
    h = engine.System(deck, precision=engine.PREC_FP64, refresh=1, noise=engine.NOISE_HOST)
    h.step(1, philox_gauss(SEED, 0, n3))
    h.step(1, philox_gauss(SEED, 1, n3))
    xh = h.get_coord()
    h.close()
    step = np.abs(xd[:, :3] - deck.coord[:, :3]).max()
    assert np.abs(xd - xh).max() <= 1e-12 * step


@pytest.fixture(scope="module")
def reference(case):
    deck, pairs, targets = case
    n3 = 3 * deck.n
    gauss = np.concatenate([philox_gauss(SEED, k, n3) for k in range(K)])
    loss = oracle_loss(deck, pairs, targets, gauss)
    gx, gp = reference_gradient(deck, pairs, targets, gauss)
    return loss, gx, gp


@pytest.mark.parametrize("prec,tol", [(engine.PREC_FP64, 1e-6), (engine.PREC_MIXED, 1e-4)])
def test_adjoint_matches_fp64_reference_gradient(case, reference, prec, tol):
    """The FP64 adjoint and the mixed-precision one (FP32 forward, FP32
    triangular solves) against the oracle's FP64 reference gradient: the
    position gradient within tol in norm, each scale-factor derivative
    within tol of its value."""
    deck, pairs, targets = case
    loss_ref, gx_ref, gp_ref = reference
    s = engine.System(deck, precision=prec, refresh=1, noise=engine.NOISE_PHILOX, seed=SEED)
    loss, gx, gp = s.adjoint(K, CKPT, pairs, targets)
    s.close()
    assert abs(loss - loss_ref) <= tol * loss_ref
    assert np.linalg.norm(gx - gx_ref) <= tol * np.linalg.norm(gx_ref), np.linalg.norm(gx - gx_ref) / np.linalg.norm(gx_ref)
    # (the LJ epsilon derivative is ~1e-3 of the others here: its error is
    # measured against that scale)
    for k in range(4):
        assert abs(gp[k] - gp_ref[k]) <= tol * max(abs(gp_ref[k]), 1e-3 * np.abs(gp_ref).max()), (k, gp[k], gp_ref[k])
