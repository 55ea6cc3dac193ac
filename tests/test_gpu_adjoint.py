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
