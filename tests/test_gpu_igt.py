"""IGT predictor-corrector steps (bdb_step_igt) against the oracle's
restatement of compute_hydro_IGT / compute_hydro_IGT_second_phase
(diff_equation.c:288-374) on the same host Gaussians: FP64 to 1e-9 of a
step, the mixed path to FP32 level; the corrector retry, and repeatable
device noise."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

from bd_box_b200 import decks, engine  # noqa: E402
import pyoracle  # noqa: E402


@pytest.fixture(scope="module")
def igt_decks(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("igt"))
    return {
        "chol": decks.read_deck(decks.write_chain_deck(d, "igt_chol", 80, seed=31, hydro="cholesky")),
        "none": decks.read_deck(decks.write_chain_deck(d, "igt_none", 60, seed=32, hydro="none")),
        # R=3 at phi=0.1: the truncated Ewald tensor is positive definite
        # (at R=2, phi=0.2 it is not, and no Cholesky path applies)
        "ewald": decks.read_deck(decks.write_suspension_deck(d, "igt_susp", 120, seed=33, ewald_r=3, phi=0.1,
                                                             extra={"hydro": "cholesky"})),
    }


def gauss(n3, k, seed):
    return np.random.default_rng(seed).standard_normal(2 * n3 * k)


@pytest.mark.parametrize("name", ["chol", "none", "ewald"])
def test_igt_fp64_matches_oracle(name, igt_decks):
    deck = igt_decks[name]
    K, n3 = 3, 3 * deck.n
    g = gauss(n3, K, seed=41)
    traj, _, rep = pyoracle.Oracle(deck).run_igt_steps(K, g)
    assert rep == 0
    s = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    prev = deck.coord
    for k in range(K):
        assert s.step_igt(1, g[2 * n3 * k:2 * n3 * (k + 1)]) == 0
        x = s.get_coord()
        disp = np.abs(traj[k][:, :3] - prev[:, :3]).max()
        err = np.abs(x[:, :3] - traj[k][:, :3]).max() / disp
        assert err < 1e-9, (k, err)
        prev = traj[k]
    s.close()


def test_igt_mixed_matches_oracle(igt_decks):
    deck = igt_decks["chol"]
    K, n3 = 3, 3 * deck.n
    g = gauss(n3, K, seed=42)
    traj, _, _ = pyoracle.Oracle(deck).run_igt_steps(K, g)
    s = engine.System(deck, precision=engine.PREC_MIXED, noise=engine.NOISE_HOST)
    prev = deck.coord
    for k in range(K):
        s.step_igt(1, g[2 * n3 * k:2 * n3 * (k + 1)])
        x = s.get_coord()
        err = np.linalg.norm(x[:, :3] - traj[k][:, :3]) / np.linalg.norm(traj[k][:, :3] - prev[:, :3])
        assert err <= 1e-5 * (k + 1), (k, err)
        prev = traj[k]
    s.close()


def test_igt_differs_from_ermak_at_second_order(igt_decks):
    """Without noise IGT is Heun's method on dr = D F dt/kT: one step differs
    from the Ermak (Euler) step by O(dt^2), far below the step itself."""
    deck = igt_decks["chol"]
    n3 = 3 * deck.n
    a = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    a.step_igt(1, np.zeros(2 * n3))
    b = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    b.step(1, np.zeros(n3))
    step = np.abs(b.get_coord()[:, :3] - deck.coord[:, :3]).max()
    diff = np.abs(a.get_coord()[:, :3] - b.get_coord()[:, :3]).max()
    assert 0 < diff < 1e-2 * step
    a.close()
    b.close()


def test_igt_corrector_retry(igt_decks):
    """The corrector again (comp_step_IGT_const's retry of the second phase)
    with new Gaussians: the oracle step with the same predictor Gaussians and
    the new corrector Gaussians."""
    deck = igt_decks["chol"]
    n3 = 3 * deck.n
    g = gauss(n3, 1, seed=43)
    g2 = np.random.default_rng(44).standard_normal(n3)
    s = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    s.step_igt(1, g)
    assert s.igt_corrector(g2) == 0
    # the same step in two calls, as a retrying caller makes it
    t = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    assert t.igt_predictor(g[:n3]) == 0
    assert t.igt_corrector(g[n3:]) == 0
    u = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    u.step_igt(1, g)
    assert np.array_equal(t.get_coord(), u.get_coord())
    t.close()
    u.close()
    traj, _, _ = pyoracle.Oracle(deck).run_igt_steps(1, np.concatenate([g[:n3], g2]))
    disp = np.abs(traj[0][:, :3] - deck.coord[:, :3]).max()
    assert np.abs(s.get_coord()[:, :3] - traj[0][:, :3]).max() / disp < 1e-9
    s.close()


def test_igt_device_noise_repeatable(igt_decks):
    deck = igt_decks["chol"]
    out = []
    for _ in range(2):
        s = engine.System(deck, precision=engine.PREC_MIXED, noise=engine.NOISE_PHILOX, seed=9)
        s.step_igt(3)
        out.append(s.get_coord())
        s.close()
    assert np.array_equal(out[0], out[1])
    assert not np.array_equal(out[0][:, :3], deck.coord[:, :3])


def test_igt_rejects_tea(tmp_path):
    deck = decks.read_deck(decks.write_chain_deck(str(tmp_path), "t", 30, seed=1, hydro="geyer"))
    s = engine.System(deck, noise=engine.NOISE_PHILOX)
    with pytest.raises(engine.BDBError):
        s.step_igt(1)
    s.close()


@pytest.mark.parametrize("restore", ["load_state", "set_coord", "checkpoint"])
def test_corrector_refused_after_a_restore(restore, igt_decks):
    """A predictor's corrector must not run after the state it belongs to
    was replaced: it would copy the predictor's start positions over the
    restored ones. Every restore cancels the pending predictor."""
    deck = igt_decks["chol"]
    n3 = 3 * deck.n
    g = gauss(n3, 1, seed=44)
    s = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    s.save_state()
    image = s.checkpoint()
    assert s.igt_predictor(g[:n3]) == 0
    if restore == "load_state":
        s.load_state()
    elif restore == "set_coord":
        s.set_coord(deck.coord)
    else:
        s.restore(image)
    with pytest.raises(engine.BDBError) as e:
        s.igt_corrector(g[n3:])
    assert e.value.code == -1
    # a new predictor re-arms the corrector
    assert s.igt_predictor(g[:n3]) == 0
    assert s.igt_corrector(g[n3:]) == 0
    s.close()
