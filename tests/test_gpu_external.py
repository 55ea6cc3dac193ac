"""External forces on the device (k_external): the electric field on charged
beads (DC, AC, RF at the force time of each step, also inside replayed step
graphs) and the bounding-sphere force of bc sphere, against the oracle's
restatement of electro_ext_force / sboundary_ext (pinned to BD_BOX by
tests/test_oracle_pin.py). FP64: forces to 1e-12, trajectories to 1e-9 of
a step, as the other parity tests."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

from bd_box_b200 import decks, engine  # noqa: E402
import pyoracle  # noqa: E402
from test_oracle_pin import EXT_DECKS, ext_deck  # noqa: E402


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("name", sorted(EXT_DECKS))
def test_external_forces_and_steps(tmp_path, name):
    deck = decks.read_deck(ext_deck(tmp_path, name))
    o = pyoracle.Oracle(deck)
    F_o, _, rep_o, _ = o.forces()
    s = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    F, _, rep, _ = s.compute_forces()
    assert rel(F, F_o) < 1e-12 and rep == rep_o
    K, n3 = 4, 3 * deck.n
    g = np.random.default_rng(17).standard_normal(K * n3)
    traj, _, _ = pyoracle.Oracle(deck).run_steps(K, g)
    prev = deck.coord
    for k in range(K):
        s.step(1, g[k * n3:(k + 1) * n3])     # replayed from the host-noise graph after the first
        x = s.get_coord()
        err = np.abs(x[:, :3] - traj[k][:, :3]).max() / np.abs(traj[k][:, :3] - prev[:, :3]).max()
        assert err < 1e-9, (k, err)
        prev = traj[k]
    t = 0.0
    for _ in range(K):
        t += deck.prm["dt"]
    assert s.get_time() == t
    s.close()


def test_rf_field_graph_replay_matches_eager(tmp_path):
    deck = decks.read_deck(ext_deck(tmp_path, "rf"))
    out = []
    for graphs in (3, 0):
        s = engine.System(deck, precision=engine.PREC_MIXED, refresh=2, noise=engine.NOISE_PHILOX, seed=4)
        s._check(s.lib.bdb_set_graphs(s.h, graphs))
        s.step(6)
        out.append(s.get_coord())
        s.close()
    assert np.array_equal(out[0], out[1])


def test_rf_field_igt_and_set_time(tmp_path):
    deck = decks.read_deck(ext_deck(tmp_path, "ac"))   # hydro none
    K, n3 = 3, 3 * deck.n
    g = np.random.default_rng(18).standard_normal(2 * K * n3)
    o = pyoracle.Oracle(deck)
    o.s.t = 0.25
    F0, _, _, _ = o.forces()
    traj, _, _ = o.run_igt_steps(K, g, F=F0)
    s = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    s.set_time(0.25)                                   # a host clock (e.g. a restart) sets the time
    prev = deck.coord
    for k in range(K):
        s.step_igt(1, g[2 * k * n3:2 * (k + 1) * n3])
        x = s.get_coord()
        err = np.abs(x[:, :3] - traj[k][:, :3]).max() / np.abs(traj[k][:, :3] - prev[:, :3]).max()
        assert err < 1e-9, (k, err)
        prev = traj[k]
    s.close()


@pytest.mark.parametrize("hydro", ["none", "cholesky"])
def test_shear_flow_steps(tmp_path, hydro):
    """A flowing solvent (vel_grad_tensor): Ermak and IGT steps against the
    oracle (pinned to BD_BOX)."""
    p = decks.write_chain_deck(str(tmp_path), "fl", 30, seed=23, hydro=hydro,
                               extra={"vel_grad_tensor": "0 0.75 0 0 0 0 0.1 0 0"})
    deck = decks.read_deck(p)
    K, n3 = 3, 3 * deck.n
    g = np.random.default_rng(3).standard_normal(K * n3)
    traj, _, _ = pyoracle.Oracle(deck).run_steps(K, g)
    s = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    prev = deck.coord
    for k in range(K):
        s.step(1, g[k * n3:(k + 1) * n3])
        x = s.get_coord()
        err = np.abs(x[:, :3] - traj[k][:, :3]).max() / np.abs(traj[k][:, :3] - prev[:, :3]).max()
        assert err < 1e-9, (k, err)
        prev = traj[k]
    s.close()
    # IGT in the flow: the corrector adds half the predictor's flow displacement
    pi = decks.write_chain_deck(str(tmp_path), "fi", 30, seed=24, hydro=hydro,
                                extra={"vel_grad_tensor": "0 0.75 0 0 0 0 0.1 0 0", "algorithm": "igt_const"})
    deck = decks.read_deck(pi)
    g = np.random.default_rng(5).standard_normal(2 * K * n3)
    traj, _, _ = pyoracle.Oracle(deck).run_igt_steps(K, g)
    s = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    prev = deck.coord
    for k in range(K):
        s.step_igt(1, g[2 * k * n3:2 * (k + 1) * n3])
        x = s.get_coord()
        err = np.abs(x[:, :3] - traj[k][:, :3]).max() / np.abs(traj[k][:, :3] - prev[:, :3]).max()
        assert err < 1e-9, ("igt", k, err)
        prev = traj[k]
    s.close()
