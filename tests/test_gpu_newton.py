"""Elastic-collision overlap removal (bdb_newton_resolve, the
comp_step_ermak_newton recovery) against the oracle's restatement of
newton.c, which is pinned to BD_BOX by tests/test_oracle_pin.py: the same
Gaussian blocks per attempt, the same number of attempts and collision
rounds, and the trajectory to 1e-9 of the step."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

from bd_box_b200 import decks, engine  # noqa: E402
import pyoracle  # noqa: E402
from test_oracle_pin import newton_deck  # noqa: E402


@pytest.mark.parametrize("hydro", ["none", "geyer"])
def test_newton_steps_match_oracle(tmp_path, hydro):
    deck = decks.read_deck(newton_deck(tmp_path, hydro))
    n3 = 3 * deck.n
    K = 4
    g = np.random.default_rng(4).standard_normal(40 * n3)
    traj, _, rc, used_o, rounds_o = pyoracle.Oracle(deck).run_newton_steps(K, g)
    assert rc == 0 and rounds_o > K
    s = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    s.compute_forces()
    prev = deck.coord
    used, rounds = 0, 0
    for k in range(K):
        u, r = s.step_newton(1, g[used * n3:])
        used += u
        rounds += r
        x = s.get_coord()
        step = np.abs(traj[k][:, :3] - prev[:, :3]).max()
        assert np.abs(x[:, :3] - traj[k][:, :3]).max() < 1e-9 * step, k
        prev = traj[k]
    assert (used, rounds) == (used_o, rounds_o)
    s.close()
