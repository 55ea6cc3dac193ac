"""Device-noise steps replay a captured CUDA graph of the steady part of a
step, and mixed-precision refreshes of D and its factor replay a second one.
Every graph mode must give the eager run's bits, across refreshes of the
stored tensor and across a change of the time step (which rebuilds the
graphs)."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

from bd_box_b200 import decks, engine  # noqa: E402


@pytest.mark.parametrize("hydro,precision,refresh", [("cholesky", engine.PREC_MIXED, 3),
                                                     ("cholesky", engine.PREC_FP64, 1),
                                                     ("geyer", engine.PREC_MIXED, 1)])
def test_graph_replay_matches_eager(hydro, precision, refresh, deck_dir):
    deck = decks.read_deck(decks.write_chain_deck(deck_dir, f"g_{hydro}{precision}", 160, seed=31, hydro=hydro))
    runs = []
    for graphs in (3, 2, 1, 0):
        s = engine.System(deck, precision=precision, refresh=refresh, noise=engine.NOISE_PHILOX, seed=77)
        s._check(s.lib.bdb_set_graphs(s.h, graphs))
        out = []
        for k in range(7):
            s.step(1)
            out.append(s.get_coord())
        s._check(s.lib.bdb_set_dt(s.h, deck.prm["dt"] / 2))
        s.step(2)
        out.append(s.get_coord())
        runs.append((np.array(out), s.launches()))
        s.close()
    a, la = runs[-1]
    for b, lb in runs[:-1]:
        assert np.array_equal(a, b)
        assert la == lb
    # the noise changes from step to step (the device counter advances)
    d1 = a[1, :, :3] - a[0, :, :3]
    d2 = a[2, :, :3] - a[1, :, :3]
    assert not np.allclose(d1, d2)


@pytest.mark.parametrize("hydro,precision,refresh", [("cholesky", engine.PREC_MIXED, 3),
                                                     ("geyer", engine.PREC_FP64, 1)])
def test_host_noise_graph_matches_eager(hydro, precision, refresh, deck_dir):
    """Steps with caller Gaussians replay their own graph (one-step calls,
    multi-step calls that stage several steps' Gaussians at once, and a time
    step change in between) and give the eager run's bits."""
    deck = decks.read_deck(decks.write_chain_deck(deck_dir, f"gh_{hydro}{precision}", 120, seed=32, hydro=hydro))
    n3 = 3 * deck.n
    g = np.random.default_rng(8).standard_normal(12 * n3)
    runs = []
    for graphs in (1, 0):
        s = engine.System(deck, precision=precision, refresh=refresh, noise=engine.NOISE_HOST)
        s._check(s.lib.bdb_set_graphs(s.h, graphs))
        out = []
        for k in range(5):
            s.step(1, g[k * n3:(k + 1) * n3])
            out.append(s.get_coord())
        s.step(3, g[5 * n3:8 * n3])
        out.append(s.get_coord())
        s._check(s.lib.bdb_set_dt(s.h, deck.prm["dt"] / 2))
        s.step(1, g[8 * n3:9 * n3])
        s.step(3, g[9 * n3:12 * n3])
        out.append(s.get_coord())
        runs.append(np.array(out))
        s.close()
    assert np.array_equal(runs[0], runs[1])
