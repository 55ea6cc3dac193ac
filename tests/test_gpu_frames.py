"""Asynchronous trajectory frames (bdb_frames_*): the frames taken are the
positions after exactly the recorded steps, bit for bit, whether the steps
ran one per call or many per call, with graph replay; recording does not
change the trajectory; a ring smaller than the number of frames loses
none; IGT steps record too."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

from bd_box_b200 import decks, engine  # noqa: E402


@pytest.fixture(scope="module")
def chain(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("frames"))
    return decks.read_deck(decks.write_chain_deck(d, "fr", 90, seed=41, hydro="cholesky"))


def snapshots(deck, nsteps, **kw):
    s = engine.System(deck, **kw)
    out = [s.get_coord()]
    for _ in range(nsteps):
        s.step(1)
        out.append(s.get_coord())
    s.close()
    return out


def test_frames_match_trajectory(chain):
    kw = dict(precision=engine.PREC_MIXED, refresh=3, noise=engine.NOISE_PHILOX, seed=5)
    ref = snapshots(chain, 15, **kw)
    s = engine.System(chain, **kw)
    s.frames_start(every=3, capacity=2)          # 6 frames through a ring of 2
    for _ in range(10):
        s.step(1)
    s.step(5)                                     # steps 11..15 in one call
    assert s.frames_pending() == 6
    steps, times, coords, energies = s.frames_take(flush=True)
    assert energies is None
    assert steps.tolist() == [0, 3, 6, 9, 12, 15]
    t = 0.0
    acc = [0.0]
    for _ in range(15):
        t += chain.prm["dt"]
        acc.append(t)
    assert times.tolist() == [acc[k] for k in steps]
    for k, c in zip(steps, coords):
        assert np.array_equal(c, ref[k]), k
    # recording did not perturb the run
    assert np.array_equal(s.get_coord(), ref[15])
    assert s.frames_pending() == 0
    s.close()


def test_frames_take_in_parts_and_restart(chain):
    s = engine.System(chain, precision=engine.PREC_FP64, noise=engine.NOISE_PHILOX, seed=6)
    s.frames_start(every=1, capacity=8)
    s.step(4)
    a = s.frames_take(max_frames=2, flush=True)
    b = s.frames_take(flush=True)
    assert a[0].tolist() == [0, 1] and b[0].tolist() == [2, 3, 4]
    s.frames_start(every=2, capacity=4)          # a new ring from the current step
    s.step(4)
    c = s.frames_take(flush=True)
    assert c[0].tolist() == [4, 6, 8]
    s.frames_stop()
    with pytest.raises(engine.BDBError):
        s.frames_take()
    s.close()


def test_frames_igt(chain):
    kw = dict(precision=engine.PREC_FP64, noise=engine.NOISE_PHILOX, seed=7)
    r = engine.System(chain, **kw)
    ref = []
    for _ in range(4):
        r.step_igt(1)
        ref.append(r.get_coord())
    r.close()
    s = engine.System(chain, **kw)
    s.frames_start(every=2, capacity=4)
    s.step_igt(4)
    steps, _, coords, _ = s.frames_take(flush=True)
    assert steps.tolist() == [0, 2, 4]
    assert np.array_equal(coords[1], ref[1]) and np.array_equal(coords[2], ref[3])
    s.close()


def test_frames_with_energies(chain):
    """Energy frames: E of each saved state equals bdb_compute_forces' E at
    that state, and the extra energy pass leaves the trajectory unchanged."""
    kw = dict(precision=engine.PREC_MIXED, refresh=3, noise=engine.NOISE_PHILOX, seed=9)
    r = engine.System(chain, **kw)
    ref_x, ref_e = [r.get_coord()], [r.compute_forces()[1]]
    for _ in range(6):
        r.step(1)
        ref_x.append(r.get_coord())
        ref_e.append(r.compute_forces()[1])
    r.close()
    s = engine.System(chain, **kw)
    s.frames_start(every=2, capacity=2, energy=True)
    s.step(6)
    steps, _, coords, energies = s.frames_take(flush=True)
    assert steps.tolist() == [0, 2, 4, 6]
    for k, c, e in zip(steps, coords, energies):
        assert np.array_equal(c, ref_x[k]) and np.array_equal(e, ref_e[k]), k
    assert np.all(energies[:, [6, 7]] != 0)
    s.close()
