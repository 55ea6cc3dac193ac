"""Fault paths, each made on the host: a bounded device wait that gives up
(the wait limit set to 0, so no wait ever succeeds: the kernels report a
time-out and the context stays usable), a tensor that is not positive
definite (BD_BOX's "Cholesky decomposition error", diff_rand.c:78-79, an
error code here), and the recovery of a system after each."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

from bd_box_b200 import decks, engine  # noqa: E402
import pyoracle  # noqa: E402

ERR_NOT_SPD, ERR_TIMEOUT = -3, -7


@pytest.mark.parametrize("prec", [engine.PREC_MIXED, engine.PREC_FP64])
def test_wait_time_out_is_reported_and_recovered(prec, deck_dir):
    """Every bounded wait of the tensor-core Cholesky, its diagonal-block
    kernel and the TMA-fed product gives up at once: the step reports
    BDB_ERR_TIMEOUT; with the limit restored, a restored state steps as a
    fresh system does."""
    deck = decks.read_deck(decks.write_chain_deck(deck_dir, f"to{prec}", 300, seed=61, hydro="cholesky"))
    g = np.random.default_rng(9).standard_normal(2 * 3 * deck.n)
    s = engine.System(deck, precision=prec, noise=engine.NOISE_HOST)
    s.step(1, g[:3 * deck.n])
    s.save_state()
    s.set_wait_limit(0)
    with pytest.raises(engine.BDBError) as e:
        s.refresh(1)
    assert e.value.code == ERR_TIMEOUT
    with pytest.raises(engine.BDBError) as e:
        s.step(1, g[3 * deck.n:])
    assert e.value.code == ERR_TIMEOUT
    s.set_wait_limit(-1)
    s.load_state()
    assert s.step(1, g[3 * deck.n:]) == 0
    x = s.get_coord()
    s.close()
    # the same two steps on a system that never timed out
    f = engine.System(deck, precision=prec, noise=engine.NOISE_HOST)
    f.step(1, g[:3 * deck.n])
    f.step(1, g[3 * deck.n:])
    xf = f.get_coord()
    f.close()
    step = np.abs(xf[:, :3] - deck.coord[:, :3]).max()
    assert np.abs(x[:, :3] - xf[:, :3]).max() <= 1e-12 * step


@pytest.mark.parametrize("prec", [engine.PREC_FP64, engine.PREC_MIXED])
def test_indefinite_tensor_is_not_spd(prec, deck_dir):
    """A dense periodic suspension with the Ewald sums cut at R = 2 has an
    indefinite truncated tensor (smallest eigenvalue about -0.02 here): the
    oracle's Cholesky (myblas.c's dpotrf semantics) fails, and so does the
    engine's, with BDB_ERR_NOT_SPD; a deck the Cholesky accepts then steps
    normally on the same process."""
    deck = decks.read_deck(decks.write_suspension_deck(deck_dir, f"ind{prec}", 120, seed=33, ewald_r=2, phi=0.2,
                                                       extra={"hydro": "cholesky"}))
    o = pyoracle.Oracle(deck)
    with pytest.raises(np.linalg.LinAlgError):
        o.cholesky(o.D())
    s = engine.System(deck, precision=prec, noise=engine.NOISE_HOST)
    with pytest.raises(engine.BDBError) as e:
        s.step(1, np.zeros(3 * deck.n))
    assert e.value.code == ERR_NOT_SPD
    s.close()
    ok = decks.read_deck(decks.write_suspension_deck(deck_dir, f"pd{prec}", 120, seed=33, ewald_r=3, phi=0.1,
                                                     extra={"hydro": "cholesky"}))
    t = engine.System(ok, precision=prec, noise=engine.NOISE_HOST)
    assert t.step(1, np.random.default_rng(2).standard_normal(3 * ok.n)) in (0, 1)
    t.close()
