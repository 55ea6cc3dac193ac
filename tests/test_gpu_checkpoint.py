"""Checkpoint and resume (bdb_checkpoint_*): a run resumed from an image
taken at the end of a refresh interval repeats the uninterrupted run (to
round-off: the resumed run rebuilds its cell lists), device noise included;
images of another bead count or of something else are refused."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

from bd_box_b200 import decks, engine  # noqa: E402


@pytest.mark.parametrize("hydro,precision", [("cholesky", engine.PREC_MIXED), ("geyer", engine.PREC_FP64)])
def test_resume_repeats_the_run(tmp_path, hydro, precision):
    deck = decks.read_deck(decks.write_chain_deck(str(tmp_path), f"ck_{hydro}", 120, seed=21, hydro=hydro))
    kw = dict(precision=precision, refresh=5, noise=engine.NOISE_PHILOX, seed=8)
    a = engine.System(deck, **kw)
    a.step(10)
    x10 = a.get_coord()
    img = a.checkpoint()
    a.step(10)
    xa = a.get_coord()
    b = engine.System(deck, **kw)
    b.restore(img)
    assert np.array_equal(b.get_coord(), x10)
    b.step(10)
    xb = b.get_coord()
    step = np.abs(xa[:, :3] - x10[:, :3]).max()
    assert np.abs(xb - xa).max() <= 1e-9 * step
    assert b.get_time() == a.get_time()
    a.close()
    b.close()


def test_foreign_images_are_refused(tmp_path):
    d1 = decks.read_deck(decks.write_chain_deck(str(tmp_path), "c1", 40, seed=1, hydro="none"))
    d2 = decks.read_deck(decks.write_chain_deck(str(tmp_path), "c2", 41, seed=1, hydro="none"))
    s1, s2 = engine.System(d1), engine.System(d2)
    img = s1.checkpoint()
    with pytest.raises(engine.BDBError):
        s2.restore(img)
    with pytest.raises(engine.BDBError):
        s1.restore(b"\0" * len(img))
    s1.close()
    s2.close()
