"""The autotuner's candidates: every TEA tile edge and every stored-matvec
segmentation must give the oracle's answers (they only regroup sums), and a
tuned system must pick one of them and keep stepping correctly."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

from bd_box_b200 import decks, engine  # noqa: E402


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def tea_deck(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("tune"))
    return decks.read_deck(decks.write_chain_deck(d, "t", 75, seed=12, hydro="geyer"))


@pytest.fixture(scope="module")
def chol_deck(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("tune_c"))
    return decks.read_deck(decks.write_chain_deck(d, "c", 300, seed=13, hydro="cholesky"))


@pytest.mark.parametrize("tile", [16, 32])
def test_tea_tile_candidates_match_oracle(tile, tea_deck):
    import pyoracle
    o = pyoracle.Oracle(tea_deck)
    n3 = 3 * tea_deck.n
    F, _, _, _ = o.forces()
    g = np.random.default_rng(4).standard_normal(n3)
    Rf_o = o.df(F, tea_deck.prm["dt"])
    Rs_o, _, _ = o.tea(g, tea_deck.prm["dt"])
    s = engine.System(tea_deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    s.set_tuning(tea_tile=tile)
    assert s.tuning()[0] == tile
    assert rel(s.compute_Rf(), Rf_o) < 1e-12
    assert rel(s.compute_r(g), Rs_o) < 1e-12


@pytest.mark.parametrize("warps", [8, 16, 32])
def test_matvec_segmentations_agree(warps, chol_deck):
    base = engine.System(chol_deck, precision=engine.PREC_FP64).compute_Rf()
    s = engine.System(chol_deck, precision=engine.PREC_FP64)
    s.set_tuning(mv_warps_per_sm=warps)
    assert rel(s.compute_Rf(), base) < 1e-13


def test_autotuned_batch_steps_like_untuned(tmp_path):
    ds = [decks.read_deck(decks.write_chain_deck(str(tmp_path), f"b{k}", n, seed=40 + k, hydro="geyer"))
          for k, n in enumerate((20, 70, 33, 90))]
    g = np.random.default_rng(5).standard_normal(3 * sum(d.n for d in ds))
    ref = engine.System(ds, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    ref.step(1, g)
    tuned = engine.System(ds, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    tuned.autotune(True)
    tuned.step(1, g)
    assert tuned.tuning()[0] in (16, 32)
    x0 = np.concatenate([d.coord for d in ds])
    disp = np.abs(ref.get_coord()[:, :3] - x0[:, :3]).max()
    assert np.abs(tuned.get_coord() - ref.get_coord()).max() <= 1e-12 * disp


def test_factor_split_candidates_give_identical_bits(deck_dir):
    """The mixed Cholesky's GPU split (SMs left to its panel chain) changes
    where the trailing updates run, not their order: every candidate gives
    the same factor and the same step, bit for bit; the autotuner picks one
    of them."""
    deck = decks.read_deck(decks.write_chain_deck(deck_dir, "fsplit", 700, seed=52, hydro="cholesky"))
    g = np.random.default_rng(8).standard_normal(3 * deck.n)
    ref = None
    for c in (16, 24, 32, 40, 48, 56, 64):
        s = engine.System(deck, precision=engine.PREC_MIXED, noise=engine.NOISE_HOST)
        s.set_factor_tuning(c)
        assert s.factor_tuning() == c
        s.step(1, g)
        out = (s.factor_error(), s.get_coord())
        s.close()
        if ref is None:
            ref = out
        else:
            # the error metric sums over blocks in arbitrary order; the
            # positions after the step are the bit-exact check
            assert abs(out[0] - ref[0]) <= 1e-12 * ref[0]
            assert np.array_equal(out[1], ref[1])
    s = engine.System(deck, precision=engine.PREC_MIXED, noise=engine.NOISE_HOST)
    s.autotune(True)
    s.step(1, g)
    assert s.factor_tuning() in (16, 24, 32, 40, 48, 56, 64)
    assert np.array_equal(s.get_coord(), ref[1])
    s.close()


def test_back_to_back_large_systems_factor_alike(deck_dir):
    """Systems created one after another in a warm process at 3N = 12288 (a
    600 MB stored matrix), each with another split: the clear of the matrix
    and the copies of a system's set-up are ordered on its own stream, so
    the tensor build (on the highest-priority stream) can never overtake
    them, and every system factors the same D to the same bits."""
    deck = decks.read_deck(decks.write_chain_deck(deck_dir, "b2b", 4096, seed=2, hydro="cholesky"))
    g = np.random.default_rng(9).standard_normal(3 * deck.n)
    ref = None
    for c in (16, 8, 32, 16):
        s = engine.System(deck, precision=engine.PREC_MIXED, refresh=10, noise=engine.NOISE_HOST)
        s.set_factor_tuning(c)
        s.refresh(1)
        fe = s.factor_error()
        r = s.compute_r(g)
        s.close()
        assert fe <= 1e-5, (c, fe)
        if ref is None:
            ref = r
        assert np.array_equal(r, ref), c
