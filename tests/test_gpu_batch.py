"""Batched replicas (bdb_create_batch): independent chains of uneven bead
counts advance together, every kernel covering all of them. Each replica must
follow the trajectory it has when run alone (and the oracle's), with the
same Gaussians."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

from bd_box_b200 import decks, engine  # noqa: E402

SIZES = (20, 37, 64, 50, 33)


def make_decks(d, hydro):
    return [decks.read_deck(decks.write_chain_deck(d, f"r{k}", n, seed=200 + k, hydro=hydro))
            for k, n in enumerate(SIZES)]


def run_alone(deck, gauss, K, precision=engine.PREC_FP64):
    s = engine.System(deck, precision=precision, noise=engine.NOISE_HOST)
    n3 = 3 * deck.n
    out = []
    for k in range(K):
        s.step(1, gauss[k * n3:(k + 1) * n3])
        out.append(s.get_coord())
    return out


@pytest.mark.parametrize("hydro", ["geyer", "none"])
def test_batch_matches_replicas_run_alone(hydro, deck_dir):
    ds = make_decks(deck_dir, hydro)
    K = 3
    rng = np.random.default_rng(5)
    g = [rng.standard_normal(3 * d.n * K) for d in ds]
    b = engine.System(ds, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    n3 = 3 * b.n
    trajs = []
    for k in range(K):
        gk = np.concatenate([gi[k * 3 * d.n:(k + 1) * 3 * d.n] for gi, d in zip(g, ds)])
        assert gk.size == n3
        b.step(1, gk)
        trajs.append(b.get_coord())
    for r, d in enumerate(ds):
        lo, hi = b.begins[r], b.begins[r] + d.n
        alone = run_alone(d, g[r], K)
        disp = np.abs(alone[0][:, :3] - d.coord[:, :3]).max()
        for k in range(K):
            err = np.abs(trajs[k][lo:hi] - alone[k]).max()
            assert err <= 1e-12 * disp, (r, k, err)


def test_batch_against_oracle_and_mixed(deck_dir):
    import pyoracle
    ds = make_decks(deck_dir, "geyer")
    K = 2
    rng = np.random.default_rng(9)
    g = [rng.standard_normal(3 * d.n * K) for d in ds]
    gk = [np.concatenate([gi[k * 3 * d.n:(k + 1) * 3 * d.n] for gi, d in zip(g, ds)]) for k in range(K)]
    b64 = engine.System(ds, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    bmx = engine.System(ds, precision=engine.PREC_MIXED, noise=engine.NOISE_HOST)
    x0 = b64.get_coord()
    for k in range(K):
        b64.step(1, gk[k])
        bmx.step(1, gk[k])
    t64, tmx = b64.get_coord(), bmx.get_coord()
    for r, d in enumerate(ds):
        lo, hi = b64.begins[r], b64.begins[r] + d.n
        traj, _, _ = pyoracle.Oracle(d).run_steps(K, g[r])
        disp = np.abs(traj[0][:, :3] - d.coord[:, :3]).max()
        assert np.abs(t64[lo:hi] - traj[-1]).max() <= 1e-9 * disp, r
        # mixed precision, per replica, against FP64 (whole displacement)
        dd = t64[lo:hi, :3] - x0[lo:hi, :3]
        dm = tmx[lo:hi, :3] - x0[lo:hi, :3]
        assert np.linalg.norm(dm - dd) / np.linalg.norm(dd) <= 1e-5, r


def test_batch_rejects_what_it_cannot_do(deck_dir):
    ds = make_decks(deck_dir, "cholesky")
    with pytest.raises(engine.BDBError) as e:
        engine.System(ds, precision=engine.PREC_FP64)
    assert e.value.args[0].startswith("bdb error -8")
    ds = make_decks(deck_dir, "geyer")
    b = engine.System(ds, precision=engine.PREC_FP64)
    with pytest.raises(engine.BDBError):
        b.compute_D()
    # a bond joining two replicas is refused
    import ctypes as C
    pairs = np.array([[0, ds[0].n]], dtype=np.int32)
    parms = np.array([[3.8, 1e10, 10.0]])
    rc = b.lib.bdb_set_bonded(b.h, 1, pairs.ctypes.data_as(C.POINTER(C.c_int)),
                              parms.ctypes.data_as(C.POINTER(C.c_double)), *([0, None, None] * 4))
    assert rc == -1
    # tiles between replicas are zero, within a replica they are the RPY tile
    assert not b.compute_Dij(0, ds[0].n).any()
    assert b.compute_Dij(0, 1).any()
