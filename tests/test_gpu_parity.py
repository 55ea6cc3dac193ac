"""Parity of the CUDA path (libbdb200.so via its C ABI) with the oracle.

The oracle is the C restatement in oracle/ (pinned to the compiled
reference by tests/test_oracle_pin.py). Sizes are small enough for the
oracle to finish in seconds. Tolerances:
  * pair counts: bit-exact;
  * FP64 path: relative 1e-12 on forces, D, D.F, Rs and trajectories
    (libm vs CUDA transcendentals and summation order differ at ~1e-16);
  * Ewald tiles (CUDA erfc/exp/cos): relative 1e-11;
  * mixed path: ||B B^T - D||/||D|| <= 1e-5 and per-step displacement error
    <= 1e-5 relative to the FP64 oracle, the stated bounds of the method.
"""
import os

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

from bd_box_b200 import decks, engine  # noqa: E402
import pyoracle  # noqa: E402


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def chain_chol(deck_dir):
    p = decks.write_chain_deck(deck_dir, "chain_chol", 96, seed=11, hydro="cholesky", steps=5)
    return decks.read_deck(p)


@pytest.fixture(scope="module")
def chain_tea(deck_dir):
    p = decks.write_chain_deck(deck_dir, "chain_tea", 150, seed=12, hydro="geyer", steps=5)
    return decks.read_deck(p)


@pytest.fixture(scope="module")
def chain_none(deck_dir):
    p = decks.write_chain_deck(deck_dir, "chain_none", 70, seed=13, hydro="none", steps=5)
    return decks.read_deck(p)


@pytest.fixture(scope="module")
def susp(deck_dir):
    p = decks.write_suspension_deck(deck_dir, "susp", 160, seed=14, ewald_r=2, phi=0.2)
    return decks.read_deck(p)


def gauss(n3, k, seed=5):
    return np.random.default_rng(seed).standard_normal(k * n3)


@pytest.mark.parametrize("name", ["chain_chol", "chain_tea", "susp"])
def test_forces_and_pair_counts(name, request):
    deck = request.getfixturevalue(name)
    o = pyoracle.Oracle(deck)
    Fo, Eo, repo, co = o.forces()
    s = engine.System(deck)
    F, E, rep, c = s.compute_forces()
    assert c == co, "pair counts must be bit-exact"
    assert rep == repo
    assert rel(F, Fo) < 1e-12
    for k in (1, 6, 7):
        if abs(Eo[k]) > 1e-12:
            assert abs(E[k] - Eo[k]) / abs(Eo[k]) < 1e-10, k


@pytest.mark.parametrize("name", ["chain_chol", "susp"])
def test_diffusion_tensor(name, request):
    deck = request.getfixturevalue(name)
    o = pyoracle.Oracle(deck)
    Do = o.D()
    s = engine.System(deck, precision=engine.PREC_FP64)
    D = s.compute_D()
    tol = 1e-11 if deck.ewald else 1e-13
    assert rel(D, Do) < tol
    assert np.allclose(s.compute_Dij(3, 1), o.tile(3, 1), rtol=tol, atol=tol * abs(Do).max())
    sm = engine.System(deck, precision=engine.PREC_MIXED)
    assert rel(sm.compute_D(), Do) < 1e-6


def test_cholesky_noise_fp64(chain_chol):
    o = pyoracle.Oracle(chain_chol)
    n3 = 3 * chain_chol.n
    s = engine.System(chain_chol, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    assert s.factor_error() < 1e-14
    g = gauss(n3, 1)
    Rs = s.compute_r(g)
    L = o.cholesky(o.D())
    Rs_o = L @ (g * np.sqrt(2 * chain_chol.prm["dt"]))
    assert rel(Rs, Rs_o) < 1e-12


def test_cholesky_mixed_error(chain_chol):
    s = engine.System(chain_chol, precision=engine.PREC_MIXED)
    err = s.factor_error()
    assert err <= 1e-5, err


@pytest.mark.parametrize("n", [5, 22, 43, 96, 171])
def test_stored_products_mixed_ragged(n, deck_dir):
    """The FP32-matrix products (Rf = pre D F from the upper triangle and
    its transpose, Rs = L X from the lower) at sizes whose 3N cuts the
    64-row strips and 128-column tiles raggedly: Rf against the same FP32
    tensor multiplied in FP64 by the oracle (only the summation order
    differs), Rs against the FP64 factor within the mixed factor's bound."""
    deck = decks.read_deck(decks.write_chain_deck(deck_dir, f"rag{n}", n, seed=60 + n, hydro="cholesky"))
    o = pyoracle.Oracle(deck)
    n3 = 3 * n
    dt = deck.prm["dt"]
    s = engine.System(deck, precision=engine.PREC_MIXED, noise=engine.NOISE_HOST)
    D32 = s.compute_D()
    up = np.triu(D32, 1)
    Dsym = up + up.T + np.diag(np.diag(D32))
    F, _, _, _ = o.forces()
    assert rel(s.compute_Rf(), o.df(F, dt, Dsym)) < 1e-11
    g = gauss(n3, 1, seed=n)
    L = o.cholesky(o.D())
    assert rel(s.compute_r(g), L @ (g * np.sqrt(2 * dt))) < 2e-5


@pytest.mark.parametrize("name", ["chain_chol", "chain_tea", "chain_none", "susp"])
def test_df(name, request):
    deck = request.getfixturevalue(name)
    o = pyoracle.Oracle(deck)
    F, _, _, _ = o.forces()
    dt = deck.prm["dt"]
    Rf_o = o.df(F, dt, o.D() if deck.prm["hydro"] == 1 else None)
    s = engine.System(deck)
    Rf = s.compute_Rf()
    assert rel(Rf, Rf_o) < (1e-11 if deck.ewald else 1e-12)


@pytest.mark.parametrize("name", ["chain_tea", "susp"])
def test_tea_noise(name, request):
    deck = request.getfixturevalue(name)
    o = pyoracle.Oracle(deck)
    n3 = 3 * deck.n
    g = gauss(n3, 1, seed=7)
    Rs_o, eps_o, beta_o = o.tea(g, deck.prm["dt"])
    s = engine.System(deck, noise=engine.NOISE_HOST)
    Rs = s.compute_r(g)
    assert rel(Rs, Rs_o) < (1e-11 if deck.ewald else 1e-12)


@pytest.mark.parametrize("name,refresh", [("chain_chol", 1), ("chain_chol", 3), ("chain_tea", 1),
                                          ("chain_none", 1), ("susp", 1)])
def test_trajectory_fp64(name, refresh, request):
    deck = request.getfixturevalue(name)
    K = 4
    n3 = 3 * deck.n
    g = gauss(n3, K, seed=21)
    o = pyoracle.Oracle(deck)
    traj, _, _ = o.run_steps(K, g, refresh=refresh)
    s = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST, refresh=refresh)
    x0 = s.get_coord()
    for k in range(K):
        s.step(1, g[k * n3:(k + 1) * n3])
        x = s.get_coord()
        ref = traj[k]
        prev = traj[k - 1] if k else deck.coord
        disp_err = np.abs(x[:, :3] - ref[:, :3]).max() / np.abs(ref[:, :3] - prev[:, :3]).max()
        assert disp_err < 1e-9, (k, disp_err)
    assert x0.shape == (deck.n, 4)


def test_trajectory_mixed_chol(chain_chol):
    deck = chain_chol
    K = 3
    n3 = 3 * deck.n
    g = gauss(n3, K, seed=22)
    o = pyoracle.Oracle(deck)
    traj, _, _ = o.run_steps(K, g, refresh=10)
    s = engine.System(deck, precision=engine.PREC_MIXED, noise=engine.NOISE_HOST, refresh=10)
    prev = deck.coord
    for k in range(K):
        s.step(1, g[k * n3:(k + 1) * n3])
        x = s.get_coord()
        step_ref = traj[k][:, :3] - prev[:, :3]
        err = np.linalg.norm(x[:, :3] - traj[k][:, :3]) / np.linalg.norm(step_ref)
        assert err <= 1e-5 * (k + 1), (k, err)
        prev = traj[k]


def test_repeatable_bits(chain_tea):
    n3 = 3 * chain_tea.n
    out = []
    for _ in range(2):
        s = engine.System(chain_tea, seed=99)
        s.step(3)
        out.append(s.get_coord())
    assert np.array_equal(out[0], out[1])


def test_philox_moments(chain_none):
    s = engine.System(chain_none, seed=1234)
    n3 = 3 * chain_none.n
    d = chain_none.prm["dt"]
    diag = 1.0537375739171604e-4 * chain_none.prm["T"] / (chain_none.prm["visc"] * chain_none.prm["vfactor"]) / 2.0
    xs = np.concatenate([s.compute_r() / np.sqrt(2 * d * diag) for _ in range(200)])
    assert abs(xs.mean()) < 0.02
    assert abs(xs.var() - 1) < 0.03


def test_tensor_core_factor_large(deck_dir):
    """tcgen05 trailing updates on FP16 hi/lo panels over many tiles (3N =
    2100, 17 super panels): ||L L^T - D||/||D|| within the stated 1e-5, and
    of the order of the SIMT FP32 factor of the same matrix. The tensor-core
    factor carries more rounding than the SIMT one (5.1e-7 against 9.0e-8
    measured here): its FP32 accumulators in tensor memory sum 3 x 256
    products per pass over C (two panels at once) before one IEEE add into
    C, where the SIMT update rounds every FMA to nearest. A wrong or missing
    update gives errors of order 1, far above the factor of 10 allowed."""
    deck = decks.read_deck(decks.write_chain_deck(deck_dir, "big_chol", 700, seed=31, hydro="cholesky"))
    s = engine.System(deck, precision=engine.PREC_MIXED)
    err_tc = s.factor_error()
    os.environ["BDB_NO_TC"] = "1"
    try:
        err_simt = engine.System(deck, precision=engine.PREC_MIXED).factor_error()
    finally:
        del os.environ["BDB_NO_TC"]
    assert err_tc <= 1e-5, err_tc
    assert err_tc <= 10 * err_simt + 1e-7, (err_tc, err_simt)


@pytest.mark.parametrize("name", ["chain_tea", "susp"])
def test_tea_mixed_within_bound(name, request):
    """Mixed precision TEA (FP32 tiles; for Ewald FP32 real-space images and
    reciprocal phases, FP64 sums) against the FP64 oracle: D.F and the noise
    within the method's 1e-5 bound."""
    deck = request.getfixturevalue(name)
    o = pyoracle.Oracle(deck)
    n3 = 3 * deck.n
    F, _, _, _ = o.forces()
    Rf_o = o.df(F, deck.prm["dt"])
    g = gauss(n3, 1, seed=9)
    Rs_o, _, _ = o.tea(g, deck.prm["dt"])
    s = engine.System(deck, precision=engine.PREC_MIXED, noise=engine.NOISE_HOST)
    assert rel(s.compute_Rf(), Rf_o) < 1e-5
    assert rel(s.compute_r(g), Rs_o) < 1e-5


def test_smith_mixed_close_to_fp64(deck_dir):
    """Smith Ewald (diff_tensor.c:102-263) on a periodic suspension with TEA
    noise: the mixed path (FP64 Smith tiles, FP32 stored/TEA arithmetic)
    against FP64 on one step with the same noise."""
    p = decks.write_suspension_deck(deck_dir, "smith_mixed", 200, seed=15, ewald_r=2, phi=0.1,
                                    extra={"ewald_method": "smith"})
    deck = decks.read_deck(p)
    g = gauss(3 * deck.n, 1, seed=16)
    out = []
    for prec in (engine.PREC_FP64, engine.PREC_MIXED):
        s = engine.System(deck, precision=prec, noise=engine.NOISE_HOST)
        s.step(1, g)
        out.append(s.get_coord()[:, :3] - deck.coord[:, :3])
        s.close()
    box = deck.box[0]
    d64, dm = [d - box * np.round(d / box) for d in out]
    assert np.linalg.norm(dm - d64) / np.linalg.norm(d64) < 1e-5
