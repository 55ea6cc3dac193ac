"""Parity at the benchmark workloads' own sizes against BD_BOX's CPU build
(oracle/_ref/ref_harness: the reference sources compiled with OpenMP and
LAPACK dpotrf/dsymv/dtrmv), on identical decks and identical Gaussians:

* a chain of 4096 beads (3N = 12288; the force field of the chain decks,
  bead radius 2 A), the tensor and its Cholesky factor rebuilt every 10
  steps (the reference's compute_D and LAPACK dpotrf on that schedule):
  3 steps. Mixed precision: every step within 1e-5 of the reference's
  displacement and the factor within 1e-5 (||L L^T - D|| / ||D||); FP64:
  within 1e-9 of a step.
* a chain of 512 beads, FP64, the tensor and the factor every step (BD_BOX's
  own schedule, compute_hydro): 5 steps within 1e-9 of a step.
* a periodic suspension of 4096 spheres at volume fraction 0.1
  (Beenakker-Ewald RPY) with the lattice sums over |m| <= R = 4
  (ewald_real = ewald_recip = 4), the smallest R whose D.F is within 1e-6
  of the R = 5 sums (the largest R BD_BOX accepts, input.c:402-409): R = 3
  is 7e-6 away, in BD_BOX's own sums as in ours. D.F against the
  reference's stored-tensor D.F (geyer_on_the_fly no), FP64 1e-11 and mixed
  1e-5; and, at 1024 spheres, the TEA noise against the reference's.

The reference runs take seconds to a minute on the host's cores.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

from bd_box_b200 import decks, engine  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")


def reference(d, prm, mode, *args):
    """Run the reference harness on deck `prm` in directory d with the
    Gaussians of d/g.bin; returns its float64 output."""
    if not os.path.exists(HARNESS):
        pytest.skip("oracle/_ref/ref_harness not built (make -C oracle ref needs the BD_BOX sources)")
    out = os.path.join(d, "out.bin")
    env = dict(os.environ, BDB_GAUSS_FILE=os.path.join(d, "g.bin"), OMP_NUM_THREADS=str(os.cpu_count() or 1))
    r = subprocess.run([HARNESS, os.path.basename(prm), mode, out, *args], cwd=d, env=env, capture_output=True,
                       text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    return np.fromfile(out)


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(b).max())


def step_errors(s, deck, g, traj, K):
    """Run K one-step calls with the reference's Gaussians; per step, the
    largest coordinate difference over the reference step's largest
    displacement."""
    n3 = 3 * deck.n
    prev = deck.coord
    errs = []
    for k in range(K):
        s.step(1, g[k * n3:(k + 1) * n3])
        x = s.get_coord()
        disp = np.abs(traj[k][:, :3] - prev[:, :3]).max()
        errs.append(float(np.abs(x[:, :3] - traj[k][:, :3]).max() / disp))
        prev = traj[k]
    return errs


@pytest.fixture(scope="module")
def chain4096(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("chain4096"))
    prm = decks.write_chain_deck(d, "c", 4096, seed=2, hydro="cholesky", steps=200)
    deck = decks.read_deck(prm)
    K = 3
    g = np.random.default_rng(2024).standard_normal(3 * deck.n * K)
    g.tofile(os.path.join(d, "g.bin"))
    traj = reference(d, prm, "steps", str(K), "10").reshape(K, deck.n, 4)
    return deck, g, traj, K


def test_chain4096_mixed_refresh10_matches_reference(chain4096):
    deck, g, traj, K = chain4096
    s = engine.System(deck, precision=engine.PREC_MIXED, refresh=10, noise=engine.NOISE_HOST)
    errs = step_errors(s, deck, g, traj, K)
    assert max(errs) <= 1e-5, errs
    fe = s.factor_error()
    assert fe <= 1e-5, fe
    s.close()


def test_chain4096_fp64_refresh10_matches_reference(chain4096):
    deck, g, traj, K = chain4096
    s = engine.System(deck, precision=engine.PREC_FP64, refresh=10, noise=engine.NOISE_HOST)
    errs = step_errors(s, deck, g, traj, K)
    assert max(errs) <= 1e-9, errs
    s.close()


def test_chain512_fp64_every_step_matches_reference(tmp_path):
    d = str(tmp_path)
    prm = decks.write_chain_deck(d, "c", 512, seed=1, hydro="cholesky")
    deck = decks.read_deck(prm)
    K = 5
    g = np.random.default_rng(2025).standard_normal(3 * deck.n * K)
    g.tofile(os.path.join(d, "g.bin"))
    traj = reference(d, prm, "steps", str(K)).reshape(K, deck.n, 4)
    s = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    errs = step_errors(s, deck, g, traj, K)
    assert max(errs) <= 1e-9, errs
    s.close()
    m = engine.System(deck, precision=engine.PREC_MIXED, noise=engine.NOISE_HOST)
    errs = step_errors(m, deck, g, traj, K)
    assert max(errs) <= 1e-5, errs
    m.close()


def suspension(d, n, R, seed=21):
    prm = decks.write_suspension_deck(d, f"s{R}", n, seed=seed, ewald_r=R, phi=0.1,
                                      extra={"geyer_on_the_fly": "no"})
    return prm, decks.read_deck(prm)


def test_suspension4096_df_matches_reference_and_R5(tmp_path):
    d = str(tmp_path)
    prm4, deck4 = suspension(d, 4096, 4)
    np.zeros(1).tofile(os.path.join(d, "g.bin"))
    ref = reference(d, prm4, "df")
    s = engine.System(deck4, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    s.compute_forces()
    df4 = s.compute_Rf()
    assert rel(df4, ref) <= 1e-11, rel(df4, ref)
    s.close()
    m = engine.System(deck4, precision=engine.PREC_MIXED, noise=engine.NOISE_HOST)
    m.compute_forces()
    assert rel(m.compute_Rf(), ref) <= 1e-5
    m.close()
    # the same spheres with the lattice sums over R = 3 and R = 5
    df = {}
    for R in (3, 5):
        _, deck = suspension(d, 4096, R)
        assert np.array_equal(deck.coord, deck4.coord)
        sr = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
        sr.compute_forces()
        df[R] = sr.compute_Rf()
        sr.close()
    assert rel(df4, df[5]) <= 1e-6, rel(df4, df[5])
    assert rel(df[3], df[5]) > 1e-6      # R = 3 does not reach 1e-6


def test_suspension1024_tea_matches_reference(tmp_path):
    d = str(tmp_path)
    prm, deck = suspension(d, 1024, 3)
    n3 = 3 * deck.n
    g = np.random.default_rng(2026).standard_normal(n3)
    g.tofile(os.path.join(d, "g.bin"))
    t = reference(d, prm, "tea")
    Rs_ref = t[:n3]
    s = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    Rs = s.compute_r(g)
    assert rel(Rs, Rs_ref) <= 1e-11, rel(Rs, Rs_ref)
    s.close()
    m = engine.System(deck, precision=engine.PREC_MIXED, noise=engine.NOISE_HOST)
    assert rel(m.compute_r(g), Rs_ref) <= 1e-5
    m.close()
