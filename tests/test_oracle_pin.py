"""Pin the oracle (C restatement in oracle/) to BD_BOX's own outputs.

The golden fixtures were produced by the reference's CPU sources
(tests/golden/make_golden.py); when the reference build is present the
same comparison also runs live on a fresh deck. The restatement follows
the reference's operation order, so D agrees bit for bit and the rest to
a few ulps (summation order of LAPACK vs the restated loops).
"""
import os
import subprocess

import numpy as np
import pytest

import golden_cases
import pyoracle
from bd_box_b200 import decks


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("name", golden_cases.names())
def test_oracle_matches_golden(name):
    deck, ref = golden_cases.load(name)
    o = pyoracle.Oracle(deck)
    n3 = 3 * deck.n
    assert np.array_equal(o.D(), ref["D"]) or rel(o.D(), ref["D"]) < 1e-15
    F, E, rep, counts = o.forces()
    assert rel(F, ref["F"]) < 1e-13
    for k in range(1, 8):
        if abs(ref["E"][k]) > 0:
            assert abs(E[k] - ref["E"][k]) <= 1e-10 * abs(ref["E"][k]) + 1e-12, (k, E[k], ref["E"][k])
    assert rep == int(ref["rep"])
    assert counts == (int(ref["counts"][0]), int(ref["counts"][1]))
    # the reference's own cell list (bucket_space) finds the same pairs
    assert (int(ref["counts"][2]), int(ref["counts"][3])) == counts
    Dst = o.D() if deck.prm["hydro"] == 1 or not deck.prm["geyer_on_the_fly"] else None
    if deck.prm["hydro"] == 2 and not deck.prm["geyer_on_the_fly"]:
        Dst = o.D()
    assert rel(o.df(F, deck.prm["dt"], Dst if deck.prm["hydro"] else None), ref["Rf"]) < 1e-13
    if "tea_Rs" in ref:
        Rs, eps, beta = o.tea(ref["gauss"][:n3], deck.prm["dt"], Dst if deck.prm["hydro"] == 2 and Dst is not None else None)
        assert rel(Rs, ref["tea_Rs"]) < 1e-13
        assert abs(eps - float(ref["tea_eps"])) <= 1e-13 * abs(eps)
    if deck.prm["algorithm"] >= decks.ALGORITHM["igt_const"]:
        traj, _, _ = pyoracle.Oracle(deck).run_igt_steps(ref["traj"].shape[0], ref["gauss"])
    else:
        traj, _, _ = o.run_steps(ref["traj"].shape[0], ref["gauss"])
    disp = np.abs(ref["traj"][0, :, :3] - deck.coord[:, :3]).max()
    assert np.abs(traj - ref["traj"]).max() <= 1e-9 * disp


def test_bonded_fixture_exercises_every_term():
    deck, ref = golden_cases.load("chain24_bonded")
    assert len(deck.angle_pairs) and len(deck.angle_cos_pairs) and len(deck.dihe_angle_pairs)
    # bonds start at their rest length r0, so the bond term enters through
    # the trajectory; angles, cosine angles, harmonic dihedrals, LJ and
    # Debye-Hueckel all contribute at the start
    assert all(abs(ref["E"][k]) > 0 for k in (2, 3, 5, 6, 7))


HARNESS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "ref_harness")


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="reference build (oracle/_ref) not present")
def test_oracle_matches_reference_live(tmp_path):
    p = decks.write_chain_deck(str(tmp_path), "live", 50, seed=77, hydro="geyer")
    deck = decks.read_deck(p)
    n3 = 3 * deck.n
    g = np.random.default_rng(1).standard_normal(2 * n3)
    g.tofile(tmp_path / "g.bin")
    env = dict(os.environ, BDB_GAUSS_FILE=str(tmp_path / "g.bin"), OMP_NUM_THREADS="1")
    subprocess.run([HARNESS, "live.prm", "steps", "out.bin", "2"], cwd=tmp_path, env=env, check=True,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    ref = np.fromfile(tmp_path / "out.bin").reshape(2, deck.n, 4)
    traj, _, _ = pyoracle.Oracle(deck).run_steps(2, g)
    assert np.abs(traj - ref).max() < 1e-12


def test_oracle_detects_a_planted_error():
    """A wrong tile (planted in the oracle's input, on the CPU) is caught."""
    deck, ref = golden_cases.load("chain32_chol")
    deck.coord[3, 3] *= 1.0001   # perturb one hydrodynamic radius
    assert rel(pyoracle.Oracle(deck).D(), ref["D"]) > 1e-8


EXT_DECKS = {
    # time-dependent RF field on the charges (cos on x, sin on z)
    "rf": dict(E_ext="yes", E_type="RF", E_freq=3.0, E_magn=0.7, E_factor=1.3, E_dir1="x", E_dir2="z"),
    # AC field on y without hydrodynamic interactions
    "ac": dict(E_ext="yes", E_type="AC", E_freq=5.0, E_magn=0.4, E_dir1="y"),
    # bounding sphere: bc sphere with the wall force on beads beyond 6 A
    "sphere": dict(bc="sphere", sphere_radius=40.0, sboundary="yes", sboundary_A=50.0, sboundary_n=2,
                   sboundary_cutoff=6.0),
}


def ext_deck(tmp_path, name, n=24, hydro="geyer"):
    extra = dict(EXT_DECKS[name])
    return decks.write_chain_deck(str(tmp_path), name, n, seed=91, hydro=hydro if name != "ac" else "none",
                                  extra=extra)


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("name", sorted(EXT_DECKS))
def test_oracle_external_forces_match_reference(tmp_path, name):
    """Electric field (DC/AC/RF at the step's force time) and bounding-sphere
    forces: the oracle's forces at the start and three steps against BD_BOX's
    own compute_forces / compute_hydro run by the harness."""
    p = ext_deck(tmp_path, name)
    deck = decks.read_deck(p)
    n3 = 3 * deck.n
    g = np.random.default_rng(2).standard_normal(4 * n3)
    g.tofile(tmp_path / "g.bin")
    env = dict(os.environ, BDB_GAUSS_FILE=str(tmp_path / "g.bin"), OMP_NUM_THREADS="1")
    prm = os.path.basename(p)
    subprocess.run([HARNESS, prm, "forces", "f.bin"], cwd=tmp_path, env=env, check=True,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    ref = np.fromfile(tmp_path / "f.bin")
    F, E, rep, _ = pyoracle.Oracle(deck).forces()
    assert rel(F, ref[:n3]) < 1e-13 and rep == int(ref[n3 + 9])
    subprocess.run([HARNESS, prm, "steps", "s.bin", "3"], cwd=tmp_path, env=env, check=True,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    traj_ref = np.fromfile(tmp_path / "s.bin").reshape(3, deck.n, 4)
    traj, _, _ = pyoracle.Oracle(deck).run_steps(3, g)
    assert np.abs(traj - traj_ref).max() < 1e-11
    # the external term is not negligible: without it the trajectory differs
    off = decks.read_deck(p, overrides={"E_ext": "no", "sboundary": "no"})
    traj_off, _, _ = pyoracle.Oracle(off).run_steps(3, g)
    assert np.abs(traj_off - traj_ref).max() > 1e-6


def newton_deck(tmp_path, hydro="none"):
    """A dense periodic suspension whose large moves overlap: ermak_newton
    resolves them by elastic collisions. (TEA with the stored tensor: BD_BOX's
    on-the-fly Ewald TEA differs, see test_reference_on_the_fly_ewald_tea.)"""
    return decks.write_suspension_deck(str(tmp_path), f"nw_{hydro}", 40, seed=5, phi=0.3, dt=0.2,
                                       extra=dict(algorithm="ermak_newton", check_overlap="yes", hydro=hydro,
                                                  geyer_on_the_fly="no"))


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("hydro", ["none", "geyer"])
def test_oracle_newton_matches_reference(tmp_path, hydro):
    """comp_step_ermak_newton with elastic collisions (newton.c): the
    oracle's steps against BD_BOX's own run by the harness, with the same
    Gaussian stream (one block per attempt)."""
    p = newton_deck(tmp_path, hydro)
    deck = decks.read_deck(p)
    n3 = 3 * deck.n
    g = np.random.default_rng(4).standard_normal(40 * n3)
    g.tofile(tmp_path / "g.bin")
    env = dict(os.environ, BDB_GAUSS_FILE=str(tmp_path / "g.bin"), OMP_NUM_THREADS="1")
    subprocess.run([HARNESS, os.path.basename(p), "steps", "s.bin", "4"], cwd=tmp_path, env=env, check=True,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    ref = np.fromfile(tmp_path / "s.bin").reshape(4, deck.n, 4)
    traj, _, rc, used, rounds = pyoracle.Oracle(deck).run_newton_steps(4, g)
    assert rc == 0 and used >= 4 and rounds > 4      # collisions happened
    assert np.abs(traj - ref).max() < 1e-10


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("method", ["beenakker", "smith"])
def test_reference_on_the_fly_ewald_tea(tmp_path, method):
    """A documented difference. BD_BOX's on-the-fly TEA (diff_rand.c:100-136)
    zeroes the tile once per bead i and calls compute_Dij(i, k) for k < i;
    the Ewald tile functions add into their output (diff_tensor.c:265-422
    and :102-263 use +=), so bead pair (i, k) gets the sum of the tiles
    (i, 0..k). Its epsilon is exactly that of the accumulated tiles, and
    differs from its own stored-tensor TEA (geyer_on_the_fly no), which the
    oracle and this library compute for both settings."""
    p = decks.write_suspension_deck(str(tmp_path), "tt", 24, seed=5, phi=0.1, dt=0.005,
                                    extra=dict(geyer_on_the_fly="yes", ewald_method=method))
    deck = decks.read_deck(p)
    n, n3 = deck.n, 3 * deck.n
    g = np.random.default_rng(4).standard_normal(n3)
    g.tofile(tmp_path / "g.bin")
    env = dict(os.environ, BDB_GAUSS_FILE=str(tmp_path / "g.bin"), OMP_NUM_THREADS="1")

    def ref_tea(prm):
        subprocess.run([HARNESS, prm, "tea", "t.bin"], cwd=tmp_path, env=env, check=True,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        return np.fromfile(tmp_path / "t.bin")

    o = pyoracle.Oracle(deck)
    acc = plain = 0.0
    for i in range(n):
        A = np.zeros((3, 3))
        for k in range(i):
            T = o.tile(i, k)
            A = A + T
            acc += A.sum()
            plain += T.sum()
    norm = 2.0 / n3 / (n3 - 1)
    eps_fly = ref_tea("tt.prm")[-1]
    assert abs(eps_fly - acc * norm) <= 1e-12 * abs(eps_fly)
    assert abs(eps_fly - plain * norm) > 0.1 * abs(eps_fly)
    # the stored-tensor TEA of BD_BOX is the oracle's (for both settings)
    stored = decks.read_deck(p, overrides={"geyer_on_the_fly": "no"})
    with open(tmp_path / "tt.prm") as f:
        text = f.read().replace("geyer_on_the_fly yes", "geyer_on_the_fly no")
    (tmp_path / "ts.prm").write_text(text)
    t = ref_tea("ts.prm")
    Rs, eps, _ = pyoracle.Oracle(stored).tea(g, deck.prm["dt"], pyoracle.Oracle(stored).D())
    assert abs(eps - t[-1]) <= 1e-12 * abs(eps)
    assert rel(Rs, t[:n3]) < 1e-12
    Rs_fly, eps2, _ = pyoracle.Oracle(deck).tea(g, deck.prm["dt"])
    assert abs(eps2 - eps) <= 1e-12 * abs(eps) and rel(Rs_fly, Rs) < 1e-12


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("hydro", ["none", "cholesky"])
def test_oracle_shear_flow_matches_reference(tmp_path, hydro):
    """A flowing solvent (vel_grad_tensor): each Ermak step adds dt G r
    (diff_equation.c:265-283). Three steps of simple shear against BD_BOX's
    own run."""
    p = decks.write_chain_deck(str(tmp_path), "fl", 30, seed=23, hydro=hydro,
                               extra={"vel_grad_tensor": "0 0.75 0 0 0 0 0.1 0 0"})
    deck = decks.read_deck(p)
    n3 = 3 * deck.n
    g = np.random.default_rng(3).standard_normal(3 * n3)
    g.tofile(tmp_path / "g.bin")
    env = dict(os.environ, BDB_GAUSS_FILE=str(tmp_path / "g.bin"), OMP_NUM_THREADS="1")
    subprocess.run([HARNESS, "fl.prm", "steps", "s.bin", "3"], cwd=tmp_path, env=env, check=True,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    ref = np.fromfile(tmp_path / "s.bin").reshape(3, deck.n, 4)
    traj, _, _ = pyoracle.Oracle(deck).run_steps(3, g)
    assert np.abs(traj - ref).max() < 1e-11
    still = decks.read_deck(p, overrides={"vel_grad_tensor": "0 0 0 0 0 0 0 0 0"})
    traj0, _, _ = pyoracle.Oracle(still).run_steps(3, g)
    assert np.abs(traj0 - ref).max() > 1e-3


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("hydro", ["none", "cholesky"])
def test_oracle_igt_in_flow_matches_reference(tmp_path, hydro):
    """IGT predictor-corrector in a flowing solvent: the corrector adds half
    the predictor's flow displacement FS (diff_equation.c:275-311)."""
    p = decks.write_chain_deck(str(tmp_path), "fi", 30, seed=24, hydro=hydro,
                               extra={"vel_grad_tensor": "0 0.75 0 0 0 0 0.1 0 0", "algorithm": "igt_const"})
    deck = decks.read_deck(p)
    n3 = 3 * deck.n
    g = np.random.default_rng(5).standard_normal(6 * n3)
    g.tofile(tmp_path / "g.bin")
    env = dict(os.environ, BDB_GAUSS_FILE=str(tmp_path / "g.bin"), OMP_NUM_THREADS="1")
    subprocess.run([HARNESS, "fi.prm", "steps", "s.bin", "3"], cwd=tmp_path, env=env, check=True,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    ref = np.fromfile(tmp_path / "s.bin").reshape(3, deck.n, 4)
    traj, _, rep = pyoracle.Oracle(deck).run_igt_steps(3, g)
    assert rep == 0 and np.abs(traj - ref).max() < 1e-11


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="reference build (oracle/_ref) not present")
def test_oracle_newton_in_sphere_matches_reference(tmp_path):
    """ermak_newton inside a reflective sphere with the wall force (bc
    sphere, sboundary): the collision moves check that every bead stays in
    the sphere (iscorrect) and the wall pushes beads back; 4 steps against
    BD_BOX's own run."""
    p = decks.write_suspension_deck(str(tmp_path), "sp", 40, seed=5, phi=0.3, dt=0.2,
                                    extra=dict(algorithm="ermak_newton", check_overlap="yes", hydro="none",
                                               bc="sphere", sphere_radius=7.5, sboundary="yes", sboundary_A=5.0,
                                               sboundary_n=2, sboundary_cutoff=3.0))
    deck = decks.read_deck(p)
    n3 = 3 * deck.n
    g = np.random.default_rng(4).standard_normal(60 * n3)
    g.tofile(tmp_path / "g.bin")
    env = dict(os.environ, BDB_GAUSS_FILE=str(tmp_path / "g.bin"), OMP_NUM_THREADS="1")
    subprocess.run([HARNESS, "sp.prm", "steps", "s.bin", "4"], cwd=tmp_path, env=env, check=True,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    ref = np.fromfile(tmp_path / "s.bin").reshape(4, deck.n, 4)
    traj, _, rc, used, rounds = pyoracle.Oracle(deck).run_newton_steps(4, g)
    assert rc == 0 and rounds > 4
    assert np.abs(traj - ref).max() < 1e-10


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="reference build (oracle/_ref) not present")
def test_oracle_igt_with_time_dependent_field_matches_reference(tmp_path):
    """IGT steps under an RF field: both force passes of a step act at
    curr_time + curr_dt (diff_equation.c:314, 327)."""
    extra = dict(EXT_DECKS["rf"], algorithm="igt_const")
    p = decks.write_chain_deck(str(tmp_path), "rfi", 24, seed=91, hydro="cholesky", extra=extra)
    deck = decks.read_deck(p)
    n3 = 3 * deck.n
    g = np.random.default_rng(8).standard_normal(6 * n3)
    g.tofile(tmp_path / "g.bin")
    env = dict(os.environ, BDB_GAUSS_FILE=str(tmp_path / "g.bin"), OMP_NUM_THREADS="1")
    subprocess.run([HARNESS, "rfi.prm", "steps", "s.bin", "3"], cwd=tmp_path, env=env, check=True,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    ref = np.fromfile(tmp_path / "s.bin").reshape(3, deck.n, 4)
    traj, _, rep = pyoracle.Oracle(deck).run_igt_steps(3, g)
    assert rep == 0 and np.abs(traj - ref).max() < 1e-11
