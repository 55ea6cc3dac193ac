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
