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
