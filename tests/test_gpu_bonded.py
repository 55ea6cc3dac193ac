"""Bonded terms one type at a time (bonds, harmonic and cosine angles,
cosine and harmonic dihedrals) against the oracle, on perturbed
configurations of the golden chains; and the fault paths of the force pass,
made on the host: a NaN coordinate (the overlap flag, BD_BOX's retry
signal), an infinite coordinate (the free-space cell list must fall back to
pairs instead of growing its grid forever) and an over-stretched FENE bond
(BD_BOX's fatal error, bond.c:73-78, an error code here).

Tolerances: forces relative 1e-12 of the largest force, energies 1e-10.
"""
import copy

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

from bd_box_b200 import engine  # noqa: E402
import golden_cases  # noqa: E402
import pyoracle  # noqa: E402

KINDS = {"bond": 2, "angle": 3, "angle_cos": 3, "dihe": 4, "dihe_angle": 4}
E_INDEX = {"bond": 1, "angle": 2, "angle_cos": 3, "dihe": 4, "dihe_angle": 5}


def only(deck, kind, nonbonded=False):
    """The deck with one bonded term type and, unless asked, no
    non-bonded terms."""
    d = copy.deepcopy(deck)
    d.prm = dict(d.prm)
    if not nonbonded:
        d.prm["alpha_lj"] = 0.0
        d.prm["elec"] = 0
    for k, w in KINDS.items():
        if k != kind:
            setattr(d, k + "_pairs", np.zeros((0, w), np.int32))
            setattr(d, k + "_parms", np.zeros((0, 3 if k == "bond" else 2)))
    if kind == "bond":
        # r_max 20 A: the FENE energy is then well conditioned (at the
        # chains' r_max of 1e10 A it is a difference of nearly equal logs)
        d.bond_parms = d.bond_parms.copy()
        d.bond_parms[:, 1] = 20.0
    return d


def source(kind):
    return golden_cases.load("chain24_cosdihe" if kind == "dihe" else "chain24_bonded")[0]


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("kind", list(KINDS))
def test_each_bonded_term_matches_oracle(kind):
    deck = only(source(kind), kind)
    assert len(getattr(deck, kind + "_pairs")) > 0
    rng = np.random.default_rng(7)
    s = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    o = pyoracle.Oracle(deck)
    for trial in range(8):
        c = deck.coord.copy()
        c[:, :3] += rng.normal(size=(deck.n, 3)) * (0.4 if trial else 0.05)
        o.set_coord(c)
        Fo, Eo, repo, _ = o.forces()
        s.set_coord(c)
        F, E, rep, _ = s.compute_forces()
        assert rep == repo
        assert rel(F, Fo) < 1e-12, (trial, rel(F, Fo))
        k = E_INDEX[kind]
        assert abs(E[k] - Eo[k]) <= 1e-10 * max(abs(Eo[k]), 1e-300), (trial, E[k], Eo[k])
    s.close()


def bare_deck(x):
    """A deck of the beads x (N, 4) with no terms at all."""
    deck = copy.deepcopy(source("angle"))
    n = len(x)
    deck.coord = np.ascontiguousarray(x, dtype=np.float64)
    deck.Q = np.zeros(n)
    deck.LJ = np.tile([2.0, 0.1], (n, 1))
    deck.prm = dict(deck.prm)
    deck.prm["alpha_lj"], deck.prm["elec"] = 0.0, 0
    for k, w in KINDS.items():
        setattr(deck, k + "_pairs", np.zeros((0, w), np.int32))
        setattr(deck, k + "_parms", np.zeros((0, 3 if k == "bond" else 2)))
    return deck


def check_against_oracle(deck, tol):
    o = pyoracle.Oracle(deck)
    Fo, Eo, repo, _ = o.forces()
    s = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    F, E, rep, _ = s.compute_forces()
    s.close()
    assert rep == repo
    assert rel(F, Fo) < tol, rel(F, Fo)
    for k in range(1, 6):
        assert abs(E[k] - Eo[k]) <= 1e-10 * max(abs(Eo[k]), 1e-12), (k, E[k], Eo[k])


def test_nearly_straight_angles():
    """Angles at and near pi: BD_BOX drops a harmonic angle within 1e-6 of
    cos theta = -1 (energy included); the cosine angle has no cut-off. Near
    pi the harmonic force divides by sqrt(1 - cos^2 theta), which amplifies
    a rounding of cos theta by 1/(1 + cos theta), up to 1e6 at the cut-off,
    so two correct evaluations agree to 1e-10 relative there, not 1e-16."""
    kinks = [0.0, 1e-9, 1e-6, 1e-4, 1e-2, 0.5]
    n = len(kinks) + 2
    x = np.zeros((n, 4))
    x[:, 3] = 2.0
    x[:, 0] = 3.8 * np.arange(n)
    x[1:n - 1, 1] = kinks                 # bead i+1 lifted off the line
    deck = bare_deck(x)
    tri = np.array([[i, i + 1, i + 2] for i in range(n - 2)], np.int32)
    deck.angle_pairs, deck.angle_parms = tri, np.tile([2.0, 3.0], (n - 2, 1))
    deck.angle_cos_pairs, deck.angle_cos_parms = tri, np.tile([-0.5, 2.0], (n - 2, 1))
    check_against_oracle(deck, 1e-9)


def test_nearly_planar_dihedrals():
    """Dihedrals near pi (an all-trans zig-zag with small out-of-plane
    offsets) and near 0 (a cis turn), where BD_BOX's harmonic-dihedral
    gradient switches between its 1/sin and 1/cos forms; sin phi stays far
    above rounding, so the float-pi wrap of phi - phi0 is not at stake."""
    offsets = [1e-4, 1e-3, 1e-2, 0.1, 0.5, -0.3, -1e-3]
    n = len(offsets) + 3
    x = np.zeros((n, 4))
    x[:, 3] = 2.0
    x[:, 0] = 3.1 * np.arange(n)
    x[:, 1] = np.where(np.arange(n) % 2, 2.2, 0.0)      # planar zig-zag, 3.8 A bonds
    x[3:, 2] = offsets
    x[-1, 1] = 2.2 if (n - 1) % 2 == 0 else 0.0          # the last bead turned cis
    deck = bare_deck(x)
    quad = np.array([[i, i + 1, i + 2, i + 3] for i in range(n - 3)], np.int32)
    deck.dihe_pairs, deck.dihe_parms = quad, np.array([[-1.5 if i % 2 else 1.2, 1 + i % 6] for i in range(n - 3)])
    deck.dihe_angle_pairs, deck.dihe_angle_parms = quad, np.tile([2.0, 0.7], (n - 3, 1))
    check_against_oracle(deck, 1e-11)


@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_non_finite_coordinate_raises_the_overlap_flag(bad):
    """A non-finite coordinate makes BD_BOX's bonded terms non-finite, which
    compute_forces reports as an overlap (the retry signal). The free-space
    cell list of a system holding such a coordinate must end (it takes the
    pair path), with the same flag."""
    deck = only(source("angle"), "angle", nonbonded=True)
    c = deck.coord.copy()
    c[5, 1] = bad
    o = pyoracle.Oracle(deck)
    o.set_coord(c)
    _, _, repo, _ = o.forces()
    assert repo == 1
    s = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    s.compute_forces()                   # builds the cell list at finite positions
    s.set_coord(c)
    _, _, rep, _ = s.compute_forces()
    assert rep == 1
    s.set_coord(deck.coord)              # and recovers once the positions are finite
    F, _, rep, _ = s.compute_forces()
    assert rep == 0 and np.isfinite(F).all()
    s.close()


def test_over_stretched_bond_is_an_error():
    """r >= r_max of a FENE bond ends BD_BOX (UNERR, bond.c:73-78); the
    engine returns BDB_ERR_BOND and stays usable."""
    deck = only(source("bond"), "bond")
    deck.bond_parms = deck.bond_parms.copy()
    deck.bond_parms[:, 1] = 5.0          # r_max 5 A, bonds of 3.8 A
    o = pyoracle.Oracle(deck)
    _, _, repo, _ = o.forces()
    assert repo == 0
    s = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    s.compute_forces()
    c = deck.coord.copy()
    b = c[10, :3] - c[9, :3]
    c[10:, :3] += 2.0 * b / np.linalg.norm(b)   # the bond 9-10 now spans 5.8 A
    o.set_coord(c)
    _, _, repo, _ = o.forces()
    assert repo == 2                     # the oracle's over-stretch code
    s.set_coord(c)
    with pytest.raises(engine.BDBError) as e:
        s.compute_forces()
    assert e.value.code == -4
    s.set_coord(deck.coord)
    _, _, rep, _ = s.compute_forces()
    assert rep == 0
    s.close()
