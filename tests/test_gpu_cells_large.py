"""Neighbour cells of segments above the shared-memory sort (16,384 beads):
such a segment is sorted by several CTAs (bitonic chunks, then merge passes
in global memory) and must give BD_BOX's forces and pair counts, not fall
back to all pairs. Checked at N = 20,000 against the oracle's O(N^2) forces
(oracle/bdb_oracle.c, force_single over all pairs): a free-space chain and a
periodic suspension, before and after the beads move far enough to force a
re-sort. Pair counts bit-exact; forces 1e-12 of the largest, energies 1e-10.
"""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

from bd_box_b200 import decks, engine  # noqa: E402
import pyoracle  # noqa: E402

N = 20000


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def check(s, o, coord):
    o.set_coord(coord)
    Fo, Eo, repo, co = o.forces()
    s.set_coord(coord)
    F, E, rep, c = s.compute_forces()
    assert rep == repo
    assert c == co, (c, co)
    assert rel(F, Fo) < 1e-12, rel(F, Fo)
    for k in range(1, 9):
        assert abs(E[k] - Eo[k]) <= 1e-10 * max(abs(Eo[k]), 1e-12), (k, E[k], Eo[k])
    nx, ny, nz, all_pairs = s.cell_grid(0)
    assert all_pairs == 0 and nx * ny * nz > 27, (nx, ny, nz, all_pairs)
    return c


@pytest.mark.parametrize("kind", ["chain", "suspension"])
def test_large_segment_cells_match_oracle(kind, tmp_path):
    d = str(tmp_path)
    if kind == "chain":
        deck = decks.read_deck(decks.write_chain_deck(d, "big", N, seed=5, hydro="none"))
    else:
        deck = decks.read_deck(decks.write_suspension_deck(d, "big", N, seed=6, phi=0.1))
    s = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    o = pyoracle.Oracle(deck)
    rng = np.random.default_rng(11)
    c0 = check(s, o, deck.coord)
    assert c0[0] + c0[1] > 0
    # a small move (within the skin: the old sort stays), then a large one
    # (every bead several angstroms: a re-sort)
    x = deck.coord.copy()
    x[:, :3] += rng.normal(size=(deck.n, 3)) * 0.05
    check(s, o, x)
    x[:, :3] += rng.normal(size=(deck.n, 3)) * 3.0
    check(s, o, x)
    # the same positions twice: the same bits
    F1 = s.compute_forces()[0]
    s.set_coord(x)
    assert np.array_equal(s.compute_forces()[0], F1)
    s.close()


@pytest.mark.parametrize("n", [3000, N])
def test_periodic_coordinates_outside_the_box(n, tmp_path):
    """A caller may set periodic coordinates outside the box (steps wrap
    them; bdb_set_coord does not): half the spheres moved by whole box
    lengths are the same configuration, so forces and pair counts match the
    oracle's minimum-image ones, for the shared-memory sort (3,000 beads)
    and the multi-CTA one (20,000)."""
    deck = decks.read_deck(decks.write_suspension_deck(str(tmp_path), "img", n, seed=8, phi=0.1))
    s = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    o = pyoracle.Oracle(deck)
    rng = np.random.default_rng(12)
    x = deck.coord.copy()
    shift = rng.integers(-2, 3, size=(n, 3)) * np.asarray(deck.box)[None, :3]
    shift[rng.random(n) < 0.5] = 0
    x[:, :3] += shift
    check(s, o, x)
    x[:, :3] += rng.normal(size=(n, 3)) * 3.0
    check(s, o, x)
    s.close()
