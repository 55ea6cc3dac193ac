"""Deck reader: BD_BOX's parsing rules (float-rounded DOUBLE keys, YESNO,
option overrides, centring, periodic wrap) and the seeded generators."""
import os

import numpy as np
import pytest

from bd_box_b200 import decks

REF_EXAMPLES = "/root/reference/examples"


def test_double_keys_are_float_rounded(tmp_path):
    p = decks.write_chain_deck(str(tmp_path), "c", 10, seed=1, dt=0.01)
    d = decks.read_deck(p)
    assert d.prm["dt"] == float(np.float32(0.01))
    assert d.prm["visc"] == float(np.float32(0.01))
    assert d.prm["lj_6_term"] == 1 and d.prm["check_overlap"] == 0


def test_overrides_win(tmp_path):
    p = decks.write_chain_deck(str(tmp_path), "c", 10, seed=1)
    d = decks.read_deck(p, {"hydro": "geyer", "dt": "0.02"})
    assert d.prm["hydro"] == 2 and d.prm["dt"] == float(np.float32(0.02))
    assert d.prm["geyer_on_the_fly"]   # YESNO keeps tolower(c) - 'n' (input.c:1041-1044)
    d = decks.read_deck(p, {"hydro": "cholesky"})
    assert d.prm["geyer_on_the_fly"] == 0   # forced off for non-TEA methods (input.c:497-501)


def test_saw_chain_geometry():
    x = decks.saw_chain(300, seed=4)
    b = np.linalg.norm(np.diff(x, axis=0), axis=1)
    assert np.allclose(b, 3.8)
    d = np.linalg.norm(x[:, None] - x[None], axis=2)
    iu = np.triu_indices(300, 2)
    assert d[iu].min() >= 4.0 - 1e-9


def test_suspension_fits_box_after_centring(tmp_path):
    p = decks.write_suspension_deck(str(tmp_path), "s", 300, seed=3, phi=0.1)
    d = decks.read_deck(p)
    L = d.box[0]
    assert np.abs(d.coord[:, :3]).max() <= L / 2 + 1e-6
    v = d.coord[:, None, :3] - d.coord[None, :, :3]
    v -= L * np.floor(v / L + 0.5)
    r = np.linalg.norm(v, axis=2) + np.eye(d.n) * 1e9
    assert r.min() >= 2.0 - 1e-9


def test_replica_sizes_are_seeded():
    a, b = decks.replica_sizes(), decks.replica_sizes()
    assert np.array_equal(a, b) and a.min() >= 64 and a.max() <= 1024 and len(a) == 256


@pytest.mark.skipif(not os.path.isdir(REF_EXAMPLES), reason="BD_BOX examples not present")
@pytest.mark.parametrize("ex", ["DNA/dna.prm", "CI2_TEA_HI/ci2.prm", "HARD_SPHERES/box.prm"])
def test_reads_reference_examples(ex):
    d = decks.read_deck(os.path.join(REF_EXAMPLES, ex))
    assert d.n > 0 and d.coord.shape == (d.n, 4)
