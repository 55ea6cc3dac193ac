"""Deck reader: BD_BOX's parsing rules (float-rounded DOUBLE keys, YESNO,
option overrides, centring, periodic wrap) and the seeded generators."""
import os

import numpy as np
import pytest

from bd_box_b200 import decks



def _reference_examples():
    """BD_BOX's example decks: $BDB_REFERENCE/examples, else next to the
    sources the oracle's reference build was compiled from (recorded by
    `make -C oracle ref` in oracle/_ref/reference_src)."""
    root = os.environ.get("BDB_REFERENCE")
    if root:
        return os.path.join(root, "examples")
    rec = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                       "reference_src")
    if os.path.exists(rec):
        with open(rec) as f:
            return os.path.join(os.path.dirname(f.read().strip()), "examples")
    return ""


REF_EXAMPLES = _reference_examples()


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


def test_external_force_and_flow_keys(tmp_path):
    """The external-field, sphere and flow keys: BD_BOX's defaults
    (electro_ext.c:30-36, sboundary.c:31-34), their ABI mapping, the sphere
    check of trans.c iscorrect, and nine doubles for vel_grad_tensor."""
    from bd_box_b200 import engine
    p = decks.write_chain_deck(str(tmp_path), "k", 12, seed=2, hydro="none")
    d = decks.read_deck(p)
    assert (d.prm["E_magn"], d.prm["sboundary_A"], d.prm["sboundary_n"], d.prm["E_factor"]) == (1.0, 1.0, 2, 1.0)
    P = engine.params_from_deck(d)
    assert (P.e_ext, P.sboundary, P.flow) == (0, 0, 0)
    d = decks.read_deck(p, overrides={"E_ext": "yes", "E_type": "RF", "E_dir1": "z", "E_dir2": "x",
                                      "vel_grad_tensor": "0 1.5 0 0 0 0 0 0 0.25"})
    P = engine.params_from_deck(d)
    # YESNO keys keep BD_BOX's value[0] - 'n' (11 for yes), which is all that is tested
    assert bool(P.e_ext) and (P.e_type, P.e_dir1, P.e_dir2) == (2, 2, 0)
    assert P.flow == 1 and list(P.vel_grad) == [0, 1.5, 0, 0, 0, 0, 0, 0, 0.25]
    with pytest.raises(ValueError):
        decks.vel_grad({"vel_grad_tensor": "1 2 3"})
    with pytest.raises(ValueError):       # beads outside the sphere (iscorrect)
        decks.read_deck(p, overrides={"bc": "sphere", "sphere_radius": 1.0})
    d = decks.read_deck(p, overrides={"bc": "sphere", "sphere_radius": 500.0})
    assert engine.params_from_deck(d).bc == 2
