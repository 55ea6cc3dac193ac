"""The mixed Cholesky step with device noise fuses rand_move
(rand_move.c:132-168) with the B.xi product and the position update
(diff_equation.c:254-283): the kernel that finishes the product moves the
beads and draws the next step's Philox Gaussians; the product draws them
itself on the first such step (or after anything else wrote the noise or
the stream index). Two launches fewer per step. It must give the same bits
as the separate noise, product and update kernels (BDB_NO_FUSE), step after
step, across refreshes of D and its factor, in free space and with
periodic wrapping, and advance the Philox stream alike.
"""
import os

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

from bd_box_b200 import decks, engine  # noqa: E402


def system(deck, fused):
    if not fused:
        os.environ["BDB_NO_FUSE"] = "1"
    try:
        return engine.System(deck, precision=engine.PREC_MIXED, refresh=10)
    finally:
        os.environ.pop("BDB_NO_FUSE", None)


@pytest.mark.parametrize("kind", ["chain", "periodic"])
def test_fused_step_matches_separate_kernels(kind, tmp_path):
    d = str(tmp_path)
    if kind == "chain":
        deck = decks.read_deck(decks.write_chain_deck(d, "f", 700, seed=41, hydro="cholesky"))
    else:
        deck = decks.read_deck(decks.write_suspension_deck(d, "f", 300, seed=42, phi=0.1,
                                                           extra={"hydro": "cholesky", "geyer_on_the_fly": "no"}))
    a, b = system(deck, True), system(deck, False)
    for k in (1, 1, 12, 25):      # eager first step, then graph replays over three refreshes
        a.step(k)
        b.step(k)
        xa, xb = a.get_coord(), b.get_coord()
        assert np.array_equal(xa, xb), float(np.abs(xa - xb).max())
    if kind == "periodic":
        L = np.asarray(deck.box[:3])
        assert (np.abs(xa[:, :3]) <= 0.5 * L + 1e-9).all()   # wrapped into the box
    x0 = deck.coord[:, :3]
    assert np.abs(xa[:, :3] - x0).max() > 0                 # the beads moved
    a.close()
    b.close()
