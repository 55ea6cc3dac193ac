"""The CUDA path against BD_BOX's own outputs (golden fixtures made by the
reference CPU build, tests/golden/make_golden.py), through the C ABI."""
import numpy as np
import pytest

from conftest import gpu_available
import golden_cases

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

from bd_box_b200 import decks, engine  # noqa: E402


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("name", golden_cases.names())
def test_engine_matches_reference_outputs(name):
    deck, ref = golden_cases.load(name)
    n3 = 3 * deck.n
    tol = 1e-11 if deck.ewald else 1e-12
    s = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    F, E, rep, counts = s.compute_forces()
    assert counts == (int(ref["counts"][0]), int(ref["counts"][1]))
    assert rep == int(ref["rep"])
    assert rel(F, ref["F"]) < 1e-12
    for k in range(1, 8):
        if abs(ref["E"][k]) > 1e-9:
            assert abs(E[k] - ref["E"][k]) <= 1e-10 * abs(ref["E"][k]), k
    assert rel(s.compute_D(), ref["D"]) < tol
    assert rel(s.compute_Rf(), ref["Rf"]) < tol
    if "tea_Rs" in ref:
        assert rel(s.compute_r(ref["gauss"][:n3]), ref["tea_Rs"]) < tol
    s2 = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    K = ref["traj"].shape[0]
    disp = np.abs(ref["traj"][0, :, :3] - deck.coord[:, :3]).max()
    igt = deck.prm["algorithm"] >= decks.ALGORITHM["igt_const"]
    for k in range(K):
        if igt:   # comp_step_IGT_const: two draws per step
            s2.step_igt(1, ref["gauss"][2 * k * n3:2 * (k + 1) * n3])
        else:
            s2.step(1, ref["gauss"][k * n3:(k + 1) * n3])
        assert np.abs(s2.get_coord() - ref["traj"][k]).max() <= 1e-9 * disp, k
