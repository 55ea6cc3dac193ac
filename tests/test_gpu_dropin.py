"""The BD_BOX drop-in (bd_box_b200/dropin): BD_BOX's own host code linked
with the drop-in and libbdb200.so in place of its seven CPU translation
units, run on the golden decks.

* ref_harness_b200 is the oracle harness (oracle/ref_harness.c) linked with
  the drop-in. Each mode calls the reference-named entry points that
  BD_BOX's callers use (compute_D, compute_forces, compute_Rf, compute_r, and
  save_curr_coord/save_curr_forces/compute_hydro as main_loop.c does). Its
  outputs must match the golden fixtures made by the CPU build.
* bd_box_b200 is BD_BOX's stock main program with its own drand48 RNG. For
  the same deck and seed its xyz trajectory and energy file must match those
  of the stock CPU program (oracle/_ref/bd_box) at the printed precision.

Both binaries are built by `make -C oracle ref dropin`, which needs the BD_BOX
sources at build time; without them these tests are skipped.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, gpu_available
import golden_cases
from bd_box_b200 import decks

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

REF = os.path.join(ROOT, "oracle", "_ref")
HARNESS = os.path.join(REF, "ref_harness_b200")
STOCK_B200 = os.path.join(REF, "bd_box_b200")
STOCK_CPU = os.path.join(REF, "bd_box")


def need(path):
    if not os.path.exists(path):
        pytest.skip(f"{os.path.basename(path)} not built (make -C oracle ref dropin needs the BD_BOX sources)")


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


def run(d, mode, *args, env=None):
    out = os.path.join(d, "out.bin")
    e = dict(os.environ, BDB_GAUSS_FILE=os.path.join(d, "g.bin"), OMP_NUM_THREADS="1", **(env or {}))
    extra = os.path.join(d, "cos_dihe.txt")
    if os.path.exists(extra):   # cosine dihedrals, added through add_dihe by the harness
        e["BDB_EXTRA_DIHE"] = extra
    r = subprocess.run([HARNESS, "c.prm", mode, out, *args], cwd=d, env=e, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    return np.fromfile(out)


def write_case(name, d):
    """the golden deck, its Gaussians and the reference outputs, in dir d"""
    z = np.load(os.path.join(golden_cases.GOLDEN, name + ".npz"))
    with open(os.path.join(d, "c.prm"), "w") as f:
        f.write(str(z["prm"]))
    with open(os.path.join(d, "c.str"), "w") as f:
        f.write(str(z["str"]))
    z["gauss"].tofile(os.path.join(d, "g.bin"))
    if "cos_dihe" in z.files:
        with open(os.path.join(d, "cos_dihe.txt"), "w") as f:
            for r in z["cos_dihe"]:
                f.write("%d %d %d %d %.17g %.17g %.17g\n" % tuple(r))
    return {k: z[k] for k in z.files if k not in ("prm", "str")}


@pytest.mark.parametrize("name", golden_cases.names())
def test_dropin_harness_matches_reference_outputs(name, tmp_path):
    need(HARNESS)
    d = str(tmp_path)
    ref = write_case(name, d)
    n3 = ref["F"].size
    tol = 1e-11 if "susp" in name else 1e-12
    D = run(d, "D").reshape(n3, n3)
    assert rel(D, ref["D"]) < tol
    f = run(d, "forces")
    F, E, rep = f[:n3], f[n3:n3 + 9], f[n3 + 9]
    assert rel(F, ref["F"]) < 1e-12
    assert rep == ref["rep"]
    for k in range(1, 8):
        if abs(ref["E"][k]) > 1e-9:
            assert abs(E[k] - ref["E"][k]) <= 1e-10 * abs(ref["E"][k]), k
    assert rel(run(d, "df"), ref["Rf"]) < tol
    if "tea_Rs" in ref:
        assert rel(run(d, "tea")[:n3], ref["tea_Rs"]) < tol
    K = ref["traj"].shape[0]
    traj = run(d, "steps", str(K)).reshape(ref["traj"].shape)
    start = decks.read_deck(os.path.join(d, "c.prm")).coord
    disp = np.abs(ref["traj"][0, :, :3] - start[:, :3]).max()
    for k in range(K):
        assert np.abs(traj[k] - ref["traj"][k]).max() <= 1e-9 * disp, k


def _numbers(path):
    vals = []
    with open(path) as f:
        for ln in f:
            for tok in ln.split():
                try:
                    vals.append(float(tok))
                except ValueError:
                    pass
    return np.array(vals)


@pytest.mark.parametrize("case", ["chain32_chol", "chain24_igt_chol"])
def test_stock_main_program_matches_cpu_build(case, tmp_path):
    """BD_BOX's own main(), main_loop() and output writers on the drop-in,
    with BD_BOX's drand48 noise: same xyz and energy files as the CPU build
    (Ermak-McCammon and IGT decks)."""
    need(STOCK_B200)
    need(STOCK_CPU)
    z = np.load(os.path.join(golden_cases.GOLDEN, case + ".npz"))
    prm = [ln for ln in str(z["prm"]).splitlines() if ln.split()[:1] != ["bdsteps"]]
    prm += ["bdsteps 5", "xyz_filename out.xyz", "enr_filename out.enr", "save_xyz_freq 1", "save_enr_freq 1"]
    outs = {}
    for tag, exe in (("cpu", STOCK_CPU), ("b200", STOCK_B200)):
        d = tmp_path / tag
        d.mkdir()
        (d / "c.prm").write_text("\n".join(prm) + "\n")
        (d / "c.str").write_text(str(z["str"]))
        r = subprocess.run([exe, "c.prm"], cwd=d, capture_output=True, text=True, timeout=300,
                           env=dict(os.environ, OMP_NUM_THREADS="1"))
        assert r.returncode == 0, (tag, r.stdout[-1000:], r.stderr[-1000:])
        outs[tag] = (_numbers(d / "out.xyz"), _numbers(d / "out.enr"))
    (xc, ec), (xb, eb) = outs["cpu"], outs["b200"]
    assert xc.size == xb.size and xc.size > 20 * 3 * 5
    assert np.abs(xc - xb).max() <= 2e-6          # xyz prints 6 decimals
    assert ec.size == eb.size and ec.size > 0
    assert np.allclose(eb, ec, rtol=1e-5, atol=2e-6)


def test_stock_main_ermak_var_retries_match_cpu_build(tmp_path):
    """comp_step_ermak's retry loop with ermak_var (diff_comp.c:152-179): a
    dense suspension with overlap checks, where almost every move overlaps
    at first and dt is halved until it does not. BD_BOX's stock main() on
    the drop-in and the CPU build take the same retries (the frame times
    show the halvings) and write the same frames."""
    need(STOCK_B200)
    need(STOCK_CPU)
    outs = {}
    for tag, exe in (("cpu", STOCK_CPU), ("b200", STOCK_B200)):
        d = tmp_path / tag
        d.mkdir()
        decks.write_suspension_deck(str(d), "c", 100, seed=5, ewald_r=2, phi=0.3, dt=0.05,
                                    extra={"hydro": "none", "check_overlap": "yes", "algorithm": "ermak_var",
                                           "bdsteps": 6, "xyz_filename": "out.xyz", "save_xyz_freq": 1,
                                           "move_attempts": 200})
        r = subprocess.run([exe, "c.prm"], cwd=d, capture_output=True, text=True, timeout=600,
                           env=dict(os.environ, OMP_NUM_THREADS="1"))
        assert r.returncode == 0, (tag, r.stdout[-1000:], r.stderr[-1000:])
        text = (d / "out.xyz").read_text()
        times = [float(ln.split()[-1]) for ln in text.splitlines() if "time" in ln]
        outs[tag] = (times, _numbers(d / "out.xyz"))
    (tc, xc), (tb, xb) = outs["cpu"], outs["b200"]
    assert tc == tb and len(tc) >= 6
    assert (np.diff(tc) < 0.05 - 1e-9).any()     # retries with a halved dt happened
    assert xc.size == xb.size
    assert np.abs(xc - xb).max() <= 2e-6


@pytest.mark.parametrize("name", ["rf", "sphere"])
def test_dropin_external_forces_match_cpu_build(name, tmp_path):
    """Electric field and bounding sphere through the drop-in: BD_BOX's own
    compute_forces / compute_hydro callers (harness modes) on the drop-in
    against the same harness on the CPU build."""
    need(HARNESS)
    cpu = os.path.join(REF, "ref_harness")
    need(cpu)
    from test_oracle_pin import ext_deck
    p = ext_deck(tmp_path, name)
    os.replace(p, os.path.join(tmp_path, "c.prm"))
    deck = decks.read_deck(os.path.join(tmp_path, "c.prm"))
    n3 = 3 * deck.n
    np.random.default_rng(6).standard_normal(8 * n3).tofile(tmp_path / "g.bin")
    d = str(tmp_path)
    e = dict(os.environ, BDB_GAUSS_FILE=os.path.join(d, "g.bin"), OMP_NUM_THREADS="1")
    ref = {}
    for mode, args in (("forces", []), ("steps", ["3"])):
        r = subprocess.run([cpu, "c.prm", mode, os.path.join(d, "ref.bin"), *args], cwd=d, env=e,
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        ref[mode] = np.fromfile(os.path.join(d, "ref.bin"))
    f = run(d, "forces")
    assert rel(f[:n3], ref["forces"][:n3]) < 1e-12 and f[n3 + 9] == ref["forces"][n3 + 9]
    traj = run(d, "steps", "3").reshape(3, deck.n, 4)
    traj_ref = ref["steps"].reshape(3, deck.n, 4)
    disp = np.abs(traj_ref[0, :, :3] - deck.coord[:, :3]).max()
    assert np.abs(traj - traj_ref).max() <= 1e-9 * disp


@pytest.mark.parametrize("hydro", ["none", "geyer"])
def test_dropin_newton_matches_cpu_build(hydro, tmp_path):
    """ermak_newton through the drop-in (bdb_newton_resolve in the retry
    loop of comp_step_ermak_newton) against the CPU build: the same
    trajectory from the same Gaussian stream."""
    need(HARNESS)
    cpu = os.path.join(REF, "ref_harness")
    need(cpu)
    from test_oracle_pin import newton_deck
    p = newton_deck(tmp_path, hydro)
    os.replace(p, os.path.join(tmp_path, "c.prm"))
    deck = decks.read_deck(os.path.join(tmp_path, "c.prm"))
    n3 = 3 * deck.n
    np.random.default_rng(4).standard_normal(40 * n3).tofile(tmp_path / "g.bin")
    d = str(tmp_path)
    e = dict(os.environ, BDB_GAUSS_FILE=os.path.join(d, "g.bin"), OMP_NUM_THREADS="1")
    r = subprocess.run([cpu, "c.prm", "steps", os.path.join(d, "ref.bin"), "4"], cwd=d, env=e,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    traj_ref = np.fromfile(os.path.join(d, "ref.bin")).reshape(4, deck.n, 4)
    traj = run(d, "steps", "4").reshape(4, deck.n, 4)
    disp = np.abs(traj_ref[0, :, :3] - deck.coord[:, :3]).max()
    assert np.abs(traj - traj_ref).max() <= 1e-9 * disp


def test_dropin_shear_flow_matches_cpu_build(tmp_path):
    """A flowing solvent (vel_grad_tensor) through the drop-in against the
    CPU build: three Ermak steps from the same Gaussian stream."""
    need(HARNESS)
    cpu = os.path.join(REF, "ref_harness")
    need(cpu)
    p = decks.write_chain_deck(str(tmp_path), "fl", 30, seed=23, hydro="cholesky",
                               extra={"vel_grad_tensor": "0 0.75 0 0 0 0 0.1 0 0"})
    os.replace(p, os.path.join(tmp_path, "c.prm"))
    deck = decks.read_deck(os.path.join(tmp_path, "c.prm"))
    np.random.default_rng(3).standard_normal(9 * deck.n).tofile(tmp_path / "g.bin")
    d = str(tmp_path)
    e = dict(os.environ, BDB_GAUSS_FILE=os.path.join(d, "g.bin"), OMP_NUM_THREADS="1")
    r = subprocess.run([cpu, "c.prm", "steps", os.path.join(d, "ref.bin"), "3"], cwd=d, env=e,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    traj_ref = np.fromfile(os.path.join(d, "ref.bin")).reshape(3, deck.n, 4)
    traj = run(d, "steps", "3").reshape(3, deck.n, 4)
    disp = np.abs(traj_ref[0, :, :3] - deck.coord[:, :3]).max()
    assert np.abs(traj - traj_ref).max() <= 1e-9 * disp
