"""Generate the golden fixtures from BD_BOX itself (test infrastructure).

Each case is a small seeded deck run through the reference's own CPU code
(oracle/_ref/ref_harness, built by `make -C oracle ref` from the BD_BOX
sources) with a shared Gaussian stream. The .npz keeps the deck text, the
Gaussians and every output, so the tests need neither the reference
sources nor the harness:

    python tests/golden/make_golden.py [case ...]   # rewrites tests/golden/*.npz
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from bd_box_b200 import decks  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")


def bonded_chain(d, name, n, seed):
    """Chain with every bonded term type and 1-2 scaled non-bonded terms."""
    p = decks.write_chain_deck(d, name, n, seed=seed, hydro="cholesky",
                               extra={"bond_lj_scale": 0.5, "bond_c_scale": 0.25, "nb_list": "brute"})
    rng = np.random.default_rng(seed)
    with open(os.path.join(d, name + ".str"), "a") as f:
        for i in range(1, n - 1):
            if i % 2:
                f.write(f"angle harm {i} {i + 1} {i + 2} {100 + 20 * rng.random():.4f} {2 + rng.random():.4f}\n")
            else:
                f.write(f"angle cosine {i} {i + 1} {i + 2} {110 + 20 * rng.random():.4f} {3 + rng.random():.4f}\n")
        for i in range(1, n - 2):
            if i % 3 == 0:
                # the reference's "cosine" dihedral line cannot be parsed
                # (input.c:621-628 rejects its third value), so the cosine
                # form is not exercised through a deck
                continue
            f.write(f"dihe harm {i} {i + 1} {i + 2} {i + 3} {-60 + 120 * rng.random():.4f} {1 + rng.random():.4f}\n")
    return p


CASES = {
    "chain32_chol": lambda d: decks.write_chain_deck(d, "c", 32, seed=101, hydro="cholesky"),
    "chain40_tea": lambda d: decks.write_chain_deck(d, "c", 40, seed=102, hydro="geyer"),
    "chain20_none": lambda d: decks.write_chain_deck(d, "c", 20, seed=103, hydro="none"),
    "susp24_ewald": lambda d: decks.write_suspension_deck(d, "c", 24, seed=104, ewald_r=2, phi=0.15,
                                                          extra={"geyer_on_the_fly": "no"}),
    "chain24_bonded": lambda d: bonded_chain(d, "c", 24, 105),
    # Smith's Ewald sums (diff_tensor.c:102-263): TEA on the stored tensor,
    # and Cholesky on a dilute suspension (positive definite at R=3)
    "susp24_smith": lambda d: decks.write_suspension_deck(d, "c", 24, seed=108, ewald_r=2, phi=0.15,
                                                          extra={"geyer_on_the_fly": "no",
                                                                 "ewald_method": "smith"}),
    "susp32_smith_chol": lambda d: decks.write_suspension_deck(d, "c", 32, seed=109, ewald_r=3, phi=0.05,
                                                               extra={"hydro": "cholesky",
                                                                      "ewald_method": "smith"}),
    # IGT predictor-corrector (comp_step_IGT_const): two 3N Gaussian draws
    # per step, the predictor's then the corrector's
    "chain24_igt_chol": lambda d: decks.write_chain_deck(d, "c", 24, seed=106, hydro="cholesky",
                                                         extra={"algorithm": "igt_const"}),
    "chain20_igt_none": lambda d: decks.write_chain_deck(d, "c", 20, seed=107, hydro="none",
                                                         extra={"algorithm": "igt_const"}),
}

def cos_dihedrals(n, seed):
    """Cosine dihedrals on every run of four consecutive beads, rows
    (i, j, k, l, k_theta, m, delta): multiplicities 1..7 in turn (7 takes
    BD_BOX's fall-back, cos(m theta) = 1 with no force, dihe.c:146-184),
    delta = +-1, k_theta in [1, 3]."""
    rng = np.random.default_rng(seed)
    return np.array([[i, i + 1, i + 2, i + 3, 1 + 2 * rng.random(), 1 + i % 7, 1.0 if i % 2 else -1.0]
                     for i in range(n - 3)])


# Cases whose cosine dihedrals are added through the harness (BDB_EXTRA_DIHE),
# because BD_BOX's .str parser cannot read them.
EXTRA_DIHE = {
    "chain24_cosdihe": lambda n: cos_dihedrals(n, 110),
}
CASES["chain24_cosdihe"] = lambda d: decks.write_chain_deck(d, "c", 24, seed=110, hydro="cholesky")

STEPS = 3


def run(d, prm, mode, *args):
    out = os.path.join(d, "out.bin")
    env = dict(os.environ, BDB_GAUSS_FILE=os.path.join(d, "g.bin"), OMP_NUM_THREADS="1")
    extra = os.path.join(d, "cos_dihe.txt")
    if os.path.exists(extra):
        env["BDB_EXTRA_DIHE"] = extra
    subprocess.run([HARNESS, os.path.basename(prm), mode, out, *args], cwd=d, env=env, check=True,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    return np.fromfile(out)


def make(name, fn):
    with tempfile.TemporaryDirectory() as d:
        prm = fn(d)
        deck = decks.read_deck(prm)
        n, n3 = deck.n, 3 * deck.n
        draws = 2 if deck.prm["algorithm"] >= decks.ALGORITHM["igt_const"] else 1
        g = np.random.default_rng(zlib.crc32(name.encode())).standard_normal(n3 * STEPS * draws)
        g.tofile(os.path.join(d, "g.bin"))
        res = {"prm": open(prm).read(), "str": open(prm[:-4] + ".str").read(), "gauss": g}
        if name in EXTRA_DIHE:
            rows = EXTRA_DIHE[name](n)
            with open(os.path.join(d, "cos_dihe.txt"), "w") as f:
                for r in rows:
                    f.write("%d %d %d %d %.17g %.17g %.17g\n" % tuple(r))
            res["cos_dihe"] = rows
        res["D"] = run(d, prm, "D").reshape(n3, n3)
        f = run(d, prm, "forces")
        res["F"], res["E"], res["rep"], res["counts"] = f[:n3], f[n3:n3 + 9], f[n3 + 9], f[n3 + 10:n3 + 14]
        res["Rf"] = run(d, prm, "df")
        if deck.prm["hydro"] == 2:
            t = run(d, prm, "tea")
            res["tea_Rs"], res["tea_eps"] = t[:n3], t[-1]
        res["traj"] = run(d, prm, "steps", str(STEPS)).reshape(STEPS, n, 4)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **res)
        print(name, n, {k: np.shape(v) for k, v in res.items() if k not in ("prm", "str")})


def main():
    if not os.path.exists(HARNESS):
        raise SystemExit("build the reference harness first: make -C oracle ref")
    only = set(sys.argv[1:])
    for name, fn in CASES.items():
        if not only or name in only:
            make(name, fn)


if __name__ == "__main__":
    main()
