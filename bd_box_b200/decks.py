"""BD_BOX input decks: the .prm/.str reader and seeded deck generators.

Reader
------
``read_deck(prm_path, overrides)`` mirrors how BD_BOX turns a control file
and a structure file into its global state:

* ``.prm`` lines are ``keyword value`` with ``#`` comments
  (input.c:273-343); ``--key=value`` overrides win over the file
  (input.c:205-233, 353-379).
* Every DOUBLE key is rounded to float on input, ``*val=(FLOAT)atof(value)``
  (input.c:1010-1013); YESNO keys are ``tolower(c)-'n'`` (input.c:1041-1044),
  normalised to 1 only for ``lj_6_term`` (input.c:469).
* ``.str`` lines ``sub name id x y z a Q 2R eps m``, ``bond i j r0 rmax H``,
  ``angle [cosine|...] i j k phi0 k``, ``dihe [cosine|...] ...``
  (input.c:505-641) are read at full double precision; ``LJ[2i]=2R/2``
  (data.c:85-109); angles are stored in radians with the float constant pi
  (angle.c:98, angle_cos.c:96, dihe_angle.c:283); a cosine dihedral stores
  ``-k*delta`` (dihe.c:208).
* ``apply_options`` derivations (input.c:353-503): ``inv_L``/``box`` under
  periodic boundaries, ``ewald = hydro != none`` there, and
  ``geyer_on_the_fly`` forced off unless ``hydro geyer`` with an E-M
  algorithm.
* ``center_coords`` (trans.c:38-99) and the first ``trans_to_box`` of every
  bead (main_loop.c:63-66), then ``init_cutoff`` (pre_func.c:197-232).

Generators
----------
Seeded decks for the five benchmark workloads (chains built as
self-avoiding walks, periodic suspensions by random sequential insertion).
They write ordinary ``.prm``/``.str`` files that BD_BOX itself reads.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

F32_PI = float(np.float32(math.pi))  # M_PIF in data.h is a float literal

# integer codes, as in diff_alg/diff_tensor.h:29-62, trans.h:43-63, bucket.h:44-50
HYDRO = {"none": 0, "cholesky": 1, "geyer": 2, "chebyshev": 3}
ALGORITHM = {"ermak_const": 0, "ermak_var": 1, "ermak_newton": 2,
             "igt_const": 3, "igt_var": 4, "igt_var_rev": 5}
BC = {"none": 0, "periodic": 1, "sphere": 2}
NB_LIST = {"brute": 0, "bucket_space": 1, "bucket_list": 2}
EWALD_METHOD = {"smith": 0, "beenakker": 1}

def _F(x: float) -> float:
    """Value of a C float literal such as ``298.15f`` widened to double."""
    return float(np.float32(x))


# key -> (type, default), defaults from the MAKE_STR_IN declarations
# (diff_decl.c:65-82, calc_func.c:51-53, LJ.c:31-33, electro.c:30-34,
#  input.c:60-89, trans.c:33-35, bucket.c:40, rand_move.c:40, main_loop.c:45,
#  electro_ext.c:30-36, sboundary.c:31-34)
PRM_KEYS = {
    "out_filename": ("STR", None), "dt": ("DOUBLE", 0.0), "visc": ("DOUBLE", 0.01),
    "vfactor": ("DOUBLE", 14.4), "T": ("DOUBLE", _F(298.15)), "epsilon_c": ("DOUBLE", _F(78.54)),
    "kappa_c": ("DOUBLE", _F(0.1)), "cutoff_c": ("DOUBLE", 0.0), "bdsteps": ("INT", 0),
    "gamma_c": ("DOUBLE", _F(331.842)), "alpha_lj": ("DOUBLE", 4.0), "cutoff_lj": ("DOUBLE", 0.0),
    "lj_6_term": ("YESNO", 1), "save_xyz_freq": ("INT", 1), "save_dcd_freq": ("INT", 1),
    "save_rst_freq": ("INT", 1), "save_enr_freq": ("INT", 1), "xbox": ("DOUBLE", 0.0),
    "ybox": ("DOUBLE", 0.0), "zbox": ("DOUBLE", 0.0), "elec": ("YESNO", 1),
    "hydro": ("HYDRO", 0), "algorithm": ("ALGORITHM", 2), "str_filename": ("STR", None),
    "xyz_filename": ("STR", None), "dcd_filename": ("STR", None), "enr_filename": ("STR", None),
    "rst_filename": ("STR", None), "pqr_filename": ("STR", None), "rand_seed": ("INT", 12345),
    "E_ext": ("YESNO", 0), "E_magn": ("DOUBLE", 1.0), "E_type": ("STR", "DC"),
    "E_freq": ("DOUBLE", 0.0), "E_dir1": ("STR", "x"), "E_dir2": ("STR", "y"),
    "E_factor": ("DOUBLE", 1.0), "bc": ("BC", 1), "sphere_radius": ("DOUBLE", 0.0),
    "bond_lj_scale": ("DOUBLE", 1.0), "bond_c_scale": ("DOUBLE", 1.0), "restart": ("STR", None),
    "move_attempts": ("INT", 10000), "vel_grad_tensor": ("STR", None), "ewald_real": ("INT", 10),
    "ewald_recip": ("INT", 10), "ewald_alpha": ("DOUBLE", 1.77245385090551602729),
    "ewald_method": ("EWALD", 0), "MPI_nprow": ("INT", 0), "MPI_npcol": ("INT", 0),
    "MPI_block": ("INT", 0), "cuda_devices": ("STR", None), "e_collision": ("DOUBLE", 1.0),
    "single_point": ("STR", None), "nb_list": ("NB", 0), "sboundary": ("YESNO", 0),
    "sboundary_A": ("DOUBLE", 1.0), "sboundary_n": ("INT", 2), "sboundary_cutoff": ("DOUBLE", 0.0),
    "check_overlap": ("YESNO", 1), "geyer_on_the_fly": ("YESNO", 1), "cuda_block": ("INT", 0),
}
_ENUMS = {"HYDRO": HYDRO, "ALGORITHM": ALGORITHM, "BC": BC, "NB": NB_LIST, "EWALD": EWALD_METHOD}


def _f32(x: float) -> float:
    return float(np.float32(float(x)))


def _apply(typ: str, value: str):
    if typ == "DOUBLE":
        return _f32(value)
    if typ == "INT":
        return int(value.split()[0])
    if typ == "YESNO":
        return ord(value[0].lower()) - ord("n")
    if typ in _ENUMS:
        if value not in _ENUMS[typ]:
            raise ValueError(f"unknown value {value!r}")
        return _ENUMS[typ][value]
    return value


@dataclass
class Deck:
    """Everything BD_BOX holds in globals after its init phase."""
    prm: dict
    coord: np.ndarray          # (N, 4) float64: x, y, z, hydrodynamic radius
    Q: np.ndarray              # (N,) charges
    LJ: np.ndarray             # (N, 2): sigma_LJ/2, epsilon_LJ
    masses: np.ndarray
    ids: np.ndarray
    bond_pairs: np.ndarray     # (B, 2) int32 bead offsets
    bond_parms: np.ndarray     # (B, 3) r0, rmax, H
    angle_pairs: np.ndarray    # (A, 3)
    angle_parms: np.ndarray    # (A, 2) phi0 [rad], k
    angle_cos_pairs: np.ndarray
    angle_cos_parms: np.ndarray  # (A, 2) cos(phi0), k
    dihe_pairs: np.ndarray     # (Dh, 4)
    dihe_parms: np.ndarray     # (Dh, 2) -k*delta, m
    dihe_angle_pairs: np.ndarray
    dihe_angle_parms: np.ndarray  # (Dh, 2) k, theta0 [rad]
    names: list = field(default_factory=list)   # bead names of the sub lines (output.c writes them)
    box: np.ndarray = field(default_factory=lambda: np.zeros(4))
    inv_L: np.ndarray = field(default_factory=lambda: np.zeros(4))
    ewald: int = 0
    max_force_cutoff: float = 0.0

    @property
    def n(self) -> int:
        return int(self.coord.shape[0])


def read_prm(path: str, overrides: dict | None = None) -> dict:
    prm = {k: d for k, (t, d) in PRM_KEYS.items()}
    seen = {}
    with open(path) as f:
        for line in f:
            line = line.split("#", 1)[0]
            parts = line.strip().split(None, 1)
            if not parts:
                continue
            if len(parts) < 2 or not parts[1].strip():
                raise ValueError(f"Wrong prm file format, no value: {line!r}")
            key, value = parts[0], parts[1].rstrip(" \t")
            if key not in PRM_KEYS:
                raise ValueError(f"Wrong prm file format, unknown token {key}")
            seen[key] = value
    for key, value in (overrides or {}).items():
        seen[key] = str(value)
    for key, value in seen.items():
        prm[key] = _apply(PRM_KEYS[key][0], value)
    if prm["lj_6_term"]:
        prm["lj_6_term"] = 1
    prm["_dir"] = os.path.dirname(os.path.abspath(path))
    return prm


def vel_grad(prm: dict):
    """The velocity-gradient tensor G (9 doubles, row-major) of a deck, or
    None: vel_grad_tensor is read as nine doubles (input.c:1110-1124, no
    float rounding)."""
    v = prm.get("vel_grad_tensor")
    if v is None:
        return None
    vals = [float(t) for t in str(v).split()]
    if len(vals) != 9:
        raise ValueError("vel_grad_tensor needs 9 values")
    return vals


def read_str(path: str):
    subs, bonds, angles, angles_cos, dihes, dihe_angles = [], [], [], [], [], []
    with open(path) as f:
        for line in f:
            line = line.split("#", 1)[0]
            tok = line.split()
            if not tok:
                continue
            tag = tok[0]
            if tag == "sub":
                if len(tok) != 11:
                    raise ValueError("Wrong line in sub")
                subs.append((int(tok[2]), [float(v) for v in tok[3:11]], tok[1]))
            elif tag == "bond":
                bonds.append(([int(v) for v in tok[1:3]], [float(v) for v in tok[3:6]]))
            elif tag == "angle":
                ids = [int(v) for v in tok[2:5]]
                vals = [float(v) for v in tok[5:7]]
                (angles_cos if tok[1] == "cosine" else angles).append((ids, vals))
            elif tag == "dihe":
                ids = [int(v) for v in tok[2:6]]
                vals = [float(v) for v in tok[6:]]
                (dihes if tok[1] == "cosine" else dihe_angles).append((ids, vals))
            else:
                raise ValueError(f"Unknow tag in str file: {tag}")
    return subs, bonds, angles, angles_cos, dihes, dihe_angles


def read_deck(prm_path: str, overrides: dict | None = None) -> Deck:
    prm = read_prm(prm_path, overrides)
    sp = prm["str_filename"]
    if sp is None:
        raise ValueError("str_filename not defined")
    if not os.path.isabs(sp):
        sp = os.path.join(prm["_dir"], sp) if not os.path.exists(sp) else sp
    subs, bonds, angles, angles_cos, dihes, dihe_angles = read_str(sp)
    n = len(subs)
    if n == 0:
        raise ValueError("Empty str file, no particles")
    ids = np.array([s[0] for s in subs], dtype=np.int32)
    vals = np.array([s[1] for s in subs], dtype=np.float64)
    coord = vals[:, 0:4].copy()
    Q = vals[:, 4].copy()
    LJ = np.stack([vals[:, 5] / 2, vals[:, 6]], axis=1)
    masses = vals[:, 7].copy()
    pos = {int(i): k for k, i in enumerate(ids)}

    def resolve(lst):
        return [pos[i] for i in lst]

    bp = np.array([resolve(b[0]) for b in bonds], dtype=np.int32).reshape(-1, 2)
    bv = np.array([b[1] for b in bonds], dtype=np.float64).reshape(-1, 3)
    ap = np.array([resolve(a[0]) for a in angles], dtype=np.int32).reshape(-1, 3)
    av = np.array([[a[1][0] * F32_PI / 180, a[1][1]] for a in angles], dtype=np.float64).reshape(-1, 2)
    acp = np.array([resolve(a[0]) for a in angles_cos], dtype=np.int32).reshape(-1, 3)
    acv = np.array([[math.cos(a[1][0] * F32_PI / 180), a[1][1]] for a in angles_cos],
                   dtype=np.float64).reshape(-1, 2)
    dp = np.array([resolve(d[0]) for d in dihes], dtype=np.int32).reshape(-1, 4)
    dv = np.array([[-d[1][0] * d[1][2], d[1][1]] for d in dihes], dtype=np.float64).reshape(-1, 2)
    dap = np.array([resolve(d[0]) for d in dihe_angles], dtype=np.int32).reshape(-1, 4)
    # parse_dihe passes (temp[1], temp[0]) = (k, theta) to add_dihe_angle (input.c:631-635)
    dav = np.array([[d[1][1], d[1][0] * F32_PI / 180] for d in dihe_angles],
                   dtype=np.float64).reshape(-1, 2)
    deck = Deck(prm=prm, coord=coord, Q=Q, LJ=LJ, masses=masses, ids=ids,
                bond_pairs=bp, bond_parms=bv, angle_pairs=ap, angle_parms=av,
                angle_cos_pairs=acp, angle_cos_parms=acv, dihe_pairs=dp, dihe_parms=dv,
                dihe_angle_pairs=dap, dihe_angle_parms=dav, names=[s[2] for s in subs])
    _apply_options(deck)
    _center_coords(deck)
    _to_box(deck)
    _init_cutoff(deck)
    return deck


def _apply_options(d: Deck) -> None:
    p = d.prm
    if p["bc"] == BC["periodic"]:
        if p["xbox"] <= 0 or p["ybox"] <= 0 or p["zbox"] <= 0:
            raise ValueError("Wrong box size")
        d.inv_L = np.array([1 / p["xbox"], 1 / p["ybox"], 1 / p["zbox"], 0.0])
        d.box = np.array([p["xbox"], p["ybox"], p["zbox"], 0.0])
        d.ewald = int(p["hydro"] != HYDRO["none"])
        if d.ewald:
            if not (p["xbox"] == p["ybox"] == p["zbox"]):
                raise ValueError("In Ewald box must be cube")
            if np.any(d.LJ[:, 0] < d.coord[:, 3]):
                raise ValueError("LJ radii too small, should be at least 2 * bead radii")
            if p["ewald_real"] != p["ewald_recip"]:
                raise ValueError("ewald_real != ewald_recip")
            if not 0 <= p["ewald_real"] <= 5:
                raise ValueError("ewald_real wrong value, only 0..5")
    if len(set(d.ids.tolist())) != d.n:
        raise ValueError("Wrong atom numeration")
    if np.any(d.coord[:, 3] <= 0):
        raise ValueError("Wrong atom radii")
    if p["vfactor"] == 0 or p["visc"] == 0:
        raise ValueError("Wrong value for vfactor/visc")
    if p["hydro"] != HYDRO["geyer"] or p["algorithm"] >= ALGORITHM["igt_const"]:
        p["geyer_on_the_fly"] = 0


def _center_coords(d: Deck) -> None:
    """trans.c:38-99: shift the centre of mass to the origin (bc != none)."""
    if not d.prm["bc"]:
        return
    # sequential left-to-right sums, as the C loop accumulates them
    g = np.cumsum(d.coord[:, :3], axis=0)[-1] / d.n
    for i in range(3):
        lo, hi = d.coord[:, i].min(), d.coord[:, i].max()
        if d.prm["bc"] == BC["periodic"] and hi - lo > d.box[i]:
            raise ValueError("Particles don't fit in the box")
    # same summation order as the C loop: coord += (0 - g)
    d.coord[:, :3] += (0.0 - g)[None, :]
    if d.prm["bc"] == BC["sphere"]:
        # iscorrect (trans.c:130-145): every bead inside the sphere
        sq = d.coord[:, 0] * d.coord[:, 0] + d.coord[:, 1] * d.coord[:, 1] + d.coord[:, 2] * d.coord[:, 2]
        if np.any(sq > d.prm["sphere_radius"] * d.prm["sphere_radius"]):
            raise ValueError("Wrong correction")


def _to_box(d: Deck) -> None:
    """trans.c:101-107 applied to every bead (main_loop.c:63-66)."""
    if d.prm["bc"] != BC["periodic"]:
        return
    for i in range(3):
        v = d.coord[:, i]
        d.coord[:, i] = v - d.box[i] * np.floor(v * d.inv_L[i] + 0.5)


def _init_cutoff(d: Deck) -> None:
    """pre_func.c:197-232 (only used when nb_list != brute)."""
    p = d.prm
    if not p["nb_list"]:
        return
    m = 0.0
    f1 = _f32(0.01)
    if p["elec"]:
        m = p["cutoff_c"] + f1
    if p["alpha_lj"] != 0:
        if p["cutoff_lj"] == -1:
            for i in range(d.n):
                if 2 * _f32(1.1225) * d.LJ[i, 0] > m:
                    m = 2 * _f32(1.1225) * d.LJ[i, 0] + f1
        elif p["cutoff_lj"] > m:
            m = p["cutoff_lj"] + f1
    for i in range(d.n):
        if 2 * d.LJ[i, 0] > m:
            m = 2 * d.LJ[i, 0] + f1
    d.max_force_cutoff = m


# ---------------------------------------------------------------------------
# Seeded generators for the benchmark workloads
# ---------------------------------------------------------------------------

def saw_chain(n: int, step: float = 3.8, min_dist: float = 4.0, seed: int = 0) -> np.ndarray:
    """Self-avoiding random walk: unit steps of length ``step`` in uniformly
    random directions; every bead keeps ``min_dist`` from all beads except its
    chain predecessor. Rejected directions are redrawn; a dead end backs up."""
    rng = np.random.default_rng(seed)
    cell = min_dist
    grid: dict = {}
    pos = np.zeros((n, 3))

    def key(p):
        return (int(math.floor(p[0] / cell)), int(math.floor(p[1] / cell)), int(math.floor(p[2] / cell)))

    def ok(p, i):
        kx, ky, kz = key(p)
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for j in grid.get((kx + dx, ky + dy, kz + dz), ()):
                        if j == i - 1:
                            continue
                        if np.sum((pos[j] - p) ** 2) < min_dist * min_dist:
                            return False
        return True

    grid.setdefault(key(pos[0]), []).append(0)
    i = 1
    fails = 0
    while i < n:
        placed = False
        for _ in range(200):
            v = rng.normal(size=3)
            v *= step / np.linalg.norm(v)
            p = pos[i - 1] + v
            if ok(p, i):
                pos[i] = p
                grid.setdefault(key(p), []).append(i)
                placed = True
                break
        if placed:
            i += 1
            continue
        fails += 1
        back = min(i - 1, 1 + fails // 4)
        for j in range(i - back, i):
            grid[key(pos[j])].remove(j)
        i -= back
    return pos


def suspension(n: int, radius: float, phi: float, seed: int = 0):
    """Random sequential insertion of ``n`` spheres of ``radius`` into a cubic
    periodic box at volume fraction ``phi``; centres keep >= 2*radius apart
    under the minimum image. Returns (positions in [-L/2, L/2), L)."""
    L = (n * 4.0 / 3.0 * math.pi * radius ** 3 / phi) ** (1.0 / 3.0)
    rng = np.random.default_rng(seed)
    dmin2 = (2 * radius) ** 2
    nc = max(1, int(L // (2 * radius)))
    cs = L / nc
    grid: dict = {}
    pos = np.zeros((n, 3))
    k = 0
    while k < n:
        p = rng.uniform(-L / 2, L / 2, size=3)
        c = tuple(int((p[a] + L / 2) // cs) % nc for a in range(3))
        good = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for j in grid.get(((c[0] + dx) % nc, (c[1] + dy) % nc, (c[2] + dz) % nc), ()):
                        d = pos[j] - p
                        d -= L * np.round(d / L)
                        if d @ d < dmin2:
                            good = False
                            break
                    if not good:
                        break
                if not good:
                    break
            if not good:
                break
        if good:
            pos[k] = p
            grid.setdefault(c, []).append(k)
            k += 1
    return _balanced_images(pos, L), L


def _balanced_images(pos: np.ndarray, L: float) -> np.ndarray:
    """Pick, per axis, the periodic window [s, s+L) whose centre is the mean
    of the points inside it, and shift that window to [-L/2, L/2).

    BD_BOX recentres the centre of mass at the origin and rejects any bead
    that then lies outside the box (trans.c:38-99); this choice of images
    keeps every bead inside while describing the same periodic system."""
    out = np.empty_like(pos)
    n = pos.shape[0]
    for a in range(3):
        x = np.sort(pos[:, a])
        total = x.sum()
        s_found = None
        for k in range(-1, n):
            s = (total + (k + 1) * L) / n - L / 2
            lo = x[k] if k >= 0 else x[-1] - L
            hi = x[k + 1] if k + 1 < n else x[0] + L
            if lo < s <= hi:
                s_found = s
                break
        if s_found is None:
            raise RuntimeError("no balanced periodic window")
        v = pos[:, a]
        v = np.where(v < s_found, v + L, v)
        v = np.where(v >= s_found + L, v - L, v)
        out[:, a] = v - (s_found + L / 2)
    return out


CHAIN_FF = dict(radius=2.0, sigma_lj=4.0, eps_lj=0.1, r0=3.8, rmax=1.0e10, H=10.0,
                cutoff=12.0)


def _prm_lines(d: dict) -> str:
    return "".join(f"{k} {v}\n" for k, v in d.items())


def write_chain_deck(dirpath: str, name: str, n: int, seed: int, hydro: str = "cholesky",
                     dt: float = 0.01, steps: int = 1000, nb_list: str = "bucket_space",
                     extra: dict | None = None) -> str:
    """Linear bead-spring chain with the chain force field (harmonic bonds,
    LJ + Debye-Hueckel, charges +-1 drawn 50/50) in free space."""
    os.makedirs(dirpath, exist_ok=True)
    ff = CHAIN_FF
    pos = saw_chain(n, step=ff["r0"], min_dist=4.0, seed=seed)
    q = np.random.default_rng(seed + 7919).choice([-1.0, 1.0], size=n)
    strp = os.path.join(dirpath, name + ".str")
    with open(strp, "w") as f:
        for i in range(n):
            f.write(f"sub B {i + 1} {pos[i, 0]:.17g} {pos[i, 1]:.17g} {pos[i, 2]:.17g} "
                    f"{ff['radius']} {q[i]:.1f} {ff['sigma_lj']} {ff['eps_lj']} 1\n")
        for i in range(n - 1):
            f.write(f"bond {i + 1} {i + 2} {ff['r0']} {ff['rmax']:g} {ff['H']}\n")
    prm = {
        "str_filename": name + ".str", "dt": dt, "T": 293, "visc": 0.01, "vfactor": 14.4,
        "bdsteps": steps, "hydro": hydro, "algorithm": "ermak_const", "bc": "none",
        "elec": "yes", "epsilon_c": 78.54, "kappa_c": 0.1, "gamma_c": 331.842,
        "cutoff_c": ff["cutoff"], "alpha_lj": 4, "cutoff_lj": ff["cutoff"], "lj_6_term": "yes",
        "bond_lj_scale": 0, "bond_c_scale": 0, "check_overlap": "no", "nb_list": nb_list,
        "rand_seed": seed, "geyer_on_the_fly": "yes",
    }
    prm.update(extra or {})
    prmp = os.path.join(dirpath, name + ".prm")
    with open(prmp, "w") as f:
        f.write(_prm_lines(prm))
    return prmp


def write_suspension_deck(dirpath: str, name: str, n: int, seed: int, ewald_r: int = 3,
                          radius: float = 1.0, phi: float = 0.10, dt: float = 0.005,
                          steps: int = 500, extra: dict | None = None) -> str:
    """Periodic suspension of soft repulsive spheres (WCA LJ), Beenakker-Ewald
    RPY hydrodynamics with Geyer-Winter TEA noise."""
    os.makedirs(dirpath, exist_ok=True)
    pos, L = suspension(n, radius, phi, seed)
    strp = os.path.join(dirpath, name + ".str")
    with open(strp, "w") as f:
        for i in range(n):
            f.write(f"sub S {i + 1} {pos[i, 0]:.17g} {pos[i, 1]:.17g} {pos[i, 2]:.17g} "
                    f"{radius} 0 {2 * radius} 0.5 1\n")
    prm = {
        "str_filename": name + ".str", "dt": dt, "T": 293, "visc": 0.01, "vfactor": 14.4,
        "bdsteps": steps, "hydro": "geyer", "algorithm": "ermak_const", "bc": "periodic",
        "xbox": f"{L:.6f}", "ybox": f"{L:.6f}", "zbox": f"{L:.6f}",
        "ewald_method": "beenakker", "ewald_real": ewald_r, "ewald_recip": ewald_r,
        "elec": "no", "alpha_lj": 4, "cutoff_lj": -1, "lj_6_term": "yes",
        "check_overlap": "no", "nb_list": "bucket_space", "rand_seed": seed,
        "geyer_on_the_fly": "yes",
    }
    prm.update(extra or {})
    prmp = os.path.join(dirpath, name + ".prm")
    with open(prmp, "w") as f:
        f.write(_prm_lines(prm))
    return prmp


def replica_sizes(count: int = 256, lo: int = 64, hi: int = 1024, seed: int = 3) -> np.ndarray:
    """Bead counts of the batched-replica workload, uniform in [lo, hi]."""
    return np.random.default_rng(seed).integers(lo, hi + 1, size=count)
