"""ctypes view of the C restatement (liboracle.so) -- TEST ORACLE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
the checker; the product path never imports this module. The library is
built by ``make -C oracle`` (gcc, no GPU); ``load()`` rebuilds it when it is
missing, so it also works on a machine that only received the sources.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class OrcSystem(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("coord", _dp), ("Q", _dp), ("LJ", _dp),
        ("bc", C.c_int), ("box", C.c_double * 3), ("inv_L", C.c_double * 3),
        ("hydro", C.c_int), ("T", C.c_double), ("visc", C.c_double), ("vfactor", C.c_double),
        ("ewald", C.c_int), ("ewald_method", C.c_int), ("ewald_real", C.c_int), ("ewald_alpha", C.c_double),
        ("elec", C.c_int), ("epsilon_c", C.c_double), ("kappa_c", C.c_double),
        ("gamma_c", C.c_double), ("cutoff_c", C.c_double),
        ("alpha_lj", C.c_double), ("cutoff_lj", C.c_double), ("lj_6_term", C.c_int),
        ("bond_lj_scale", C.c_double), ("bond_c_scale", C.c_double), ("check_overlap", C.c_int),
        ("n_bond", C.c_int), ("bond_pairs", _ip), ("bond_parms", _dp),
        ("n_angle", C.c_int), ("angle_pairs", _ip), ("angle_parms", _dp),
        ("n_angle_cos", C.c_int), ("angle_cos_pairs", _ip), ("angle_cos_parms", _dp),
        ("n_dihe", C.c_int), ("dihe_pairs", _ip), ("dihe_parms", _dp),
        ("n_dihe_angle", C.c_int), ("dihe_angle_pairs", _ip), ("dihe_angle_parms", _dp),
        ("e_ext", C.c_int), ("e_type", C.c_int), ("e_dir1", C.c_int), ("e_dir2", C.c_int),
        ("e_factor", C.c_double), ("e_magn", C.c_double), ("e_freq", C.c_double),
        ("sboundary", C.c_int), ("sboundary_n", C.c_int),
        ("sboundary_A", C.c_double), ("sboundary_cutoff", C.c_double), ("sphere_radius", C.c_double),
        ("t", C.c_double),
        ("flow", C.c_int), ("vel_grad", C.c_double * 9),
    ]


def load():
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "bdb_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    lib = C.CDLL(path)
    P = C.POINTER(OrcSystem)
    lib.orc_tile.argtypes = [P, C.c_int, C.c_int, _dp]
    lib.orc_D.argtypes = [P, _dp]
    lib.orc_cholesky.argtypes = [C.c_int, _dp, C.c_int]
    lib.orc_cholesky.restype = C.c_int
    lib.orc_trmv_lower.argtypes = [C.c_int, _dp, C.c_int, _dp, _dp]
    lib.orc_symv_upper.argtypes = [C.c_int, _dp, C.c_int, _dp, _dp]
    lib.orc_df.argtypes = [P, _dp, _dp, C.c_double, _dp]
    lib.orc_tea.argtypes = [P, _dp, _dp, C.c_double, _dp, _dp, _dp]
    lib.orc_forces.argtypes = [P, _dp, _dp, C.POINTER(C.c_longlong)]
    lib.orc_forces.restype = C.c_int
    lib.orc_run_steps.argtypes = [P, _dp, _dp, C.c_double, C.c_int, _dp, C.c_int, _dp]
    lib.orc_run_steps.restype = C.c_int
    lib.orc_run_igt_steps.argtypes = [P, _dp, _dp, C.c_double, C.c_int, _dp, _dp]
    lib.orc_run_igt_steps.restype = C.c_int
    lib.orc_run_newton_steps.argtypes = [P, _dp, _dp, C.c_double, C.c_int, _dp, C.c_int, _dp, C.c_double, C.c_int,
                                         _dp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.orc_run_newton_steps.restype = C.c_int
    _LIB = lib
    return lib


def _p(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _ip_(a):
    return a.ctypes.data_as(_ip)


class Oracle:
    """Oracle bound to one deck (bd_box_b200.decks.Deck)."""

    def __init__(self, deck):
        self.lib = load()
        self.deck = deck
        p = deck.prm
        self.coord = np.ascontiguousarray(deck.coord, dtype=np.float64).copy()
        self._keep = []

        def arr(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            if a.size == 0:
                a = np.zeros(1, dtype=dt)
            self._keep.append(a)
            return a

        s = OrcSystem()
        s.n = deck.n
        s.coord = _p(self.coord)
        s.Q = _p(arr(deck.Q, np.float64))
        s.LJ = _p(arr(deck.LJ, np.float64))
        s.bc = p["bc"]
        s.e_ext = p["E_ext"]
        s.e_type = {"DC": 0, "AC": 1, "RF": 2}[p["E_type"]]
        s.e_dir1, s.e_dir2 = "xyz".index(p["E_dir1"][0]), "xyz".index(p["E_dir2"][0])
        s.e_factor, s.e_magn, s.e_freq = p["E_factor"], p["E_magn"], p["E_freq"]
        s.sboundary, s.sboundary_n = p["sboundary"], p["sboundary_n"]
        s.sboundary_A, s.sboundary_cutoff = p["sboundary_A"], p["sboundary_cutoff"]
        s.sphere_radius = p["sphere_radius"]
        s.t = 0.0
        G = None if p.get("vel_grad_tensor") is None else [float(v) for v in str(p["vel_grad_tensor"]).split()]
        if G is not None and p["bc"] != 2:
            s.flow = 1
            for k in range(9):
                s.vel_grad[k] = G[k]
        for k in range(3):
            s.box[k] = deck.box[k]
            s.inv_L[k] = deck.inv_L[k]
        s.hydro = p["hydro"]
        s.T, s.visc, s.vfactor = p["T"], p["visc"], p["vfactor"]
        s.ewald = deck.ewald
        s.ewald_method = p["ewald_method"]
        s.ewald_real = p["ewald_real"]
        s.ewald_alpha = p["ewald_alpha"]
        s.elec = p["elec"]
        s.epsilon_c, s.kappa_c, s.gamma_c, s.cutoff_c = p["epsilon_c"], p["kappa_c"], p["gamma_c"], p["cutoff_c"]
        s.alpha_lj, s.cutoff_lj, s.lj_6_term = p["alpha_lj"], p["cutoff_lj"], p["lj_6_term"]
        s.bond_lj_scale, s.bond_c_scale, s.check_overlap = p["bond_lj_scale"], p["bond_c_scale"], p["check_overlap"]
        s.n_bond = len(deck.bond_pairs)
        s.bond_pairs = _ip_(arr(deck.bond_pairs, np.int32))
        s.bond_parms = _p(arr(deck.bond_parms, np.float64))
        s.n_angle = len(deck.angle_pairs)
        s.angle_pairs = _ip_(arr(deck.angle_pairs, np.int32))
        s.angle_parms = _p(arr(deck.angle_parms, np.float64))
        s.n_angle_cos = len(deck.angle_cos_pairs)
        s.angle_cos_pairs = _ip_(arr(deck.angle_cos_pairs, np.int32))
        s.angle_cos_parms = _p(arr(deck.angle_cos_parms, np.float64))
        s.n_dihe = len(deck.dihe_pairs)
        s.dihe_pairs = _ip_(arr(deck.dihe_pairs, np.int32))
        s.dihe_parms = _p(arr(deck.dihe_parms, np.float64))
        s.n_dihe_angle = len(deck.dihe_angle_pairs)
        s.dihe_angle_pairs = _ip_(arr(deck.dihe_angle_pairs, np.int32))
        s.dihe_angle_parms = _p(arr(deck.dihe_angle_parms, np.float64))
        self.s = s

    @property
    def n3(self):
        return 3 * self.deck.n

    def set_coord(self, coord):
        self.coord[...] = coord

    def tile(self, i, j):
        out = np.zeros(9)
        self.lib.orc_tile(C.byref(self.s), i, j, _p(out))
        return out.reshape(3, 3)

    def D(self):
        out = np.zeros((self.n3, self.n3))
        self.lib.orc_D(C.byref(self.s), _p(out))
        return out

    def forces(self):
        F = np.zeros(self.n3)
        E = np.zeros(9)
        counts = (C.c_longlong * 2)()
        rep = self.lib.orc_forces(C.byref(self.s), _p(F), _p(E), counts)
        return F, E, rep, (int(counts[0]), int(counts[1]))

    def df(self, F, dt, D=None):
        out = np.zeros(self.n3)
        self.lib.orc_df(C.byref(self.s), _p(D), _p(np.ascontiguousarray(F)), dt, _p(out))
        return out

    def tea(self, gauss, dt, D=None):
        Rs = np.zeros(self.n3)
        eps = C.c_double()
        beta = C.c_double()
        self.lib.orc_tea(C.byref(self.s), _p(D), _p(np.ascontiguousarray(gauss)), dt, _p(Rs),
                         C.pointer(eps), C.pointer(beta))
        return Rs, eps.value, beta.value

    def cholesky(self, A):
        L = np.ascontiguousarray(A, dtype=np.float64).copy()
        info = self.lib.orc_cholesky(L.shape[0], _p(L), L.shape[0])
        if info:
            raise np.linalg.LinAlgError(f"not SPD at pivot {info}")
        return np.tril(L)

    def run_steps(self, K, gauss, dt=None, refresh=1, F=None):
        dt = self.deck.prm["dt"] if dt is None else dt
        if F is None:
            F, _, _, _ = self.forces()
        F = np.ascontiguousarray(F, dtype=np.float64).copy()
        traj = np.zeros((K, self.deck.n, 4))
        g = np.ascontiguousarray(gauss, dtype=np.float64)
        rep = self.lib.orc_run_steps(C.byref(self.s), _p(self.coord), _p(F), dt, K, _p(g), refresh, _p(traj))
        return traj, F, rep

    def run_newton_steps(self, K, gauss, masses=None, e_collision=None, move_attempts=None, dt=None, F=None):
        """K ermak_newton steps (orc_run_newton_steps); gauss holds 3N
        Gaussians per attempt. Returns (traj, F, rc, blocks used, collision
        rounds)."""
        p = self.deck.prm
        dt = p["dt"] if dt is None else dt
        if F is None:
            F, _, _, _ = self.forces()
        F = np.ascontiguousarray(F, dtype=np.float64).copy()
        m = np.ascontiguousarray(self.deck.masses if masses is None else masses, dtype=np.float64)
        traj = np.zeros((K, self.deck.n, 4))
        g = np.ascontiguousarray(gauss, dtype=np.float64)
        used, rounds = C.c_int(), C.c_int()
        rc = self.lib.orc_run_newton_steps(C.byref(self.s), _p(self.coord), _p(F), dt, K, _p(g), g.size // self.n3,
                                           _p(m), p["e_collision"] if e_collision is None else e_collision,
                                           p["move_attempts"] if move_attempts is None else move_attempts,
                                           _p(traj), C.byref(used), C.byref(rounds))
        return traj, F, rc, used.value, rounds.value

    def run_igt_steps(self, K, gauss, dt=None, F=None):
        """K IGT predictor-corrector steps (orc_run_igt_steps); gauss holds
        K*2*3N Gaussians, the predictor's then the corrector's per step."""
        dt = self.deck.prm["dt"] if dt is None else dt
        if F is None:
            F, _, _, _ = self.forces()
        F = np.ascontiguousarray(F, dtype=np.float64).copy()
        traj = np.zeros((K, self.deck.n, 4))
        g = np.ascontiguousarray(gauss, dtype=np.float64)
        rep = self.lib.orc_run_igt_steps(C.byref(self.s), _p(self.coord), _p(F), dt, K, _p(g), _p(traj))
        return traj, F, rep
