"""ctypes binding of libbdb200.so and a host mirror of BD_BOX's hot-path API.

``System`` wraps one ``bdb_system`` (include/bdb200.h) built from a BD_BOX
deck. Its methods carry the names and meaning of the reference functions
they stand for:

=====================  ==========================================================
method                 reference
=====================  ==========================================================
``compute_forces``     compute_forces (potentials/calc_func.c:106-186)
``compute_D``          compute_D / compute_single_D (diff_alg/diff_tensor.c:472-544)
``compute_Dij``        compute_Dij (diff_tensor.c:437-470)
``compute_Rf``         compute_Rf (diff_alg/diff_equation.c:119-214)
``compute_r``          compute_r (diff_alg/diff_rand.c:47-236)
``step``               comp_step_ermak + compute_hydro_ermak, no retries
``compute_hydro``      comp_step_ermak with the overlap retry loop (diff_comp.c:152-179)
``save_curr_coord``    save_curr_coord + save_curr_forces (diff_decl.c:219-227)
``load_coord``         load_coord + load_forces (diff_decl.c:229-237)
=====================  ==========================================================

Errors raise ``BDBError`` instead of exiting (the reference's UNERR,
err.c:48-90). The CUDA library is required: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import decks as _decks

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbdb200.so")

PREC_FP64, PREC_MIXED = 0, 1
NOISE_PHILOX, NOISE_HOST = 0, 1

EXPORTS = [
    "bdb_version", "bdb_last_error", "bdb_create", "bdb_create_batch", "bdb_destroy", "bdb_set_bonded",
    "bdb_set_coord", "bdb_get_coord", "bdb_save_state", "bdb_load_state",
    "bdb_compute_forces", "bdb_compute_D", "bdb_compute_Dij", "bdb_compute_Rf",
    "bdb_compute_r", "bdb_step", "bdb_step_igt", "bdb_step_igt_predictor", "bdb_step_igt_corrector", "bdb_set_graphs", "bdb_set_dt", "bdb_adjoint", "bdb_autotune", "bdb_get_tuning",
    "bdb_set_tuning", "bdb_factor_error", "bdb_profile", "bdb_phase_stats",
    "bdb_reset_stats", "bdb_launches", "bdb_stream", "bdb_stored_matvec_noalloc", "bdb_shard_replicas",
    "bdb_frames_start", "bdb_frames_take", "bdb_frames_pending", "bdb_frames_flush", "bdb_frames_stop",
    "bdb_set_time", "bdb_get_time", "bdb_newton_resolve",
    "bdb_checkpoint_size", "bdb_checkpoint_save", "bdb_checkpoint_load", "bdb_refresh",
    "bdb_get_factor_tuning", "bdb_set_factor_tuning", "bdb_set_wait_limit", "bdb_cell_grid",
]


class BDBError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"bdb error {code}: {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("bc", C.c_int), ("box", C.c_double * 3),
        ("hydro", C.c_int), ("ewald", C.c_int), ("ewald_real", C.c_int),
        ("T", C.c_double), ("visc", C.c_double), ("vfactor", C.c_double), ("dt", C.c_double),
        ("elec", C.c_int), ("epsilon_c", C.c_double), ("kappa_c", C.c_double),
        ("gamma_c", C.c_double), ("cutoff_c", C.c_double),
        ("alpha_lj", C.c_double), ("cutoff_lj", C.c_double), ("lj_6_term", C.c_int),
        ("bond_lj_scale", C.c_double), ("bond_c_scale", C.c_double),
        ("check_overlap", C.c_int), ("nb_list", C.c_int), ("max_force_cutoff", C.c_double),
        ("precision", C.c_int), ("refresh", C.c_int), ("noise", C.c_int), ("seed", C.c_uint64),
        ("ewald_method", C.c_int), ("ewald_alpha", C.c_double),
        ("e_ext", C.c_int), ("e_type", C.c_int), ("e_dir1", C.c_int), ("e_dir2", C.c_int),
        ("e_factor", C.c_double), ("e_magn", C.c_double), ("e_freq", C.c_double),
        ("sboundary", C.c_int), ("sboundary_n", C.c_int), ("sboundary_A", C.c_double),
        ("sboundary_cutoff", C.c_double), ("sphere_radius", C.c_double),
        ("flow", C.c_int), ("vel_grad", C.c_double * 9),
    ]


_lib = None
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def load_library(path: str = LIB_PATH):
    """Load libbdb200.so; raise if it is missing (no fallback path exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `python -m bd_box_b200.build` (nvcc, sm_100a)")
    lib = C.CDLL(path)
    lib.bdb_version.restype = C.c_char_p
    lib.bdb_last_error.restype = C.c_char_p
    lib.bdb_create.argtypes = [C.POINTER(C.c_void_p), C.POINTER(Params), _dp, _dp, _dp]
    lib.bdb_create_batch.argtypes = [C.POINTER(C.c_void_p), C.POINTER(Params), C.c_int, _ip, _dp, _dp, _dp]
    lib.bdb_destroy.argtypes = [C.c_void_p]
    lib.bdb_set_bonded.argtypes = [C.c_void_p] + [C.c_int, _ip, _dp] * 5
    for name in ("bdb_set_coord", "bdb_get_coord"):
        getattr(lib, name).argtypes = [C.c_void_p, _dp]
    lib.bdb_save_state.argtypes = [C.c_void_p]
    lib.bdb_load_state.argtypes = [C.c_void_p]
    lib.bdb_compute_forces.argtypes = [C.c_void_p, _dp, _dp, C.POINTER(C.c_longlong)]
    lib.bdb_compute_D.argtypes = [C.c_void_p, _dp]
    lib.bdb_compute_Dij.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
    lib.bdb_compute_Rf.argtypes = [C.c_void_p, _dp]
    lib.bdb_compute_r.argtypes = [C.c_void_p, _dp, _dp]
    lib.bdb_step.argtypes = [C.c_void_p, C.c_int, _dp]
    lib.bdb_step_igt.argtypes = [C.c_void_p, C.c_int, _dp]
    lib.bdb_refresh.argtypes = [C.c_void_p, C.c_int]
    lib.bdb_step_igt_predictor.argtypes = [C.c_void_p, _dp]
    lib.bdb_step_igt_corrector.argtypes = [C.c_void_p, _dp]
    lib.bdb_set_dt.argtypes = [C.c_void_p, C.c_double]
    lib.bdb_set_graphs.argtypes = [C.c_void_p, C.c_int]
    lib.bdb_autotune.argtypes = [C.c_void_p, C.c_int]
    lib.bdb_get_tuning.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.bdb_set_tuning.argtypes = [C.c_void_p, C.c_int, C.c_int]
    lib.bdb_get_factor_tuning.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
    lib.bdb_set_wait_limit.argtypes = [C.c_void_p, C.c_longlong]
    lib.bdb_set_factor_tuning.argtypes = [C.c_void_p, C.c_int]
    lib.bdb_adjoint.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _ip, _dp, _dp, _dp, _dp]
    lib.bdb_factor_error.argtypes = [C.c_void_p, _dp]
    lib.bdb_profile.argtypes = [C.c_void_p, C.c_int]
    lib.bdb_phase_stats.argtypes = [C.c_void_p, C.c_char_p, _dp, C.POINTER(C.c_longlong)]
    lib.bdb_reset_stats.argtypes = [C.c_void_p]
    lib.bdb_launches.argtypes = [C.c_void_p, C.POINTER(C.c_longlong)]
    lib.bdb_cell_grid.argtypes = [C.c_void_p, C.c_int, _ip]
    lib.bdb_stream.argtypes = [C.c_void_p]
    lib.bdb_stream.restype = C.c_void_p
    lib.bdb_stored_matvec_noalloc.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                              C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.bdb_shard_replicas.argtypes = [C.c_int, _ip, C.c_int, _ip]
    lib.bdb_frames_start.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
    lib.bdb_frames_take.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_longlong), _dp, _dp, _dp, _ip]
    lib.bdb_frames_pending.argtypes = [C.c_void_p, _ip]
    lib.bdb_frames_flush.argtypes = [C.c_void_p]
    lib.bdb_set_time.argtypes = [C.c_void_p, C.c_double]
    lib.bdb_newton_resolve.argtypes = [C.c_void_p, C.c_double, _dp, C.c_int, _ip]
    lib.bdb_checkpoint_size.argtypes = [C.c_void_p]
    lib.bdb_checkpoint_size.restype = C.c_size_t
    lib.bdb_checkpoint_save.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
    lib.bdb_checkpoint_load.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
    lib.bdb_get_time.argtypes = [C.c_void_p, _dp]
    lib.bdb_frames_stop.argtypes = [C.c_void_p]
    _lib = lib
    return lib


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _ip_(a):
    return None if a is None or a.size == 0 else a.ctypes.data_as(_ip)


def params_from_deck(deck, precision=PREC_FP64, refresh=1, noise=NOISE_PHILOX, seed=None) -> Params:
    p = deck.prm
    P = Params()
    P.n = deck.n
    P.bc = p["bc"]
    for k in range(3):
        P.box[k] = deck.box[k]
    P.hydro = p["hydro"]
    P.ewald = deck.ewald
    P.ewald_real = p["ewald_real"]
    # the deck's ewald_method: 0 smith, 1 beenakker (diff_decl.c); the ABI's
    # BDB_EWALD_*: 0 beenakker, 1 smith
    P.ewald_method = 1 if p["ewald_method"] == 0 else 0
    P.ewald_alpha = p["ewald_alpha"]
    P.T, P.visc, P.vfactor, P.dt = p["T"], p["visc"], p["vfactor"], p["dt"]
    P.elec = p["elec"]
    P.epsilon_c, P.kappa_c, P.gamma_c, P.cutoff_c = p["epsilon_c"], p["kappa_c"], p["gamma_c"], p["cutoff_c"]
    P.alpha_lj, P.cutoff_lj, P.lj_6_term = p["alpha_lj"], p["cutoff_lj"], p["lj_6_term"]
    P.bond_lj_scale, P.bond_c_scale = p["bond_lj_scale"], p["bond_c_scale"]
    P.check_overlap = p["check_overlap"]
    P.nb_list = p["nb_list"]
    P.max_force_cutoff = deck.max_force_cutoff
    P.precision = precision
    P.refresh = refresh
    P.noise = noise
    P.seed = p["rand_seed"] if seed is None else seed
    P.e_ext = p["E_ext"]
    P.e_type = {"DC": 0, "AC": 1, "RF": 2}[p["E_type"]]
    P.e_dir1, P.e_dir2 = "xyz".index(p["E_dir1"][0]), "xyz".index(p["E_dir2"][0])
    P.e_factor, P.e_magn, P.e_freq = p["E_factor"], p["E_magn"], p["E_freq"]
    P.sboundary, P.sboundary_n = p["sboundary"], p["sboundary_n"]
    P.sboundary_A, P.sboundary_cutoff = p["sboundary_A"], p["sboundary_cutoff"]
    P.sphere_radius = p["sphere_radius"]
    G = _decks.vel_grad(p)
    if G is not None:
        P.flow = 1
        for k in range(9):
            P.vel_grad[k] = G[k]
    return P


class System:
    """One bead system resident on the current CUDA device, or, given a list
    of decks, a batch of independent replicas advanced together
    (bdb_create_batch; the parameters come from the first deck)."""

    def __init__(self, deck, precision=PREC_FP64, refresh=1, noise=NOISE_PHILOX, seed=None):
        self.lib = load_library()
        decks = list(deck) if isinstance(deck, (list, tuple)) else [deck]
        self.decks = decks
        self.deck = decks[0]
        self.counts = np.array([d.n for d in decks], dtype=np.int32)
        self.begins = np.concatenate([[0], np.cumsum(self.counts)[:-1]]).astype(np.int64)
        self.n = int(self.counts.sum())
        self.params = params_from_deck(self.deck, precision, refresh, noise, seed)
        self.params.n = self.n
        h = C.c_void_p()
        coord = np.ascontiguousarray(np.concatenate([d.coord for d in decks]), dtype=np.float64)
        Q = np.ascontiguousarray(np.concatenate([d.Q for d in decks]), dtype=np.float64)
        LJ = np.ascontiguousarray(np.concatenate([d.LJ for d in decks]), dtype=np.float64)
        if len(decks) == 1:
            rc = self.lib.bdb_create(C.byref(h), C.byref(self.params), _p(coord), _p(Q), _p(LJ))
        else:
            rc = self.lib.bdb_create_batch(C.byref(h), C.byref(self.params), len(decks),
                                           self.counts.ctypes.data_as(_ip), _p(coord), _p(Q), _p(LJ))
        self._check(rc)
        self.h = h
        names = ("bond", "angle", "angle_cos", "dihe", "dihe_angle")
        self._bonded = []
        for nm in names:
            pairs = [np.asarray(getattr(d, nm + "_pairs"), dtype=np.int32) + b for d, b in zip(decks, self.begins)]
            parms = [np.asarray(getattr(d, nm + "_parms"), dtype=np.float64) for d in decks]
            self._bonded.append(np.ascontiguousarray(np.concatenate(pairs), dtype=np.int32))
            self._bonded.append(np.ascontiguousarray(np.concatenate(parms), dtype=np.float64))
        b = self._bonded
        args = []
        for k in range(5):
            args += [len(b[2 * k]), _ip_(b[2 * k]), _p(b[2 * k + 1]) if b[2 * k + 1].size else None]
        self._check(self.lib.bdb_set_bonded(self.h, *args))

    def _check(self, rc):
        if rc < 0:
            raise BDBError(rc, self.lib.bdb_last_error().decode())
        return rc

    def close(self):
        if getattr(self, "h", None):
            self.lib.bdb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def n3(self):
        return 3 * self.n

    # -- state --------------------------------------------------------------
    def get_coord(self) -> np.ndarray:
        out = np.zeros((self.n, 4))
        self._check(self.lib.bdb_get_coord(self.h, _p(out)))
        return out

    def set_coord(self, coord):
        c = np.ascontiguousarray(coord, dtype=np.float64).reshape(self.n, 4)
        self._check(self.lib.bdb_set_coord(self.h, _p(c)))

    def save_curr_coord(self):
        self._check(self.lib.bdb_save_state(self.h))

    def load_coord(self):
        self._check(self.lib.bdb_load_state(self.h))

    # -- reference entry points --------------------------------------------
    def compute_forces(self, energies: bool = True):
        F = np.zeros(self.n3)
        E = np.zeros(9) if energies else None
        counts = (C.c_longlong * 2)()
        rep = self._check(self.lib.bdb_compute_forces(self.h, _p(F), _p(E), counts))
        return F, E, rep, (int(counts[0]), int(counts[1]))

    def compute_D(self) -> np.ndarray:
        D = np.zeros((self.n3, self.n3))
        self._check(self.lib.bdb_compute_D(self.h, _p(D)))
        return D

    def compute_Dij(self, i, j) -> np.ndarray:
        out = np.zeros(9)
        self._check(self.lib.bdb_compute_Dij(self.h, i, j, _p(out)))
        return out.reshape(3, 3)

    def compute_Rf(self) -> np.ndarray:
        out = np.zeros(self.n3)
        self._check(self.lib.bdb_compute_Rf(self.h, _p(out)))
        return out

    def compute_r(self, gauss=None) -> np.ndarray:
        out = np.zeros(self.n3)
        g = None if gauss is None else np.ascontiguousarray(gauss, dtype=np.float64)
        self._check(self.lib.bdb_compute_r(self.h, _p(g), _p(out)))
        return out

    def step(self, K: int = 1, gauss=None) -> int:
        g = None if gauss is None else np.ascontiguousarray(gauss, dtype=np.float64)
        return self._check(self.lib.bdb_step(self.h, K, _p(g)))

    def refresh(self, count: int = 1):
        """Rebuild the stored tensor and its Cholesky factor `count` times
        at the current positions (bdb_refresh)."""
        self._check(self.lib.bdb_refresh(self.h, int(count)))

    def step_igt(self, K: int = 1, gauss=None) -> int:
        """K IGT predictor-corrector steps (bdb_step_igt); gauss: K*2*3N
        host Gaussians (predictor then corrector per step) in host-noise
        mode. Returns the overlap flags (1: at the predicted positions, 2:
        after the step)."""
        g = None if gauss is None else np.ascontiguousarray(gauss, dtype=np.float64)
        return self._check(self.lib.bdb_step_igt(self.h, K, _p(g)))

    def igt_predictor(self, gauss=None) -> int:
        """The predictor half of an IGT step (bdb_step_igt_predictor);
        returns 1 when the forces at the predicted positions overlap."""
        g = None if gauss is None else np.ascontiguousarray(gauss, dtype=np.float64)
        return self._check(self.lib.bdb_step_igt_predictor(self.h, _p(g)))

    def igt_corrector(self, gauss=None) -> int:
        """The corrector of the pending IGT step, or again after an overlap,
        with fresh Gaussians (bdb_step_igt_corrector); returns 1 on an
        overlap."""
        g = None if gauss is None else np.ascontiguousarray(gauss, dtype=np.float64)
        return self._check(self.lib.bdb_step_igt_corrector(self.h, _p(g)))

    def compute_hydro(self, gauss_attempts=None, move_attempts=None) -> int:
        """One step with comp_step_ermak's retry loop: on an overlap the saved
        coordinates and forces come back and a new noise vector is drawn
        (dt halving of ermak_var is not modelled). Returns the attempts used."""
        limit = self.deck.prm["move_attempts"] if move_attempts is None else move_attempts
        count = 0
        self.save_curr_coord()
        while True:
            g = None if gauss_attempts is None else gauss_attempts[count]
            if not self.step(1, g):
                return count + 1
            self.load_coord()
            count += 1
            if count > limit:
                raise BDBError(-5, "Wrong conformation, can't move")

    def adjoint(self, K: int, checkpoint: int, pairs, targets):
        """bdb_adjoint: (loss, dloss/dx_0 as (N, 3), dloss/d scale factors
        (LJ epsilon, LJ sigma, bond H, Debye length))."""
        pairs = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
        targets = np.ascontiguousarray(targets, dtype=np.float64).reshape(-1)
        loss = C.c_double()
        gx = np.zeros(self.n3)
        gp = np.zeros(4)
        self._check(self.lib.bdb_adjoint(self.h, K, checkpoint, len(pairs), pairs.ctypes.data_as(_ip), _p(targets),
                                         C.byref(loss), _p(gx), _p(gp)))
        return loss.value, gx.reshape(self.n, 3), gp

    def autotune(self, enable: bool = True):
        self._check(self.lib.bdb_autotune(self.h, int(enable)))

    def tuning(self):
        """(TEA tile edge, stored-matvec warps per SM) in use."""
        a, b = C.c_int(), C.c_int()
        self._check(self.lib.bdb_get_tuning(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_tuning(self, tea_tile: int = 0, mv_warps_per_sm: int = 0):
        self._check(self.lib.bdb_set_tuning(self.h, tea_tile, mv_warps_per_sm))

    def set_wait_limit(self, tries: int):
        """Tries of every bounded device wait (bdb_set_wait_limit; < 0: the
        default)."""
        self._check(self.lib.bdb_set_wait_limit(self.h, int(tries)))

    def factor_tuning(self) -> int:
        """SMs the mixed Cholesky's bulk updates leave to its panel chain."""
        a = C.c_int()
        self._check(self.lib.bdb_get_factor_tuning(self.h, C.byref(a)))
        return a.value

    def set_factor_tuning(self, chain_sms: int):
        self._check(self.lib.bdb_set_factor_tuning(self.h, int(chain_sms)))

    def factor_error(self) -> float:
        out = C.c_double()
        self._check(self.lib.bdb_factor_error(self.h, C.byref(out)))
        return out.value

    def profile(self, enable: bool = True):
        self._check(self.lib.bdb_profile(self.h, int(enable)))

    def phase_stats(self, name="step"):
        """(total device ms, calls) of a profiled phase since the last reset."""
        tot = C.c_double()
        calls = C.c_longlong()
        self._check(self.lib.bdb_phase_stats(self.h, name.encode(), C.byref(tot), C.byref(calls)))
        return tot.value, calls.value

    def reset_stats(self):
        self._check(self.lib.bdb_reset_stats(self.h))

    def save_state(self):
        self._check(self.lib.bdb_save_state(self.h))

    def load_state(self):
        self._check(self.lib.bdb_load_state(self.h))

    def step_newton(self, K: int, gauss_attempts, masses=None, e_collision=None, move_attempts=None):
        """K ermak_newton steps as comp_step_ermak_newton runs them
        (diff_comp.c:181-210): a move that overlaps is redone by elastic
        collisions (bdb_newton_resolve) and, if that still overlaps, reverted
        to try the next Gaussians. gauss_attempts: host Gaussians, 3N per
        attempt, or None for device noise. Returns (attempts used, collision
        rounds)."""
        p = self.deck.prm
        m = np.ascontiguousarray(self.deck.masses if masses is None else masses, dtype=np.float64)
        e = p["e_collision"] if e_collision is None else e_collision
        ma = p["move_attempts"] if move_attempts is None else move_attempts
        g = None if gauss_attempts is None else np.ascontiguousarray(gauss_attempts, dtype=np.float64)
        used, rounds = 0, 0
        for _ in range(K):
            count = C.c_int(0)
            self.save_state()
            while True:
                gk = None if g is None else g[used * self.n3:(used + 1) * self.n3]
                if gk is not None and gk.size < self.n3:
                    raise BDBError(-1, "out of Gaussians")
                used += 1
                if self.step(1, gk) == 0:
                    break
                rc = self._check(self.lib.bdb_newton_resolve(self.h, e, _p(m), ma, C.byref(count)))
                if rc == 0:
                    break
                self.load_state()
            rounds += count.value
        return used, rounds

    def checkpoint(self) -> bytes:
        """The resume image (bdb_checkpoint_save)."""
        buf = C.create_string_buffer(self.lib.bdb_checkpoint_size(self.h))
        self._check(self.lib.bdb_checkpoint_save(self.h, buf, len(buf)))
        return buf.raw

    def restore(self, image: bytes):
        """Resume from an image of a system with the same parameters."""
        buf = C.create_string_buffer(bytes(image), len(image))
        self._check(self.lib.bdb_checkpoint_load(self.h, buf, len(image)))

    def set_time(self, t: float):
        self._check(self.lib.bdb_set_time(self.h, float(t)))

    def get_time(self) -> float:
        out = C.c_double()
        self._check(self.lib.bdb_get_time(self.h, C.byref(out)))
        return out.value

    # asynchronous trajectory frames (bdb_frames_*)
    def frames_start(self, every: int = 1, capacity: int = 16, energy: bool = False):
        self._frames_energy = bool(energy)
        self._check(self.lib.bdb_frames_start(self.h, int(every), int(capacity), int(bool(energy))))

    def frames_pending(self) -> int:
        out = C.c_int()
        self._check(self.lib.bdb_frames_pending(self.h, C.byref(out)))
        return out.value

    def frames_take(self, max_frames: int | None = None, flush: bool = False):
        """(steps, times, coords (k, N, 4), energies (k, 9) or None) of the
        finished frames, oldest first; with flush, after waiting for every
        copy in flight."""
        if flush:
            self._check(self.lib.bdb_frames_flush(self.h))
        m = self.frames_pending() if max_frames is None else int(max_frames)
        steps = np.zeros(max(m, 1), dtype=np.int64)
        times = np.zeros(max(m, 1))
        coord = np.zeros((max(m, 1), self.n, 4))
        energy = np.zeros((max(m, 1), 9)) if getattr(self, "_frames_energy", False) else None
        got = C.c_int()
        self._check(self.lib.bdb_frames_take(self.h, m, steps.ctypes.data_as(C.POINTER(C.c_longlong)), _p(times),
                                             _p(coord), _p(energy), C.byref(got)))
        k = got.value
        return steps[:k], times[:k], coord[:k], None if energy is None else energy[:k]

    def frames_stop(self):
        self._check(self.lib.bdb_frames_stop(self.h))

    def launches(self) -> int:
        out = C.c_longlong()
        self._check(self.lib.bdb_launches(self.h, C.byref(out)))
        return out.value

    def cell_grid(self, segment: int = 0):
        """(nx, ny, nz, all_pairs) of a segment's neighbour-cell grid after
        the last force evaluation (bdb_cell_grid)."""
        d = np.zeros(4, np.int32)
        self._check(self.lib.bdb_cell_grid(self.h, segment, d.ctypes.data_as(C.POINTER(C.c_int))))
        return tuple(int(x) for x in d)


def shard_replicas(beads, nshards: int) -> np.ndarray:
    """Shard index of every replica (bdb_shard_replicas): N^2 + N cost,
    longest-processing-time greedy, the same answer on every process."""
    lib = load_library()
    b = np.ascontiguousarray(beads, dtype=np.int32)
    out = np.zeros(b.size, dtype=np.int32)
    rc = lib.bdb_shard_replicas(b.size, _ip_(b), int(nshards), _ip_(out))
    if rc:
        raise BDBError(rc, lib.bdb_last_error().decode())
    return out


def open_deck(prm_path: str, overrides=None, **kw) -> System:
    return System(_decks.read_deck(prm_path, overrides), **kw)
