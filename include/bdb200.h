/* bdb200 -- B200-native Brownian-dynamics step for BD_BOX decks (C ABI).
 *
 * Two layers are declared here.
 *
 * 1. The engine ABI (bdb_*): plain pointers and sizes, no CUDA or torch
 *    types. One bdb_system holds one bead system (or a batch of independent
 *    replicas) resident on the current CUDA device. Host arrays use BD_BOX's
 *    layouts: coord is double[4N] (x, y, z, hydrodynamic radius; data.h:315),
 *    Q double[N], LJ double[2N] (sigma_LJ/2, epsilon_LJ; data.c:97-100),
 *    forces double[3N], energies double[BDB_E_LAST+1] indexed like
 *    enum ENERGY_TYPE (data.h:278-289), diffusion tensors double[3N*3N]
 *    row-major and symmetric.
 *
 * 2. The BD_BOX drop-in (libbdb200_bdbox.a): the reference's own extern "C"
 *    entry points of src/diff_alg and src/potentials (diff_tensor.h:166-253,
 *    calc_func.h:60-106), implemented on the engine and linked in place of
 *    the CPU translation units, exactly as BD_BOX swaps its CUDA build in
 *    (src/Makefile.am:44-78). Those symbols read and write BD_BOX's
 *    globals, so their declarations are BD_BOX's own headers; they are
 *    defined in bd_box_b200/dropin/bdbox_dropin.c.
 *
 * Every bdb_* call returns BDB_OK (0) or a negative BDB_ERR_* code;
 * bdb_last_error() gives the message of the last failure on this thread.
 * No call exits the process (the reference's UNERR, err.c:48-90, does).
 */
#ifndef BDB200_H
#define BDB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BDB_OK 0
#define BDB_ERR_ARG (-1)       /* invalid argument or size */
#define BDB_ERR_CUDA (-2)      /* CUDA runtime error */
#define BDB_ERR_NOT_SPD (-3)   /* Cholesky met a non-positive pivot (diff_rand.c:78-79) */
#define BDB_ERR_BOND (-4)      /* over-stretched FENE bond (bond.c:73-78) */
#define BDB_ERR_STATE (-5)     /* call out of order (e.g. no coordinates yet) */
#define BDB_ERR_NOMEM (-6)     /* device allocation failed */
#define BDB_ERR_TIMEOUT (-7)   /* a bounded device wait gave up */
#define BDB_ERR_UNSUPPORTED (-8)

/* energy slots, enum ENERGY_TYPE (data.h:278-289) */
enum { BDB_E_NONE, BDB_E_BOND, BDB_E_ANGLE, BDB_E_ANGLE_COS, BDB_E_DIHE,
       BDB_E_DIHE_ANGLE, BDB_E_LJ, BDB_E_COULOMB, BDB_E_LAST };

/* hydrodynamic methods, DIFF_* (diff_tensor.h:44-52) */
enum { BDB_HYDRO_NONE = 0, BDB_HYDRO_CHOLESKY = 1, BDB_HYDRO_GEYER = 2 };
/* Ewald-summed tensor (ewald_method, diff_decl.c): Beenakker
 * (diff_tensor.c:265-422) or Smith (:102-263) */
enum { BDB_EWALD_BEENAKKER = 0, BDB_EWALD_SMITH = 1 };

/* arithmetic of the diffusion part of the step */
enum {
    BDB_PREC_FP64 = 0,   /* everything in FP64 (the plain GPU path) */
    BDB_PREC_MIXED = 1   /* FP32 tensor and stored D/L, FP16-split tcgen05 Cholesky
                            updates with FP64 diagonal tiles, FP64 sums */
};

/* noise sources */
enum {
    BDB_NOISE_PHILOX = 0,  /* Philox-4x32-10 Gaussians generated on the device */
    BDB_NOISE_HOST = 1     /* caller passes 3N Gaussians per step (parity runs) */
};

/* Parameters of one system: the .prm keys the hot path reads (after BD_BOX's
 * float rounding of DOUBLE keys, input.c:1010-1013) plus engine choices. */
typedef struct {
    int n;                    /* beads */
    int bc;                   /* 0 none, 1 periodic box, 2 sphere (trans.h:43-63) */
    double box[3];            /* xbox, ybox, zbox */
    int hydro;                /* BDB_HYDRO_* */
    int ewald;                /* 1: Ewald-summed tensor (periodic, hydro != none), see ewald_method */
    int ewald_real;           /* lattice radius R (ewald_real == ewald_recip, 0..5) */
    double T, visc, vfactor, dt;
    int elec;                 /* Debye-Hueckel on */
    double epsilon_c, kappa_c, gamma_c, cutoff_c;
    double alpha_lj, cutoff_lj;
    int lj_6_term;
    double bond_lj_scale, bond_c_scale;
    int check_overlap;
    int nb_list;              /* 0 all pairs, otherwise cell list */
    double max_force_cutoff;  /* cell size (init_cutoff, pre_func.c:197-232) */
    /* engine choices; no reference counterpart */
    int precision;            /* BDB_PREC_* */
    int refresh;              /* rebuild D and its factor every `refresh` steps (>= 1) */
    int noise;                /* BDB_NOISE_* */
    uint64_t seed;            /* Philox key */
    int ewald_method;         /* BDB_EWALD_* (after the engine choices, so that zeroed structs mean Beenakker) */
    double ewald_alpha;       /* Smith's splitting parameter in units of 1/L (ewald_alpha; <= 0: sqrt(pi)) */
    /* external forces, added per bead after the bonded terms (bonded_inter,
     * pre_func.c:135-158); zeroed structs switch them off */
    int e_ext;                /* E_ext: field on charged beads (electro_ext_force, electro_ext.c:38-51) */
    int e_type;               /* E_type: 0 DC, 1 AC (cos), 2 RF (cos on e_dir1, sin on e_dir2) */
    int e_dir1, e_dir2;       /* E_dir1, E_dir2: 0 x, 1 y, 2 z */
    double e_factor, e_magn, e_freq;   /* E_factor, E_magn, E_freq */
    int sboundary;            /* bounding-sphere force, bc 2 only (sboundary_ext, sboundary.c:36-73) */
    int sboundary_n;          /* sboundary_n >= 0 */
    double sboundary_A, sboundary_cutoff;
    double sphere_radius;     /* bc 2: the reflective sphere around the origin (trans.c:35) */
    /* flowing solvent (vel_grad_tensor, diff_decl.c:72): each Ermak step adds
     * dt G r, r the bead's start position (diff_equation.c:265-283); an IGT
     * corrector adds half the predictor's flow displacement (:303-311); off
     * with bc 2, as BD_BOX turns it off there (input.c:462-468) */
    int flow;
    double vel_grad[9];       /* G, row-major */
} bdb_params;

typedef struct bdb_system bdb_system;

/* Library identity and the last error message on this thread. */
const char* bdb_version(void);
const char* bdb_last_error(void);

/* Create a system on the current device from host arrays (copied).
 * Replaces init_diff_tensor (diff_decl.c:83-175) + init_forces
 * (calc_func.c:411-415) + init_cuda (cuda.c:88-148). */
int bdb_create(bdb_system** out, const bdb_params* p, const double* coord,
               const double* Q, const double* LJ);
int bdb_destroy(bdb_system* s);   /* free_diff_tensor + free_forces + free_cuda */

/* A batch of nseg independent systems (replicas) that share the parameters
 * and advance together, every kernel of a step covering all of them. Beads
 * are stored back to back: segment g holds counts[g] >= 2 beads, p->n is
 * their sum, and coord/Q/LJ are the concatenated host arrays. Each segment
 * has its own cell list, tensor tiles and TEA normalisation (eps, beta);
 * bonded terms may not join two segments. Overlap flags and energies are
 * summed over the batch. hydro cholesky is single-system only
 * (BDB_ERR_UNSUPPORTED); bdb_compute_D is not formed for a batch. No
 * reference counterpart: BD_BOX runs one system per process. */
int bdb_create_batch(bdb_system** out, const bdb_params* p, int nseg, const int* counts,
                     const double* coord, const double* Q, const double* LJ);

/* Asynchronous trajectory frames (no reference counterpart; BD_BOX writes
 * XYZ/DCD frames from the host coord after each saved step, output.c:64-100
 * and save_output :250-257, which needs the positions on the host every
 * such step). bdb_frames_start records the current state as a frame, then
 * the state after every `every`-th step of bdb_step / bdb_step_igt, by an
 * asynchronous copy into a ring of `capacity` pinned host frames: no step
 * waits for output. With with_energy, each frame also carries the energies
 * at its positions (a force pass with energies on each saved step, as BD_BOX
 * forms E only on the steps it writes, main_loop.c:102-112).
 * bdb_frames_take hands over up to max_frames finished frames, oldest
 * first, without blocking: steps[i] (steps since the system was created),
 * times[i] (simulated time, the sum of dt), coord[4N * i ..] (x, y, z,
 * radius per bead, BD_BOX's coord layout), energies[(BDB_E_LAST + 1) * i ..]
 * (may be NULL; ignored without with_energy); *nframes is how many.
 * When the ring is full, recording the next frame waits for the oldest one
 * and keeps it on the host, so frames are never dropped. bdb_frames_pending
 * counts frames not yet taken, finished or not; bdb_frames_flush waits for
 * every copy in flight; bdb_frames_stop (and bdb_destroy) free the ring,
 * discarding frames not taken. Starting again discards the old ring. */
int bdb_frames_start(bdb_system* s, int every, int capacity, int with_energy);
int bdb_frames_take(bdb_system* s, int max_frames, long long* steps, double* times, double* coord,
                    double* energies, int* nframes);
int bdb_frames_pending(bdb_system* s, int* nframes);
int bdb_frames_flush(bdb_system* s);
int bdb_frames_stop(bdb_system* s);

/* Elastic-collision overlap removal (algorithm ermak_newton): the recovery
 * of comp_step_ermak_newton (diff_comp.c:181-210) after a step whose move
 * overlapped, with the step's start saved by bdb_save_state. Velocities
 * v = (r - r_start) / dt and r = r_start (newton_init_vel, newton.c:202-213),
 * then ballistic moves to just before the earliest contact of approaching
 * pairs and elastic collisions of the pairs that reach it (restitution
 * e_collision, bead masses[N]), until dt has elapsed (newton_moves and
 * comp_time, newton.c:57-200); then the forces at the result. *count
 * accumulates the collision rounds of the step (BD_BOX's count); more than
 * move_attempts fails ("Ermak Newton error"). Returns 0 when the result is
 * free of overlaps, 1 when not (the caller restores the start with
 * bdb_load_state and tries new Gaussians, as BD_BOX does), < 0 on error.
 * bdb_save_state / bdb_load_state also keep the step count and the time. */
int bdb_newton_resolve(bdb_system* s, double e_collision, const double* masses, int move_attempts, int* count);

/* Checkpoints for resume (no reference counterpart; BD_BOX's restart files,
 * restart.c:315-486, hold its globals, coordinates and RNG state). The
 * image holds the positions, the Philox stream index, the step count, the
 * time, dt and the refresh phase; bdb_checkpoint_size gives its bytes.
 * bdb_checkpoint_load restores it into a system created with the same
 * parameters and bead count. Forces are recomputed and a stored tensor and
 * its factor are rebuilt at the next step, so a resumed run repeats the
 * uninterrupted one (to round-off: the cell lists are rebuilt) when the
 * image was taken at the end of a refresh interval or with refresh 1. */
size_t bdb_checkpoint_size(bdb_system* s);
int bdb_checkpoint_save(bdb_system* s, void* buf, size_t bytes);
int bdb_checkpoint_load(bdb_system* s, const void* buf, size_t bytes);

/* Simulated time of the current state (curr_time, main_loop.c:47): the
 * time-dependent field (E_type AC, RF) acts at curr_time + dt on the forces
 * after a step (diff_comp.c:161). Steps advance it by dt; a host that keeps
 * its own clock (a restart, BD_BOX's curr_time) sets it here. */
int bdb_set_time(bdb_system* s, double t);
int bdb_get_time(bdb_system* s, double* t);

/* Replicas over processes (one per GPU): shard_of[k] in [0, nshards) for
 * replica k of beads[k] beads, balancing the per-step cost, taken as N^2
 * (the tensor tiles, TEA and D.F of a replica) plus N (forces, noise,
 * update). Longest-processing-time greedy: replicas in decreasing cost
 * (ties: lower index first) go to the least-loaded shard (ties: lower
 * shard), so every process computes the same answer without a collective;
 * the largest load is at most 4/3 of the optimum. Host-only, needs no
 * device. No reference counterpart: BD_BOX's MPI ranks split the pair
 * loops of one system (diff_tensor.c:486, calc_func.c:205). */
int bdb_shard_replicas(int nrep, const int* beads, int nshards, int* shard_of);

/* Bonded terms, BD_BOX's arrays as read by read_str_file (input.c:567-641):
 * bond_pairs int[2B], bond_parms double[3B] (r0, rmax, H) (bond.c:94-111);
 * angle_pairs int[3A], angle_parms double[2A] (phi0 [rad], k) (angle.c:88-100);
 * angle_cos_* (cos phi0, k) (angle_cos.c:84-97); dihe_pairs int[4D],
 * dihe_parms (-k*delta, m) (dihe.c:188-209); dihe_angle_* (k, theta0 [rad])
 * (dihe_angle.c:257-276). Counts may be 0 and pointers NULL. */
int bdb_set_bonded(bdb_system* s,
                   int n_bond, const int* bond_pairs, const double* bond_parms,
                   int n_angle, const int* angle_pairs, const double* angle_parms,
                   int n_angle_cos, const int* angle_cos_pairs, const double* angle_cos_parms,
                   int n_dihe, const int* dihe_pairs, const double* dihe_parms,
                   int n_dihe_angle, const int* dihe_angle_pairs, const double* dihe_angle_parms);

/* Host <-> device coordinates (double[4N]); save_curr_coord/load_coord
 * (diff_decl.c:219-237) keep a device copy instead. */
int bdb_set_coord(bdb_system* s, const double* coord);
int bdb_get_coord(bdb_system* s, double* coord);
int bdb_save_state(bdb_system* s);     /* save_curr_coord + save_curr_forces */
int bdb_load_state(bdb_system* s);     /* load_coord + load_forces */

/* compute_forces (calc_func.c:106-186): forces at the current coordinates
 * into the device force buffer; optional host copies of F (3N), E
 * (BDB_E_LAST+1) and the pair counts {pairs with r <= cutoff_c, pairs in the
 * LJ range of force_single (calc_func.c:378-395)}. Returns the overlap/NaN
 * flag (0 or 1) or a negative error. */
int bdb_compute_forces(bdb_system* s, double* F, double* E, long long* counts);

/* The neighbour-cell grid of a segment (system or replica) as the last force
 * evaluation built it: dims[0..2] cells along x, y, z, dims[3] 1 where the
 * segment takes all pairs instead (a grid of fewer than 3 periodic cells
 * along an axis, or a non-finite coordinate). BD_BOX keeps its bucket grid
 * internal (bucket.c:173-379, bucket_space); this query is for checking that
 * a large system uses cells. Synchronises the system's stream. */
int bdb_cell_grid(bdb_system* s, int segment, int* dims);

/* compute_D / compute_single_D (diff_tensor.c:472-544): the full symmetric
 * 3N x 3N tensor at the current coordinates, row-major, into host D. */
int bdb_compute_D(bdb_system* s, double* D);

/* compute_Dij (diff_tensor.c:437-470): one 3x3 tile, row-major. */
int bdb_compute_Dij(bdb_system* s, int i, int j, double* tD);

/* compute_Rf (diff_equation.c:119-214): Rf = dt/(kB T) D.F with the current
 * forces, into host Rf (3N). Cholesky systems use the stored D (rebuilt if
 * stale), Geyer/none recompute the tiles on the fly. */
int bdb_compute_Rf(bdb_system* s, double* Rf);

/* compute_r (diff_rand.c:47-236): random displacement Rs (3N) from 3N unit
 * Gaussians `gauss` (host; NULL draws Philox), into host Rs. */
int bdb_compute_r(bdb_system* s, const double* gauss, double* Rs);

/* Ermak-McCammon steps (comp_step_ermak + compute_hydro_ermak,
 * diff_comp.c:152-179, diff_equation.c:216-286): K steps on the device.
 * gauss: K*3N host Gaussians when noise == BDB_NOISE_HOST, else NULL.
 * Returns the OR of the overlap flags of the steps (retries are the
 * caller's, as in comp_step_ermak) or a negative error. */
int bdb_step(bdb_system* s, int K, const double* gauss);

/* The refresh of the stored-tensor path that bdb_step runs every `refresh`
 * steps -- compute_D (diff_tensor.c:472-544) then the Cholesky factor of
 * compute_r (diff_rand.c:64-85) -- `count` times at the current positions,
 * replayed from its CUDA graph after the first (mixed precision), on the
 * system's stream; the next bdb_step reuses the last factor for `refresh`
 * steps. For timing the refresh by itself. BDB_ERR_UNSUPPORTED unless
 * hydro is cholesky. */
int bdb_refresh(bdb_system* s, int count);

/* IGT predictor-corrector steps (comp_step_IGT_const, diff_comp.c:76-107;
 * compute_hydro_IGT + compute_hydro_IGT_second_phase,
 * diff_equation.c:288-374) for hydro none or cholesky (one system): a
 * predictor Ermak-McCammon step to r', forces and D(r') F' there, then
 * r += (D(r)F + D(r')F') dt/(2 kB T) + L X2 with L the Cholesky factor of
 * (D(r) + D(r'))/2 and fresh Gaussians; D is rebuilt and factored twice per
 * step (the refresh interval does not apply). gauss: K*2*3N host Gaussians
 * (predictor then corrector, per step) when noise == BDB_NOISE_HOST, else
 * NULL. Returns the OR over the steps of 1 (overlap in the forces at r') and
 * 2 (overlap after the step), or a negative error; retries are the
 * caller's. */
int bdb_step_igt(bdb_system* s, int K, const double* gauss);

/* One IGT step in two calls, for callers that retry like
 * comp_step_IGT_const (diff_comp.c:76-107); gauss: 3N host Gaussians, or
 * NULL for Philox. bdb_step_igt_predictor is compute_hydro_IGT up to the
 * corrector (diff_equation.c:317-368): the predictor, forces at r' and,
 * unless they overlap (return 1), D(r') F' and the factor of the averaged
 * tensor. bdb_step_igt_corrector is compute_hydro_IGT_second_phase
 * (:288-315): from the step's start positions, fresh Gaussians with that
 * factor and deterministic displacement, then forces; it may be called again
 * after an overlap (return 1). Both return 0 otherwise, or a negative
 * error. */
int bdb_step_igt_predictor(bdb_system* s, const double* gauss);
int bdb_step_igt_corrector(bdb_system* s, const double* gauss);

/* Autotuner (no reference counterpart). With autotuning on, the first use
 * of each tunable site times its candidates on the system's stream and
 * keeps the fastest: the TEA tile edge (16 or 32 beads; the matrix-free
 * D.F and TEA noise) and the column segmentation of the FP64 stored-matrix
 * product (8, 16 or 32 warps per SM; the mixed-precision product is a
 * persistent kernel with one CTA per SM and ignores it). Different choices
 * sum in different orders, so results can differ at rounding level between
 * tuned runs; bdb_set_tuning pins the values (0 keeps one) and
 * bdb_get_tuning reports them. Off by default (32-bead tiles, 16 warps per
 * SM).
 * Switch it on before the first step. */
int bdb_autotune(bdb_system* s, int enable);
int bdb_get_tuning(bdb_system* s, int* tea_tile, int* mv_warps_per_sm);
int bdb_set_tuning(bdb_system* s, int tea_tile, int mv_warps_per_sm);

/* Bounded device waits (no reference counterpart). Every wait of this
 * system's kernels on another warp's or the copy engine's progress (mbarrier
 * try_wait loops in the tensor-core Cholesky, its diagonal-block kernel and
 * the TMA-fed stored-matrix product) gives up after `tries` tries (default
 * 2^22, restored by a negative value): the kernel then sets its time-out
 * flag, lets the copies and tensor-core operations it has in flight finish,
 * frees its tensor memory and returns, and the call reports
 * BDB_ERR_TIMEOUT with the context still usable; the next step rebuilds the
 * factor. 0 makes every such wait give up at once, which tests that path
 * without a hung GPU. */
int bdb_set_wait_limit(bdb_system* s, long long tries);

/* The third tunable site (no reference counterpart): how the mixed-precision
 * Cholesky splits the GPU. Its panel chain (panel solve, next block-column
 * update, next diagonal block) runs beside the bulk trailing updates, which
 * leave chain_sms SMs to it (16, 24, 32, 40, 48, 56 or 64 tried at the first
 * refresh when autotuning is on, each as a replayed refresh graph; 32
 * otherwise; 16 on the FP64 path, which is not tuned).
 * bdb_set_factor_tuning pins it (0 keeps the value). */
int bdb_get_factor_tuning(bdb_system* s, int* chain_sms);
int bdb_set_factor_tuning(bdb_system* s, int chain_sms);

/* CUDA graphs (no reference counterpart). Mode bit 1: steps (profiling
 * off) replay the steady part of a step -- noise, D.F and the random
 * displacement, the update, the forces -- from a graph captured on the
 * second step; steps with caller Gaussians use a second graph that reads
 * them from a fixed device staging slot. Bit 2: on the mixed path, refreshes of
 * D and its factor (tensor build and the three-stream factorisation) replay a
 * graph captured on the second refresh. Default 3 (both); 0 runs
 * everything eagerly. */
int bdb_set_graphs(bdb_system* s, int mode);

/* Time step of the following steps (curr_dt, diff_decl.c:68): the variable
 * step of comp_step_ermak halves it on overlap (diff_comp.c:162-165). */
int bdb_set_dt(bdb_system* s, double dt);

/* Hand-written adjoint of K Ermak-McCammon steps (no reference counterpart).
 * From the current state, runs K device-noise steps (Philox noise, a fixed
 * sequence given the seed and the stream position at the call), evaluates
 * loss = (1/P) sum_p (|x_{b_p} - x_{a_p}| - targets[p])^2 at the final
 * positions (pairs int[2P] = a_0, b_0, a_1, ...), and propagates it back
 * through every step -- D(x) F(x), the forces and the Cholesky noise factor
 * B(x) X -- recomputing the forward pass from the positions saved every
 * `checkpoint` steps. Outputs: *loss, grad_coord[3N] = dloss/dx_0 and
 * grad_params[4] = dloss/ds for scale factors s multiplying every bead's LJ
 * epsilon, every bead's LJ sigma, every bond's H and the Debye length 1/kappa
 * (so dloss/d epsilon = grad_params[0] / epsilon for a uniform epsilon).
 * Leaves the system at the final positions. Needs one free-space system,
 * hydro cholesky, BDB_PREC_FP64, refresh 1, BDB_NOISE_PHILOX, and bonds as
 * the only bonded terms (else BDB_ERR_UNSUPPORTED). */
int bdb_adjoint(bdb_system* s, int K, int checkpoint, int npairs, const int* pairs,
                const double* targets, double* loss, double* grad_coord, double* grad_params);

/* Cholesky of the stored tensor at the current coordinates (diagnostics):
 * rel_err = ||L L^T - D||_F / ||D||_F evaluated on the device in FP64. */
int bdb_factor_error(bdb_system* s, double* rel_err);

/* Measurement hooks (no reference counterpart). With profiling on, every
 * phase of a step is bracketed by CUDA events on the system's stream;
 * bdb_phase_stats returns the summed device time in ms and the number of
 * calls of a phase since the last reset: "step" (whole bdb_step calls),
 * "refresh" (tensor build + Cholesky), "build", "factor", "matvec", "tea",
 * "forces", "noise", "update". bdb_launches counts kernel launches issued
 * since the system was created (or the last reset). */
int bdb_profile(bdb_system* s, int enable);
int bdb_phase_stats(bdb_system* s, const char* phase, double* total_ms, long long* calls);
int bdb_reset_stats(bdb_system* s);
int bdb_launches(bdb_system* s, long long* count);

/* The CUDA stream all work of this system is issued on (cudaStream_t). */
void* bdb_stream(bdb_system* s);

/* No-allocation variant of the Cholesky path's per-step products; it has no
 * counterpart in the reference. For callers that cannot call cudaMalloc --
 * a host whose device memory is entirely owned by its own pool allocator, or
 * a real-time loop that must not allocate -- this computes, on buffers the
 * caller already owns (all device pointers):
 *     Rf = pre * (D F)   and   Rs = L X
 * from an FP32 matrix M (ld floats per row, 16-byte aligned, ld a multiple
 * of 4) whose strict upper triangle holds D, whose lower triangle including
 * the diagonal holds its Cholesky factor L, and from dD = diag(D). It
 * allocates nothing: its partial sums live in a fixed array in the
 * library's device memory (2.5 MB on every device that loads the library,
 * held until the process exits), so 3N is limited to 3072 (1024 beads) and
 * larger sizes are rejected with BDB_ERR_ARG. The first call on a device
 * looks up that array's device address (cudaGetSymbolAddress) and the SM
 * count, and looks them up again after the device's context has been
 * destroyed and created anew (cudaDeviceReset); make that first call before
 * any stream capture. All calls share the array: calls
 * whose work overlaps on the GPU (different streams, or different host
 * threads) race and must be serialised by the caller. `stream` is a
 * cudaStream_t or NULL for the default stream. */
int bdb_stored_matvec_noalloc(const float* M, int n3, int ld, const double* dD,
                              const double* F, const double* X, double pre,
                              double* Rf, double* Rs, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* BDB200_H */
