/* BD_BOX drop-in: the reference's diff_alg and potentials entry points on
 * the bdb200 engine.
 *
 * BD_BOX builds its CUDA variant by linking other translation units in
 * place of seven CPU ones (src/Makefile.am:44-78): potentials/calc_func.c,
 * diff_alg/diff_tensor.c, diff_rand.c, diff_comp.c, diff_decl.c,
 * diff_equation.c and newton.c. This file replaces the same seven. It
 * defines the globals and functions that the rest of BD_BOX (main.c,
 * main_loop.c, input.c, output.c, restart.c) binds, with the signatures of
 * diff_alg/diff_tensor.h:166-253 and potentials/calc_func.h:60-106, and runs
 * the work through the C ABI of include/bdb200.h on the current CUDA device.
 *
 * It is compiled against BD_BOX's own headers (data.h, input.h, ...) and the
 * host program's config.h; see bd_box_b200/dropin/Makefile.
 *
 * State. BD_BOX's host globals stay canonical (coord, F, E, Q, LJ, the bonded
 * arrays; data.h:315-361). The engine keeps a device copy. Host coordinates
 * are uploaded whenever they differ from the last copy exchanged with the
 * device, and they are read back after every step, because output.c reads
 * `coord` directly.
 *
 * Noise. By default each step draws its 3N Gaussians from the host's
 * gauss_rand (rand_move.h), once per attempt, exactly where diff_rand.c:52
 * draws them. So the drop-in follows the same random stream as the CPU build
 * for the same seed. With BDB_NOISE=philox in the environment, the engine
 * draws Philox Gaussians on the device instead (keyed by rand_seed), and no
 * host-to-device copy of noise happens.
 *
 * Engine choices come from the environment, since the .prm grammar has no
 * keys for them: BDB_PRECISION=fp64|mixed (default fp64) and
 * BDB_REFRESH=K (rebuild D and its Cholesky factor every K steps; default 1,
 * the reference schedule).
 *
 * Supported beyond the plain Ermak-McCammon step: ermak_var (dt halving on
 * overlaps), ermak_newton (elastic-collision overlap removal,
 * bdb_newton_resolve), igt_const / igt_var with hydro none or cholesky,
 * external electric fields (DC, AC, RF), the bounding sphere (bc sphere,
 * sboundary) and flowing solvent (vel_grad_tensor). Reported through the
 * host's unexpected_error (err.c:48-90) like any other fatal input error:
 * the IGT algorithms with hydro geyer, comp_step_rev_IGT (unimplemented in
 * BD_BOX itself), hydro methods other than none, cholesky and geyer (the
 * Chebyshev noise), a tensor that is not positive definite, an
 * over-stretched bond and CUDA errors.
 */
#if HAVE_CONFIG_H
#include <config.h>
#endif
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "data.h"
#include "err.h"
#include "input.h"
#include "rand_move.h"
#include "trans.h"
#include "diff_alg/diff_tensor.h"
#include "potentials/LJ.h"
#include "potentials/angle.h"
#include "potentials/angle_cos.h"
#include "potentials/bond.h"
#include "potentials/bucket.h"
#include "potentials/calc_func.h"
#include "potentials/dihe.h"
#include "potentials/dihe_angle.h"
#include "potentials/electro.h"
#include "potentials/electro_ext.h"
#include "potentials/sboundary.h"

#include "bdb200.h"

/* main_loop.c:47 */
extern DOUBLE curr_time;

/* ---- input variables of the replaced units (same names, types, defaults) */

/* diff_decl.c:66-81 */
MAKE_STR_IN(DOUBLE, visc, 0.01, "solvent viscosity [P]")
MAKE_STR_IN(DOUBLE, vfactor, 14.4, "viscosity unit conversion factor")
MAKE_STR_IN(DOUBLE, curr_dt, 0, "inner value: time step of the current move")
MAKE_STR_IN(NO_CHOLS_GEYER, hydro, 0, "hydrodynamic interactions: none, cholesky or geyer")
MAKE_STR_IN(ERMAK_IGTCONST_IGTVAR, algorithm, 2, "integration algorithm")
MAKE_STR_IN(INT, move_attempts, 10000, "attempts at a move before giving up after overlaps")
MAKE_STR_IN(PTR_DOUBLE9, vel_grad_tensor, NULL, "velocity gradient tensor (row, column)")
MAKE_STR_IN(DOUBLE, e_collision, 1, "restitution of the elastic-collision overlap removal")
MAKE_STR_IN(INT, ewald_real, 10, "real-space lattice radius of the Ewald sums")
MAKE_STR_IN(INT, ewald_recip, 10, "reciprocal-space lattice radius of the Ewald sums")
MAKE_STR_IN(DOUBLE, ewald_alpha, 1.77245385090551602729, "Ewald splitting parameter")
MAKE_STR_IN(EWALD_METHOD, ewald_method, 0, "Ewald tensor: smith or beenakker")
MAKE_STR_IN(YESNO, geyer_on_the_fly, 1, "TEA/D.F from 3x3 tiles (yes) or from the stored D (no)")

/* calc_func.c:62-64 */
MAKE_STR_IN(DOUBLE, bond_lj_scale, 1.0, "LJ scaling between bonded beads")
MAKE_STR_IN(DOUBLE, bond_c_scale, 1.0, "electrostatic scaling between bonded beads")
MAKE_STR_IN(YESNO, check_overlap, 1, "detect overlaps after each step")

/* ---- other globals of the replaced units (diff_tensor.h:166-253) */
INT ewald = 0;
DOUBLE preDii, preDij;
DOUBLE* D = NULL;
DOUBLE* Ds = NULL;
DOUBLE* diag_D = NULL;
DOUBLE* inv_diag_D = NULL;
DOUBLE* X = NULL;
DOUBLE** Rf = NULL;
DOUBLE** Rs = NULL;
DOUBLE* epsilon = NULL;
DOUBLE* FS = NULL;
DOUBLE* Rf0 = NULL;
DOUBLE* S[2] = {NULL, NULL};
INT save_iter = 0;
INT curr_iter = 0;
DOUBLE* E = NULL;   /* calc_func.c */

/* ---- engine state ------------------------------------------------------- */

static bdb_system* g_sys = NULL;
static DOUBLE* g_dev_coord = NULL;  /* coordinates last exchanged with the device */
static DOUBLE* g_zero_q = NULL;     /* charges when the deck has none */
static int g_noise_host = 1;

static void fatal(const char* what, int rc)
{
    static char msg[768];
    snprintf(msg, sizeof msg, "bdb200: %s failed (%d): %s", what, rc, bdb_last_error());
    UNERR(msg)
}

#define CHK(call)                         \
    do {                                  \
        int rc_ = (call);                 \
        if (rc_ < 0) fatal(#call, rc_);   \
    } while (0)

static int env_choice(const char* key, const char* a, const char* b, int def)
{
    const char* v = getenv(key);
    if (!v || !*v) return def;
    if (!strcmp(v, a)) return 0;
    if (!strcmp(v, b)) return 1;
    fprintf(stderr, "bdb200: %s=%s is neither %s nor %s\n", key, v, a, b);
    UNERR("bad engine choice in the environment")
    return def;
}

static size_t coord_bytes(void) { return sizeof(DOUBLE) * DIMS1 * (size_t)size; }

static void check_supported(void)
{
    if (algorithm == DIFF_ALG_IGT_VAR_REV) UNERR("Unimplemented method: comp_step_rev_IGT")
    if ((algorithm == DIFF_ALG_IGT_CONST || algorithm == DIFF_ALG_IGT_VAR) && hydro == DIFF_GEYER)
        UNERR("bdb200: the IGT algorithms need hydro none or cholesky")
    if (hydro != DIFF_NONE && hydro != DIFF_CHOLESKY && hydro != DIFF_GEYER)
        UNERR("bdb200: hydro must be none, cholesky or geyer")
}

static void make_params(bdb_params* p)
{
    const char* r = getenv("BDB_REFRESH");
    memset(p, 0, sizeof *p);
    p->n = size;
    p->bc = bc == BC_BOX ? 1 : (bc == BC_SPHERE ? 2 : 0);
    p->box[0] = box[0];
    p->box[1] = box[1];
    p->box[2] = box[2];
    p->hydro = hydro;
    p->ewald = ewald;
    p->ewald_real = ewald_real;
    p->ewald_method = ewald_method == EWALD_METHOD_SMITH ? BDB_EWALD_SMITH : BDB_EWALD_BEENAKKER;
    p->ewald_alpha = ewald_alpha;
    p->T = T;
    p->visc = visc;
    p->vfactor = vfactor;
    p->dt = dt;
    p->elec = elec;
    p->epsilon_c = epsilon_c;
    p->kappa_c = kappa_c;
    p->gamma_c = gamma_c;
    p->cutoff_c = cutoff_c;
    p->alpha_lj = alpha_lj;
    p->cutoff_lj = cutoff_lj;
    p->lj_6_term = lj_6_term;
    p->bond_lj_scale = bond_lj_scale;
    p->bond_c_scale = bond_c_scale;
    p->check_overlap = check_overlap;
    p->nb_list = nb_list;
    p->max_force_cutoff = max_force_cutoff;
    /* external forces (pre_func.c:135-158) */
    p->e_ext = E_ext;
    p->e_type = E_type;
    p->e_dir1 = E_dir1 - 'x';
    p->e_dir2 = E_dir2 - 'x';
    p->e_factor = E_factor;
    p->e_magn = E_magn;
    p->e_freq = E_freq;
    p->sboundary = sboundary;
    p->sboundary_n = sboundary_n;
    p->sboundary_A = sboundary_A;
    p->sboundary_cutoff = sboundary_cutoff;
    p->sphere_radius = sphere_radius;
    /* flowing solvent (diff_decl.c:72); input.c:462-468 already dropped it for bc sphere */
    p->flow = vel_grad_tensor != NULL;
    if (vel_grad_tensor)
        for (int k = 0; k < 9; ++k) p->vel_grad[k] = vel_grad_tensor[k];
    p->precision = env_choice("BDB_PRECISION", "fp64", "mixed", 0) ? BDB_PREC_MIXED : BDB_PREC_FP64;
    p->refresh = r && atoi(r) > 0 ? atoi(r) : 1;
    p->noise = g_noise_host ? BDB_NOISE_HOST : BDB_NOISE_PHILOX;
    p->seed = (uint64_t)(unsigned)rand_seed;
}

/* the engine for the deck in BD_BOX's globals; created once, after
 * init_cutoff has set max_force_cutoff */
static void engine(void)
{
    bdb_params p;
    const DOUBLE* q = Q;
    if (g_sys) return;
    check_supported();
    g_noise_host = !env_choice("BDB_NOISE", "host", "philox", 0);
    make_params(&p);
    if (!q) {
        g_zero_q = (DOUBLE*)calloc((size_t)size, sizeof(DOUBLE));
        CHMEM(g_zero_q);
        q = g_zero_q;
    }
    CHK(bdb_create(&g_sys, &p, coord, q, LJ));
    CHK(bdb_set_bonded(g_sys, bond_size, bond_pairs, bond_parms, angle_size, angle_pairs, angle_phis,
                       angle_cos_size, angle_cos_pairs, angle_cos_phis, dihe_size, dihe_pairs, dihe_parms,
                       dihe_angle_size, dihe_angle_pairs, dihe_angle_parms));
    g_dev_coord = (DOUBLE*)malloc(coord_bytes());
    CHMEM(g_dev_coord);
    memcpy(g_dev_coord, coord, coord_bytes());
}

/* host coordinates -> device, when the host changed them */
static void push_coord(void)
{
    engine();
    if (memcmp(g_dev_coord, coord, coord_bytes()) != 0) {
        CHK(bdb_set_coord(g_sys, coord));
        memcpy(g_dev_coord, coord, coord_bytes());
    }
}

/* device coordinates -> `out` */
static void pull_coord(DOUBLE* out)
{
    CHK(bdb_get_coord(g_sys, out));
    memcpy(g_dev_coord, out, coord_bytes());
}

/* ---- potentials (calc_func.h:60-106) ------------------------------------ */

void init_forces(void)
{
    init_cutoff();   /* max_force_cutoff (pre_func.c:197-232) */
    init_Fs();       /* host F, ES, E, repeat (pre_func.c:234-266) */
    engine();
}

void free_forces(void)
{
    if (g_sys) bdb_destroy(g_sys);
    g_sys = NULL;
    free(g_dev_coord);
    g_dev_coord = NULL;
    free(g_zero_q);
    g_zero_q = NULL;
    free_Fs();
    free(E);
    E = NULL;
}

/* Forces at the host coordinates into F[0] (and energies into _E when it is
 * not NULL). Returns the overlap flag like the CPU version: nonzero only if
 * check_overlap is on and an LJ pair overlaps or a term is not finite. */
INT compute_forces(DOUBLE* _E, DOUBLE t)
{
    int rc;
    push_coord();
    CHK(bdb_set_time(g_sys, t));   /* the time-dependent field acts at t */
    rc = bdb_compute_forces(g_sys, F[0], _E, NULL);
    if (rc < 0) fatal("bdb_compute_forces", rc);
    return rc;
}

/* ---- diffusion tensor (diff_tensor.h:166-253) --------------------------- */

void init_tensor(void)
{
    /* diff_tensor.c:546-559: Beenakker's splitting parameter is fixed by the box */
    if (ewald_method == EWALD_METHOD_BEENAKKER) ewald_alpha = SQRTPI * inv_L[0];
}

void init_diff_tensor(void)
{
    INT i;
    const INT n3 = DIMS0 * size;
    check_supported();
    preDii = kB_1_6PI * T / (visc * vfactor);
    preDij = kB_1_8PI * T / (visc * vfactor);
    diag_D = (DOUBLE*)malloc(sizeof(DOUBLE) * n3);
    CHMEM(diag_D);
    inv_diag_D = (DOUBLE*)malloc(sizeof(DOUBLE) * n3);
    CHMEM(inv_diag_D);
    for (i = 0; i < n3; ++i) {
        diag_D[i] = preDii / coord[DIMS1 * (i / DIMS0) + 3];
        inv_diag_D[i] = 1 / diag_D[i];
    }
    X = (DOUBLE*)malloc(sizeof(DOUBLE) * n3);
    CHMEM(X);
    Rf = (DOUBLE**)malloc(sizeof(DOUBLE*) * g_threads);
    CHMEM(Rf);
    Rs = (DOUBLE**)malloc(sizeof(DOUBLE*) * g_threads);
    CHMEM(Rs);
    for (i = 0; i < g_threads; ++i) {
        Rf[i] = (DOUBLE*)calloc((size_t)DIMS1 * size + 1, sizeof(DOUBLE));
        CHMEM(Rf[i]);
        Rs[i] = (DOUBLE*)calloc((size_t)DIMS1 * size + 1, sizeof(DOUBLE));
        CHMEM(Rs[i]);
    }
    Rf0 = (DOUBLE*)calloc((size_t)DIMS1 * size, sizeof(DOUBLE));
    CHMEM(Rf0);
    epsilon = (DOUBLE*)calloc((size_t)g_threads, sizeof(DOUBLE));
    CHMEM(epsilon);
    if (hydro && !geyer_on_the_fly) {
        Ds = (DOUBLE*)calloc((size_t)n3 * n3, sizeof(DOUBLE));
        CHMEM(Ds);
    }
    init_tensor();
}

void free_diff_tensor(void)
{
    INT i;
    for (i = 0; Rf && i < g_threads; ++i) free(Rf[i]);
    for (i = 0; Rs && i < g_threads; ++i) free(Rs[i]);
    free(Rf);
    free(Rs);
    Rf = Rs = NULL;
    free(Rf0);
    free(epsilon);
    free(Ds);
    free(D);
    free(X);
    free(diag_D);
    free(inv_diag_D);
    Rf0 = epsilon = Ds = D = X = diag_D = inv_diag_D = NULL;
}

/* Upper triangle of the 3N x 3N tensor, column-major with LD = 3N, as
 * compute_D fills it (diff_tensor.c:472-544); nothing without hydrodynamics. */
void compute_D(DOUBLE* _D)
{
    const size_t n3 = (size_t)DIMS0 * size;
    size_t r, c;
    DOUBLE* full;
    if (!hydro) return;
    push_coord();
    full = (DOUBLE*)malloc(sizeof(DOUBLE) * n3 * n3);
    CHMEM(full);
    CHK(bdb_compute_D(g_sys, full));
    for (c = 0; c < n3; ++c)
        for (r = 0; r <= c; ++r) _D[r + c * n3] = full[r * n3 + c];
    free(full);
}

void compute_single_D(DOUBLE* _D) { compute_D(_D); }

/* One 3x3 tile D_ij, row-major (diff_tensor.c:437-470). */
void compute_Dij(INT i, INT j, DOUBLE* tD)
{
    push_coord();
    CHK(bdb_compute_Dij(g_sys, i, j, tD));
}

void diff_tensor_calc_pos(INT i, INT j, DOUBLE* tD)
{
    if (ewald) UNERR("bdb200: the free-space tile of an Ewald-summed system is not exported")
    compute_Dij(i, j, tD);
}

void diff_tensor_calc_ewald_beenakker(INT i, INT j, DOUBLE* tD)
{
    if (!ewald || ewald_method != EWALD_METHOD_BEENAKKER) UNERR("bdb200: the system is not Beenakker-Ewald-summed")
    compute_Dij(i, j, tD);
}

void diff_tensor_calc_ewald_beenakker_diag(INT i, DOUBLE* tD)
{
    diff_tensor_calc_ewald_beenakker(i, i, tD);
}

void diff_tensor_calc_ewald_smith(INT i, INT j, DOUBLE* tD)
{
    if (!ewald || ewald_method != EWALD_METHOD_SMITH) UNERR("bdb200: the system is not Smith-Ewald-summed")
    compute_Dij(i, j, tD);
}

void diff_tensor_calc_ewald_smith_diag(INT i, DOUBLE* tD) { diff_tensor_calc_ewald_smith(i, i, tD); }

/* ---- Ermak-McCammon step (diff_equation.c, diff_rand.c, diff_comp.c) ---- */

static void set_dt(void) { CHK(bdb_set_dt(g_sys, curr_dt > 0 ? curr_dt : dt)); }

/* _Rf[0] = curr_dt/(kB T) D.F with the forces of the last compute_forces
 * (diff_equation.c:119-214); the engine uses its stored or on-the-fly D. */
void compute_Rf(DOUBLE** _Rf, DOUBLE* _D)
{
    (void)_D;
    push_coord();
    set_dt();
    CHK(bdb_compute_Rf(g_sys, _Rf[0]));
}

/* Rs[0] = the random displacement of diff_rand.c:47-236 at the current
 * coordinates. In host-noise mode X receives the 3N unit Gaussians drawn
 * here (the CPU version leaves them scaled). */
void compute_r(DOUBLE* _D)
{
    (void)_D;
    push_coord();
    set_dt();
    if (g_noise_host) {
        gauss_rand(X, DIMS0 * size);
        CHK(bdb_compute_r(g_sys, X, Rs[0]));
    } else {
        CHK(bdb_compute_r(g_sys, NULL, Rs[0]));
    }
}

/* one attempt: Rf, Rs, r += Rf + Rs, forces at the new positions;
 * returns the overlap flag */
static int attempt(void)
{
    int rc;
    set_dt();
    CHK(bdb_set_time(g_sys, curr_time));   /* BD_BOX's clock; a retried step starts from it again */
    if (g_noise_host) gauss_rand(X, DIMS0 * size);
    rc = bdb_step(g_sys, 1, g_noise_host ? X : NULL);
    if (rc < 0) fatal("bdb_step", rc);
    return rc;
}

/* comp_step_ermak (diff_comp.c:152-179) and comp_step_ermak_newton
 * (:181-210): an overlapping move is redone by elastic collisions
 * (bdb_newton_resolve) and reverted to try new Gaussians if that fails */
static DOUBLE ermak_step(DOUBLE* _E)
{
    INT count = 0;
    int rounds = 0;
    curr_dt = dt;
    curr_iter++;
    push_coord();
    CHK(bdb_save_state(g_sys));
    for (;;) {
        if (!attempt()) break;
        if (algorithm == DIFF_ALG_ERMAK_NEWTON) {
            int rc = bdb_newton_resolve(g_sys, e_collision, masses, move_attempts, &rounds);
            if (rc < 0) fatal("bdb_newton_resolve", rc);
            if (rc == 0) break;
            CHK(bdb_load_state(g_sys));
            if (bc != BC_SPHERE) warning("Revert move in none sphere case", __FILE__, __LINE__);
            continue;
        }
        if (algorithm == DIFF_ALG_ERMAK_VAR && count < 16) curr_dt /= 2;
        CHK(bdb_load_state(g_sys));
        ++count;
        if (count > move_attempts) UNERR("Wrong conformation, can't move")
    }
    pull_coord(coord);
    if (_E) CHK(bdb_compute_forces(g_sys, F[0], _E, NULL));
    return algorithm == DIFF_ALG_ERMAK_NEWTON ? dt : curr_dt;
}

static DOUBLE igt_step(DOUBLE* _E);

void compute_hydro(DOUBLE* _E)
{
    engine();
    if (algorithm == DIFF_ALG_IGT_CONST || algorithm == DIFF_ALG_IGT_VAR)
        curr_time += igt_step(_E);
    else
        curr_time += ermak_step(_E);
}

/* the move alone, into coord_out (diff_equation.c:216-286); the engine also
 * evaluates the forces at the new positions */
void compute_hydro_ermak(DOUBLE* coord_out)
{
    push_coord();
    attempt();
    pull_coord(coord_out);
}

/* ---- IGT predictor-corrector (diff_equation.c:288-374, diff_comp.c:76-144) */

/* the corrector from the step's start positions with fresh Gaussians (the
 * averaged factor of the predictor is kept); 2 on an overlap */
INT compute_hydro_IGT_second_phase(DOUBLE* _E)
{
    int rc;
    if (g_noise_host) gauss_rand(X, DIMS0 * size);
    rc = bdb_step_igt_corrector(g_sys, g_noise_host ? X : NULL);
    if (rc < 0) fatal("bdb_step_igt_corrector", rc);
    pull_coord(coord);
    if (_E && !rc) CHK(bdb_compute_forces(g_sys, F[0], _E, NULL));
    return rc ? 2 : 0;
}

/* predictor, forces at r' (1 on an overlap there), then the corrector */
INT compute_hydro_IGT(DOUBLE* _E)
{
    int rc;
    engine();
    push_coord();
    set_dt();
    CHK(bdb_set_time(g_sys, curr_time));
    if (g_noise_host) gauss_rand(X, DIMS0 * size);
    rc = bdb_step_igt_predictor(g_sys, g_noise_host ? X : NULL);
    if (rc < 0) fatal("bdb_step_igt_predictor", rc);
    if (rc) return 1;
    curr_iter++;
    return compute_hydro_IGT_second_phase(_E);
}

/* comp_step_IGT_const and comp_step_IGT_var (diff_comp.c:76-144): after an
 * overlap in the corrector the constant-step variant repeats only the
 * corrector; otherwise the step is revoked (the variable-step variant also
 * halves dt, at most 16 times) and taken again with new Gaussians */
static DOUBLE igt_step(DOUBLE* _E)
{
    INT count = 0;
    curr_dt = dt;
    curr_iter++;
    push_coord();
    CHK(bdb_save_state(g_sys));
    for (;;) {
        INT res = compute_hydro_IGT(_E);
        if (!res) break;
        if (algorithm == DIFF_ALG_IGT_CONST && res == 2) {
            while (compute_hydro_IGT_second_phase(_E)) {
                ++count;
                if (count > move_attempts) UNERR("Wrong conformation, can't move")
            }
            break;
        }
        if (algorithm == DIFF_ALG_IGT_VAR && count < 16) curr_dt /= 2;
        CHK(bdb_load_state(g_sys));
        ++count;
        if (count > move_attempts) UNERR("Wrong conformation, can't move")
    }
    pull_coord(coord);
    return curr_dt;
}

/* ---- state save/restore (diff_decl.c:219-237) ---------------------------- */

void save_curr_coord(void)
{
    memcpy(save_coord, coord, coord_bytes());
    push_coord();
    CHK(bdb_save_state(g_sys));
}

void save_curr_forces(void) { memcpy(save_forces, F[0], sizeof(DOUBLE) * DIMS0 * size); }

void load_coord(void)
{
    memcpy(coord, save_coord, coord_bytes());
    engine();
    CHK(bdb_load_state(g_sys));
    memcpy(g_dev_coord, coord, coord_bytes());
}

void load_forces(void) { memcpy(F[0], save_forces, sizeof(DOUBLE) * DIMS0 * size); }
