/* CPU restatement of BD_BOX's per-step hot path -- TEST ORACLE ONLY.
 *
 * This library is test infrastructure: only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg load it, and only as the checker or the
 * timed CPU baseline. The product (libbdb200.so) never calls it.
 *
 * Every function restates one reference function on explicit arguments
 * instead of BD_BOX's globals; the file:line of the restated code is given
 * beside each declaration. Arithmetic follows the reference's operation
 * order and constant types (float literals such as M_PIF included), so that,
 * compiled without FMA contraction, it reproduces the reference's double
 * results. Pinning: tests/test_oracle_pin.py compares it with the compiled
 * reference (oracle/_ref/ref_harness) and with committed golden fixtures.
 */
#ifndef BDB_ORACLE_H
#define BDB_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int n;                      /* beads */
    const double* coord;        /* 4n: x, y, z, hydrodynamic radius */
    const double* Q;            /* n charges */
    const double* LJ;           /* 2n: sigma_LJ/2, epsilon_LJ */
    int bc;                     /* 0 none, 1 periodic box */
    double box[3], inv_L[3];
    /* hydrodynamics */
    int hydro;                  /* 0 none, 1 cholesky, 2 geyer */
    double T, visc, vfactor;
    int ewald;                  /* Ewald-summed tensor (periodic + hydro) */
    int ewald_method;           /* 0 smith, 1 beenakker (the reference's EWALD_METHOD_*) */
    int ewald_real;
    double ewald_alpha;         /* Smith's splitting parameter, in units of 1/L */
    /* non-bonded */
    int elec;
    double epsilon_c, kappa_c, gamma_c, cutoff_c;
    double alpha_lj, cutoff_lj;
    int lj_6_term;
    double bond_lj_scale, bond_c_scale;
    int check_overlap;
    /* bonded */
    int n_bond;        const int* bond_pairs;       const double* bond_parms;       /* (r0, rmax, H) */
    int n_angle;       const int* angle_pairs;      const double* angle_parms;      /* (phi0, k) */
    int n_angle_cos;   const int* angle_cos_pairs;  const double* angle_cos_parms;  /* (cos phi0, k) */
    int n_dihe;        const int* dihe_pairs;       const double* dihe_parms;       /* (-k delta, m) */
    int n_dihe_angle;  const int* dihe_angle_pairs; const double* dihe_angle_parms; /* (k, theta0) */
    /* external forces (pre_func.c:135-158): electro_ext_force
     * (electro_ext.c:38-51) and sboundary_ext (sboundary.c:36-73, bc 2) */
    int e_ext, e_type, e_dir1, e_dir2;   /* E_type 0 DC, 1 AC, 2 RF; dirs 0..2 */
    double e_factor, e_magn, e_freq;
    int sboundary, sboundary_n;
    double sboundary_A, sboundary_cutoff, sphere_radius;
    double t;                   /* time of the state: forces act at t (curr_time + curr_dt after a step) */
    int flow;                   /* vel_grad_tensor set (diff_equation.c:265-283), Ermak steps */
    double vel_grad[9];         /* G, row-major */
} orc_system;

/* ENERGY_TYPE indices (data.h:278-289); energy arrays hold 9 doubles. */
enum { ORC_E_NONE, ORC_E_BOND, ORC_E_ANGLE, ORC_E_ANGLE_COS, ORC_E_DIHE,
       ORC_E_DIHE_ANGLE, ORC_E_LJ, ORC_E_COULOMB, ORC_E_LAST };

/* preDii, preDij and the per-bead diagonal (diff_decl.c:83-101). */
void orc_prefactors(const orc_system* s, double* preDii, double* preDij);

/* One 3x3 tile of D, compute_Dij (diff_alg/diff_tensor.c:437-470): free
 * space with overlap correction (:45-92) or Beenakker Ewald (:265-422). */
void orc_tile(const orc_system* s, int i, int j, double tD[9]);

/* Full symmetric 3N x 3N D, row-major (compute_D, diff_tensor.c:472-544). */
void orc_D(const orc_system* s, double* D);

/* Lower Cholesky factor in place of a row-major n x n SPD matrix (only the
 * lower triangle is read and written); the role of my_dpotrf (myblas.c:45-92).
 * Returns 0, or the 1-based index of the first non-positive pivot. */
int orc_cholesky(int n, double* A, int lda);

/* y = L x for the lower triangle of L (my_dtrmv, myblas.c:94-118). */
void orc_trmv_lower(int n, const double* L, int lda, const double* x, double* y);

/* y = A x for symmetric A read from its upper triangle (dsymv "U",
 * diff_alg/diff_equation.c:152-159). */
void orc_symv_upper(int n, const double* A, int lda, const double* x, double* y);

/* Rf = dt/(kB T) D.F (compute_Rf / compute_Rf_geyer_in_fly,
 * diff_alg/diff_equation.c:55-214). D == NULL recomputes tiles on the fly. */
void orc_df(const orc_system* s, const double* D, const double* F, double dt, double* Rf);

/* Geyer-Winter TEA noise (compute_r DIFF_GEYER branch, diff_rand.c:86-230).
 * gauss: 3N unit Gaussians; D == NULL recomputes tiles on the fly. Outputs
 * Rs (3N); optional eps/beta. */
void orc_tea(const orc_system* s, const double* D, const double* gauss, double dt,
             double* Rs, double* eps_out, double* beta_out);

/* Forces and energies (compute_forces, potentials/calc_func.c:106-186, with
 * force_single :370-409 and bonded_inter pre_func.c:97-159), all pairs in
 * brute-force order. F: 3N; E: 9 or NULL; counts (nullable): pairs with
 * r <= cutoff_c (elec on) and pairs inside the LJ range. Returns the overlap
 * flag (the forces are completed even when it is set). */
int orc_forces(const orc_system* s, double* F, double* E, long long counts[2]);

/* K Ermak-McCammon steps (compute_hydro_ermak, diff_equation.c:216-286, and
 * comp_step_ermak, diff_comp.c:152-179) from coord (updated in place); s->t
 * is the starting time and advances by dt per step (diff_comp.c:216).
 * gauss: K*3N Gaussians. refresh: rebuild D and its factor every `refresh`
 * steps (1 = every step, the reference schedule). F: 3N forces at the start
 * (updated). traj (nullable): 4N coords after each step. Returns the OR of
 * overlap flags, or -1 on a failed Cholesky. */
int orc_run_steps(orc_system* s, double* coord, double* F, double dt, int K,
                  const double* gauss, int refresh, double* traj);

/* K IGT predictor-corrector steps (comp_step_IGT_const without retries,
 * diff_comp.c:76-107; diff_equation.c:288-374). gauss: K*2*3N Gaussians
 * (predictor, then corrector, per step). Hydro none or cholesky. Returns the
 * OR of overlap flags (1: forces at the predicted positions, 2: forces
 * after the step), or -1 on a failed Cholesky. */
int orc_run_igt_steps(orc_system* s, double* coord, double* F, double dt, int K,
                      const double* gauss, double* traj);

/* K steps of comp_step_ermak_newton (diff_comp.c:181-210): a move that
 * overlaps is redone as ballistic moves with elastic collisions
 * (newton_init_vel, newton_moves, comp_time; newton.c), and reverted to try
 * new Gaussians if the result still overlaps. gauss: n_gauss blocks of 3N,
 * one per attempt; *used: blocks consumed; *rounds: collision rounds.
 * masses: N bead masses. Returns 0, -1 (failed Cholesky), -2 (more rounds
 * than move_attempts: "Ermak Newton error") or -3 (out of Gaussians). */
int orc_run_newton_steps(orc_system* s, double* coord, double* F, double dt, int K, const double* gauss,
                         int n_gauss, const double* masses, double e_collision, int move_attempts, double* traj,
                         int* used, int* rounds);

#ifdef __cplusplus
}
#endif
#endif
