/* Test-oracle harness (test infrastructure only; never part of the product).
 *
 * Links the BD_BOX CPU objects compiled from the reference sources (every
 * file of src/ except main.c and rand_move.c, see oracle/Makefile) and drives
 * their own public functions on a .prm/.str deck, dumping float64 arrays:
 *
 *   ref_harness DECK.prm MODE OUT [args] [--key=value ...]
 *
 *   D       full symmetric 3N x 3N diffusion tensor, row-major, from
 *           compute_D (diff_alg/diff_tensor.c:472-544); the lower triangle is
 *           mirrored from the stored upper one, as single_point_print does
 *           (main_loop.c:129-160).
 *   forces  F[0] (3N), E[0..ENERGY_LAST] and the overlap flag returned by
 *           compute_forces (potentials/calc_func.c:106-186), then four pair
 *           counts: brute-force pairs with r <= cutoff_c and within the LJ
 *           range of force_single (calc_func.c:370-409), and the same two
 *           counts over the pairs that the bucket_space cell list
 *           (potentials/bucket.c:390-569) proposes.
 *   df      Rf[0] = dt/kT * D.F from compute_Rf (diff_alg/diff_equation.c:119-214)
 *           at the deck's start position, after compute_forces.
 *   tea     one compute_r (diff_alg/diff_rand.c:47-236) with the deck's hydro
 *           setting; dumps Rs[0] (3N), the scaled X (3N), Rf[0] (3N, the TEA
 *           normalisation factors) and epsilon[0].
 *   steps K [R]
 *           K Ermak-McCammon steps exactly as main_loop.c:80-115 runs them
 *           (compute_forces at t=0, then save_curr_* + compute_hydro per
 *           step), dumping the 4N coordinates after each step. With R > 1
 *           (hydro cholesky only) the diffusion tensor and its Cholesky factor
 *           are rebuilt only every R steps, by calling the reference's own
 *           compute_D, my_dpotrf, my_dtrmv, dsymv_ and compute_forces.
 *
 *   output K
 *           K steps as main_loop.c:89-116 runs them, with BD_BOX's own output
 *           code writing the files the deck names (init_save, save_output,
 *           free_save; output.c:250-311): xyz_filename / dcd_filename /
 *           enr_filename with their save_*_freq, the energies formed on the
 *           steps the energy file is written (main_loop.c:89, 102, 112). OUT
 *           gets, at the start and after each step, the 4N coordinates and
 *           E[0..ENERGY_LAST] (current on the written steps only).
 *
 * The Gaussian stream comes from BDB_GAUSS_FILE (oracle/ref_rand_file.c).
 *
 * BDB_EXTRA_DIHE, if set, names a text file of cosine dihedrals, one per
 * line: "i j k l k_theta m delta" with 0-based bead positions. They are added
 * through BD_BOX's own add_dihe (potentials/dihe.c:186-204) after the .str
 * file is read, because BD_BOX's .str parser rejects the cosine dihedral
 * line (input.c:621-628: parse_doubles(temp, 2) is followed by a check that
 * no third column exists). The deck must hold no other cosine dihedral, so
 * that add_dihe starts from an empty array.
 */
#if HAVE_CONFIG_H
#include <config.h>
#endif
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "data.h"
#include "input.h"
#include "main_loop.h"
#include "math_help.h"
#include "output.h"
#include "myblas.h"
#include "rand_move.h"
#include "trans.h"
#include "diff_alg/diff_tensor.h"
#include "potentials/bucket.h"
#include "potentials/bond.h"
#include "potentials/calc_func.h"
#include "potentials/dihe.h"
#include "potentials/electro.h"
#include "potentials/LJ.h"

/* defined in diff_alg/diff_equation.c:119 without a header declaration */
void compute_Rf(DOUBLE** _Rf, DOUBLE* _D);

static FILE* open_out(const char* path)
{
    FILE* f = fopen(path, "wb");
    if (!f) {
        fprintf(stderr, "harness: cannot open %s\n", path);
        exit(2);
    }
    return f;
}

static void put(FILE* f, const double* v, size_t n)
{
    if (fwrite(v, sizeof(double), n, f) != n) {
        fprintf(stderr, "harness: short write\n");
        exit(2);
    }
}

static double* full_D(void)
{
    int n = DIMS0 * size;
    double* buf = (double*)calloc((size_t)n * n, sizeof(double));
    double* out = (double*)calloc((size_t)n * n, sizeof(double));
    int r, c;
    if (!buf || !out) exit(5);
    if (hydro) {
        compute_D(buf);
        for (r = 0; r < n; ++r)
            for (c = 0; c < n; ++c)
                out[(size_t)r * n + c] = r <= c ? buf[r + (size_t)c * n] : buf[c + (size_t)r * n];
    } else {
        for (r = 0; r < n; ++r) out[(size_t)r * n + r] = diag_D[r];
    }
    free(buf);
    return out;
}

static int lj_in_range(int i, int j, double r_norm)
{
    double lim = cutoff_lj > 0.0 ? cutoff_lj
                                 : 1.122462f * (LJ[2 * i + LJ_SIGMA_OFF] + LJ[2 * j + LJ_SIGMA_OFF]);
    return alpha_lj != 0.0 && r_norm <= lim;
}

static void pair_counts(double out[4])
{
    int i, j;
    double e[3], r_norm, r_sq;
    long long c_b = 0, lj_b = 0, c_c = 0, lj_c = 0;
    for (i = 0; i < size; ++i)
        for (j = i + 1; j < size; ++j) {
            get_v2_norms(i, j, e, &r_norm, &r_sq);
            if (elec && r_norm <= cutoff_c) c_b++;
            if (lj_in_range(i, j, r_norm)) lj_b++;
        }
    {
        bucket_f* br = init_bucket_f(size, (DOUBLE4*)coord, NULL, max_force_cutoff);
        if (br) {
            for (i = 0; i < size; ++i) {
                int sizes[64];
                int* ids[64];
                int k, l;
                get_neighbours(br, (DOUBLE4*)coord + i, sizes, ids);
                for (k = 0; k < 64 && sizes[k]; ++k)
                    for (l = 0; l < sizes[k]; ++l) {
                        j = ids[k][l];
                        if (i < j) {
                            get_v2_norms(i, j, e, &r_norm, &r_sq);
                            if (elec && r_norm <= cutoff_c) c_c++;
                            if (lj_in_range(i, j, r_norm)) lj_c++;
                        }
                    }
            }
            free_bucket_f(br, size, (DOUBLE4*)coord);
        } else {
            c_c = c_b;
            lj_c = lj_b;
        }
    }
    out[0] = (double)c_b;
    out[1] = (double)lj_b;
    out[2] = (double)c_c;
    out[3] = (double)lj_c;
}

static void steps_refresh(int K, int R, FILE* f)
{
    int n = DIMS0 * size;
    int s, i;
    double* Dsave = (double*)malloc(sizeof(double) * (size_t)n * n);
    double* L = (double*)malloc(sizeof(double) * (size_t)n * n);
    double* rf = (double*)malloc(sizeof(double) * n);
    double* xs = (double*)malloc(sizeof(double) * n);
    double* rs = (double*)malloc(sizeof(double) * n);
    double pre, a, t = 0.0;
    if (!Dsave || !L || !rf || !xs || !rs) exit(5);
    curr_dt = dt;
    for (s = 0; s < K; ++s) {
        if (s % R == 0) {
            memset(L, 0, sizeof(double) * (size_t)n * n);
            compute_D(L);
            memcpy(Dsave, L, sizeof(double) * (size_t)n * n);
            if (my_dpotrf(L, n, n)) {
                fprintf(stderr, "harness: Cholesky failed\n");
                exit(6);
            }
        }
        pre = curr_dt / (kB * T);
        {
            double one = 1.0, zero = 0.0;
            int ione = 1;
            dsymv_("U", &n, &one, Dsave, &n, F[0], &ione, &zero, rf, &ione);
        }
        for (i = 0; i < n; ++i) rf[i] *= pre;
        gauss_rand(xs, n);
        a = sqrt(2 * curr_dt);
        for (i = 0; i < n; ++i) xs[i] *= a;
        my_dtrmv(L, xs, rs, n, n);
        for (i = 0; i < size; ++i) {
            coord[i * DIMS1] = rf[i * DIMS0] + rs[i * DIMS0] + coord[i * DIMS1];
            coord[i * DIMS1 + 1] = rf[i * DIMS0 + 1] + rs[i * DIMS0 + 1] + coord[i * DIMS1 + 1];
            coord[i * DIMS1 + 2] = rf[i * DIMS0 + 2] + rs[i * DIMS0 + 2] + coord[i * DIMS1 + 2];
            trans_to_box(coord + DIMS1 * i);
        }
        t += curr_dt;
        compute_forces(NULL, t);
        put(f, coord, (size_t)DIMS1 * size);
    }
    free(Dsave);
    free(L);
    free(rf);
    free(xs);
    free(rs);
}

int main(int argc, char** argv)
{
    const char* mode;
    const char* out;
    char* pargv[64];
    int pargc = 0, i, argi = 4;
    FILE* f;
    if (argc < 4) {
        fprintf(stderr, "usage: ref_harness DECK.prm MODE OUT [args] [--key=value ...]\n");
        return 1;
    }
    mode = argv[2];
    out = argv[3];
#ifdef _OPENMP
    g_threads = omp_get_max_threads();
#endif
    pargv[pargc++] = argv[0];
    pargv[pargc++] = argv[1];
    for (i = 4; i < argc && pargc < 63; ++i)
        if (strncmp(argv[i], "--", 2) == 0) pargv[pargc++] = argv[i];
    pargv[pargc] = NULL;
    if (!parse_args(pargc, pargv)) return 1;
    read_prm_file();
    apply_options(0);
    init_rand(rand_seed);
    read_str_file();
    if (getenv("BDB_EXTRA_DIHE")) {
        FILE* df = fopen(getenv("BDB_EXTRA_DIHE"), "r");
        int q[4];
        double kt, m, delta;
        if (!df || dihe_size) {
            fprintf(stderr, "harness: cannot add cosine dihedrals\n");
            return 2;
        }
        while (fscanf(df, "%d %d %d %d %lf %lf %lf", q, q + 1, q + 2, q + 3, &kt, &m, &delta) == 7) {
            if (q[0] < 0 || q[1] < 0 || q[2] < 0 || q[3] < 0 || q[0] >= size || q[1] >= size || q[2] >= size ||
                q[3] >= size) {
                fprintf(stderr, "harness: dihedral bead out of range\n");
                return 2;
            }
            add_dihe(q[0], q[1], q[2], q[3], kt, m, delta);
        }
        fclose(df);
        end_dihe();
    }
    init_diff_tensor();
    init_forces();
    for (i = 0; i < DIMS1 * size; i += DIMS1) trans_to_box(coord + i);

    f = open_out(out);
    if (strcmp(mode, "D") == 0) {
        double* d = full_D();
        put(f, d, (size_t)DIMS0 * size * DIMS0 * size);
        free(d);
    } else if (strcmp(mode, "forces") == 0) {
        double rep, counts[4];
        rep = (double)compute_forces(E, 0.0);
        put(f, F[0], (size_t)DIMS0 * size);
        put(f, E, ENERGY_LAST + 1);
        put(f, &rep, 1);
        pair_counts(counts);
        put(f, counts, 4);
    } else if (strcmp(mode, "df") == 0) {
        compute_forces(NULL, 0.0);
        curr_dt = dt;
        compute_Rf(Rf, Ds);
        put(f, Rf[0], (size_t)DIMS0 * size);
    } else if (strcmp(mode, "tea") == 0) {
        double eps;
        curr_dt = dt;
        if (Ds) compute_D(Ds);
        compute_r(Ds);
        eps = epsilon[0];
        put(f, Rs[0], (size_t)DIMS0 * size);
        put(f, X, (size_t)DIMS0 * size);
        put(f, Rf[0], (size_t)DIMS0 * size);
        put(f, &eps, 1);
    } else if (strcmp(mode, "steps") == 0) {
        int K = argc > argi && argv[argi][0] != '-' ? atoi(argv[argi++]) : 1;
        int R = argc > argi && argv[argi][0] != '-' ? atoi(argv[argi++]) : 1;
        if (compute_forces(NULL, 0.0)) fprintf(stderr, "harness: overlap at start (ignored)\n");
        if (R > 1) {
            if (hydro != 1) {
                fprintf(stderr, "harness: refresh schedule needs hydro cholesky\n");
                return 1;
            }
            steps_refresh(K, R, f);
        } else {
            int s;
            for (s = 0; s < K; ++s) {
                save_curr_coord();
                save_curr_forces();
                compute_hydro(NULL);
                put(f, coord, (size_t)DIMS1 * size);
            }
        }
    } else if (strcmp(mode, "output") == 0) {
        int K = argc > argi && argv[argi][0] != '-' ? atoi(argv[argi++]) : 1;
        init_save();
        step = 0;
        if (compute_forces(enr_file ? E : NULL, 0.0)) fprintf(stderr, "harness: overlap at start (ignored)\n");
        save_output();
        put(f, coord, (size_t)DIMS1 * size);
        put(f, E, ENERGY_LAST + 1);
        for (step = 1; step <= K; ++step) {
            const int comp_E = enr_file && (step % save_enr_freq) == 0;
            save_curr_coord();
            save_curr_forces();
            compute_hydro(comp_E ? E : NULL);
            save_output();
            put(f, coord, (size_t)DIMS1 * size);
            put(f, E, ENERGY_LAST + 1);
        }
        free_save();
    } else {
        fprintf(stderr, "harness: unknown mode %s\n", mode);
        return 1;
    }
    fclose(f);
    return 0;
}
