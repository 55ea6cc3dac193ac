/* CPU restatement of BD_BOX's per-step hot path -- TEST ORACLE ONLY.
 * See bdb_oracle.h for the contract; every function cites the reference
 * code it restates. Compile without FMA contraction (plain x86-64 gcc -O2
 * has no FMA) so the operation order below gives the reference's doubles. */
#include "bdb_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* constants of data.h:207-211 (double build) and the float literal pi */
#define KB 0.001986248532617
#define KB_1_8PI 0.00007903031804378703
#define KB_1_6PI 0.00010537375739171604
#define SQRTPI 1.77245385090551602729
#define M1_SQRTPI 0.5641895835
#define M_PIF 3.14159265358979323846f

void orc_prefactors(const orc_system* s, double* preDii, double* preDij)
{
    *preDii = KB_1_6PI * s->T / (s->visc * s->vfactor);
    *preDij = KB_1_8PI * s->T / (s->visc * s->vfactor);
}

/* trans_dist_vec (trans.c:111-121): v = v2 - v1, minimum image when periodic */
static void dist_vec(const orc_system* s, const double* v1, const double* v2, double* v)
{
    int k;
    for (k = 0; k < 3; ++k) v[k] = v2[k] - v1[k];
    if (s->bc != 1) return;
    for (k = 0; k < 3; ++k) v[k] -= s->box[k] * floor(v[k] * s->inv_L[k] + 0.5f);
}

/* diff_tensor_calc_pos(a, b) (diff_tensor.c:45-92) */
static void tile_free(const orc_system* s, double preDii, double preDij, int a, int b, double* tD)
{
    const double* c = s->coord;
    double sigma_i = c[4 * b + 3], sigma_j = c[4 * a + 3];
    double e[3], r_sq, r_norm, inv;
    int i, j;
    e[0] = c[4 * a] - c[4 * b];
    e[1] = c[4 * a + 1] - c[4 * b + 1];
    e[2] = c[4 * a + 2] - c[4 * b + 2];
    r_sq = e[0] * e[0] + e[1] * e[1] + e[2] * e[2];
    r_norm = sqrt(r_sq);
    inv = 1 / r_norm;
    e[0] *= inv;
    e[1] *= inv;
    e[2] *= inv;
    if (r_norm < sigma_i + sigma_j) {
        double sigma = (sigma_i + sigma_j) / 2;
        double pre = preDii / sigma;
        double part1 = (1 - (9 * r_norm / (32 * sigma)));
        tD[0] = tD[4] = tD[8] = part1;
        for (i = 0; i < 3; ++i) {
            tD[i + 3 * i] += 3 * e[i] * e[i] * r_norm / (32 * sigma);
            tD[i + 3 * i] *= pre;
            for (j = 0; j < i; ++j) {
                tD[j + 3 * i] = pre * 3 * e[i] * e[j] * r_norm / (32 * sigma);
                tD[i + 3 * j] = tD[j + 3 * i];
            }
        }
    } else {
        double pre = preDij / r_norm;
        double sigm_r = (sigma_i * sigma_i + sigma_j * sigma_j) / r_sq;
        tD[0] = tD[4] = tD[8] = 1 + sigm_r / 3;
        for (i = 0; i < 3; ++i) {
            tD[i + 3 * i] += e[i] * e[i] * (1 - sigm_r);
            tD[i + 3 * i] *= pre;
            for (j = 0; j < i; ++j) {
                tD[j + 3 * i] = pre * e[i] * e[j] * (1 - sigm_r);
                tD[i + 3 * j] = tD[j + 3 * i];
            }
        }
    }
}

/* get_ev2_norms (math_help.c:85-101) */
static void ev2(double x, double y, double z, double* e, double* r_norm, double* r_sq)
{
    double inv;
    e[0] = x;
    e[1] = y;
    e[2] = z;
    *r_sq = x * x + y * y + z * z;
    *r_norm = sqrt(*r_sq);
    inv = 1 / *r_norm;
    e[0] *= inv;
    e[1] *= inv;
    e[2] *= inv;
}

/* diff_tensor_calc_ewald_beenakker(i, j) (diff_tensor.c:265-401) with the
 * constants of init_tensor (diff_tensor.c:546-559) */
static void tile_beenakker(const orc_system* s, double preDii, double preDij, int i, int j, double* _tD)
{
    const double* coord = s->coord;
    double sigma_i = coord[4 * j + 3], sigma_j = coord[4 * i + 3];
    double v[3], r[3];
    const double sigma_sq = 0.5 * (sigma_i * sigma_i + sigma_j * sigma_j);
    int k, l, f, g, h;
    double Op[9] = {0}, Qp[9] = {0};
    const double preQ = s->inv_L[0] * s->inv_L[0] * s->inv_L[0];
    const double ewald_alpha = SQRTPI * s->inv_L[0];
    const double alpha2 = ewald_alpha * ewald_alpha;
    const double alpha3 = ewald_alpha * alpha2;
    const double inv_alpha2 = 1.0f / alpha2;
    const int ewald_rr = s->ewald_real;
    const int rr_sq = s->ewald_real * s->ewald_real;
    const double L = s->box[0];
    r[0] = coord[4 * j] - coord[4 * i];
    r[1] = coord[4 * j + 1] - coord[4 * i + 1];
    r[2] = coord[4 * j + 2] - coord[4 * i + 2];

    if ((r[0] * r[0] + r[1] * r[1] + r[2] * r[2]) < (sigma_i + sigma_j) * (sigma_i + sigma_j) && i != j) {
        double r_norm, r_sq, e[3];
        int a, b;
        ev2(r[0], r[1], r[2], e, &r_norm, &r_sq);
        {
            double sigma = (sigma_i + sigma_j) / 2;
            double pre = preDii / sigma;
            double part1 = (1 - (9 * r_norm / (32 * sigma)));
            for (a = 0; a < 3; ++a) {
                _tD[a + 3 * a] += pre * (part1 + 3 * e[a] * e[a] * r_norm / (32 * sigma));
                for (b = 0; b < a; ++b) {
                    double vval = pre * 3 * e[a] * e[b] * r_norm / (32 * sigma);
                    _tD[b + 3 * a] += vval;
                    _tD[a + 3 * b] += vval;
                }
            }
        }
        {
            double pre = preDij / r_norm;
            double sigm_r = (sigma_i * sigma_i + sigma_j * sigma_j) / r_sq;
            double part1 = 1 + sigm_r / 3;
            for (a = 0; a < 3; ++a) {
                _tD[a + 3 * a] -= pre * (part1 + e[a] * e[a] * (1 - sigm_r));
                for (b = 0; b < a; ++b) {
                    double vval = pre * e[a] * e[b] * (1 - sigm_r);
                    _tD[b + 3 * a] -= vval;
                    _tD[a + 3 * b] -= vval;
                }
            }
        }
    }
    v[0] = r[0] * s->inv_L[0];
    v[1] = r[1] * s->inv_L[1];
    v[2] = r[2] * s->inv_L[2];
    for (h = -ewald_rr; h <= ewald_rr; ++h) {
        int next_f = (int)sqrt(rr_sq - h * h);
        for (f = -next_f; f <= next_f; ++f) {
            int next_g = (int)sqrt(rr_sq - h * h - f * f);
            for (g = -next_g; g <= next_g; ++g) {
                double r_norm, r_sq, e[3], inv_r, inv_r2, inv_r3, sc, sc2;
                ev2(r[0] + L * h, r[1] + L * f, r[2] + L * g, e, &r_norm, &r_sq);
                if (r_norm != 0.0f) {
                    inv_r = 1 / r_norm;
                    inv_r2 = 1 / r_sq;
                    inv_r3 = inv_r * inv_r2;
                    sc = ewald_alpha * sigma_sq * inv_r2;
                    sc += 14 * alpha3 * sigma_sq;
                    sc += -4.5f * ewald_alpha;
                    sc += -20 * alpha2 * alpha3 * sigma_sq * r_sq;
                    sc += 3 * alpha3 * r_sq;
                    sc += 4 * alpha3 * alpha2 * alpha2 * sigma_sq * r_sq * r_sq;
                    sc *= exp(-alpha2 * r_sq);
                    sc /= SQRTPI;
                    sc += erfc(r_norm * ewald_alpha) * (0.75f * inv_r + 0.5f * sigma_sq * inv_r3);

                    sc2 = -3 * ewald_alpha * sigma_sq * inv_r2;
                    sc2 += -2 * alpha3 * sigma_sq;
                    sc2 += 1.5f * ewald_alpha;
                    sc2 += 16 * alpha2 * alpha3 * sigma_sq * r_sq;
                    sc2 += -3 * alpha3 * r_sq;
                    sc2 += -4 * alpha3 * alpha2 * alpha2 * sigma_sq * r_sq * r_sq;
                    sc2 *= exp(-alpha2 * r_sq);
                    sc2 /= SQRTPI;
                    sc2 += erfc(r_norm * ewald_alpha) * (0.75f * inv_r - 1.5f * sigma_sq * inv_r3);
                    for (k = 0; k < 3; ++k) {
                        double sc_ek = e[k] * sc2;
                        Op[k * 4] += sc + sc_ek * e[k];
                        for (l = 0; l < k; ++l) Op[k + l * 3] += e[l] * sc_ek;
                    }
                }
                ev2(h, f, g, e, &r_norm, &r_sq);
                if (r_norm != 0.0f) {
                    r_norm *= 2 * M_PIF;
                    r_sq *= 4 * M_PIF * M_PIF;
                    sc = 1 - sigma_sq * r_sq / 3;
                    sc *= 1 + (inv_alpha2 * r_sq / 4) * (1 + inv_alpha2 * r_sq / 2);
                    sc *= 6 * M_PIF * exp(-inv_alpha2 * r_sq / 4) / r_sq;
                    sc *= cos(2 * M_PIF * (v[0] * h + v[1] * f + v[2] * g));
                    for (k = 0; k < 3; ++k) {
                        double sc_ek = sc * e[k];
                        Qp[k * 4] += sc - sc_ek * e[k];
                        for (l = 0; l < k; ++l) Qp[k + l * 3] -= e[l] * sc_ek;
                    }
                }
            }
        }
    }
    for (k = 0; k < 3; ++k) {
        _tD[k * 4] += preDii * (Op[k * 4] + preQ * Qp[k * 4]);
        for (l = 0; l < k; ++l) {
            _tD[k + l * 3] += preDii * (Op[k + l * 3] + preQ * Qp[k + l * 3]);
            _tD[l + k * 3] += preDii * (Op[k + l * 3] + preQ * Qp[k + l * 3]);
        }
    }
}

/* 1/sqrt(pi) as the reference's double build spells it (data.h:228) */
#define M1_SQRTPI_REF 0.5641895835

/* diff_tensor_calc_ewald_smith(i, j) (diff_tensor.c:102-243) with the
 * constants of init_tensor (diff_tensor.c:546-559): distances in units of
 * L, alpha = ewald_alpha, preO = 0.75/L, preQ = sigma^2/(2 L^3),
 * M_PI_ALPHA_SQ = -pi_f^2/alpha^2 (pi_f^2 formed in float) */
static void tile_smith(const orc_system* s, double preDii, double preDij, int i, int j, double* _tD)
{
    const double* coord = s->coord;
    double sigma_i = coord[4 * j + 3], sigma_j = coord[4 * i + 3];
    double v[3];
    const double sigma_sq = 0.5 * (sigma_i * sigma_i + sigma_j * sigma_j);
    int k, l, f, g, h;
    double Op[9] = {0}, Qp[9] = {0};
    const double ewald_alpha = s->ewald_alpha;
    const double alpha2 = ewald_alpha * ewald_alpha;
    const double alpha3 = ewald_alpha * alpha2;
    const float pif2 = -M_PIF * M_PIF;
    const double m_pi_alpha_sq = pif2 / alpha2;
    const double preO = 0.75 * s->inv_L[0];
    const double preQ = 0.5 * sigma_sq * s->inv_L[0] * s->inv_L[0] * s->inv_L[0];
    const int ewald_rr = s->ewald_real;
    const int rr_sq = s->ewald_real * s->ewald_real;
    /* dist_vec(coord_j, coord_i): v = r_i - r_j, no minimum image */
    v[0] = coord[4 * i] - coord[4 * j];
    v[1] = coord[4 * i + 1] - coord[4 * j + 1];
    v[2] = coord[4 * i + 2] - coord[4 * j + 2];
    if ((v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) < (sigma_i + sigma_j) * (sigma_i + sigma_j) && i != j) {
        double r_norm, r_sq, e[3];
        int a, b;
        ev2(v[0], v[1], v[2], e, &r_norm, &r_sq);
        {
            double sigma = (sigma_i + sigma_j) / 2;
            double pre = preDii / sigma;
            double part1 = (1 - (9 * r_norm / (32 * sigma)));
            for (a = 0; a < 3; ++a) {
                _tD[a + 3 * a] += pre * (part1 + 3 * e[a] * e[a] * r_norm / (32 * sigma));
                for (b = 0; b < a; ++b) {
                    double vval = pre * 3 * e[a] * e[b] * r_norm / (32 * sigma);
                    _tD[b + 3 * a] += vval;
                    _tD[a + 3 * b] += vval;
                }
            }
        }
        {
            double pre = preDij / r_norm;
            double sigm_r = (sigma_i * sigma_i + sigma_j * sigma_j) / r_sq;
            double part1 = 1 + sigm_r / 3;
            for (a = 0; a < 3; ++a) {
                _tD[a + 3 * a] -= pre * (part1 + e[a] * e[a] * (1 - sigm_r));
                for (b = 0; b < a; ++b) {
                    double vval = pre * e[a] * e[b] * (1 - sigm_r);
                    _tD[b + 3 * a] -= vval;
                    _tD[a + 3 * b] -= vval;
                }
            }
        }
    }
    v[0] *= s->inv_L[0];
    v[1] *= s->inv_L[1];
    v[2] *= s->inv_L[2];
    for (h = -ewald_rr; h <= ewald_rr; ++h) {
        int next_f = (int)sqrt(rr_sq - h * h);
        for (f = -next_f; f <= next_f; ++f) {
            int next_g = (int)sqrt(rr_sq - h * h - f * f);
            for (g = -next_g; g <= next_g; ++g) {
                double r_norm, r_sq, e[3], inv_r, inv_r3, sc, sc2;
                /* real space: O (Oseen) and Q (sigma^2) sums */
                ev2(v[0] + h, v[1] + f, v[2] + g, e, &r_norm, &r_sq);
                if (r_norm != 0.0f) {
                    inv_r = 1 / r_norm;
                    inv_r3 = 1 / (r_norm * r_sq);
                    sc = erfc(r_norm * ewald_alpha) * inv_r;
                    sc2 = 2 * ewald_alpha * M1_SQRTPI_REF * exp(-alpha2 * r_sq);
                    for (k = 0; k < 3; ++k) {
                        double sc_ek = e[k] * (sc + sc2);
                        Op[k * 4] += sc + sc_ek * e[k];
                        for (l = 0; l < k; ++l) Op[k + l * 3] += e[l] * sc_ek;
                    }
                    sc = inv_r3 * (erfc(r_norm * ewald_alpha) +
                                   2 * ewald_alpha * r_norm * M1_SQRTPI_REF * exp(-alpha2 * r_sq));
                    sc2 = -4 * alpha3 * M1_SQRTPI_REF * exp(-alpha2 * r_sq);
                    for (k = 0; k < 3; ++k) {
                        double sc_ek = (-3 * sc + sc2) * e[k];
                        Qp[k * 4] += sc + sc_ek * e[k];
                        for (l = 0; l < k; ++l) Qp[k + l * 3] += e[l] * sc_ek;
                    }
                }
                /* reciprocal space */
                ev2(h, f, g, e, &r_norm, &r_sq);
                if (r_norm != 0.0f) {
                    const double ph = cos(2 * M_PIF * (v[0] * h + v[1] * f + v[2] * g));
                    sc = 2 * exp(m_pi_alpha_sq * r_sq) / (M_PIF * r_sq);
                    sc2 = -1 + m_pi_alpha_sq * r_sq;
                    sc *= ph;
                    sc2 *= sc;
                    for (k = 0; k < 3; ++k) {
                        double sc_ek = sc2 * e[k];
                        Op[k * 4] += sc + sc_ek * e[k];
                        for (l = 0; l < k; ++l) Op[k + l * 3] += e[l] * sc_ek;
                    }
                    sc = 4 * M_PIF * exp(m_pi_alpha_sq * r_sq);
                    sc *= ph;
                    for (k = 0; k < 3; ++k) {
                        double sc_ek = sc * e[k];
                        Qp[k * 4] += sc_ek * e[k];
                        for (l = 0; l < k; ++l) Qp[k + l * 3] += e[l] * sc_ek;
                    }
                }
            }
        }
    }
    for (k = 0; k < 3; ++k) {
        _tD[k * 4] += preDii * (preO * Op[k * 4] + preQ * Qp[k * 4]);
        for (l = 0; l < k; ++l) {
            _tD[k + l * 3] += preDii * (preO * Op[k + l * 3] + preQ * Qp[k + l * 3]);
            _tD[l + k * 3] += preDii * (preO * Op[k + l * 3] + preQ * Qp[k + l * 3]);
        }
    }
}

void orc_tile(const orc_system* s, int i, int j, double tD[9])
{
    double preDii, preDij;
    int k;
    orc_prefactors(s, &preDii, &preDij);
    for (k = 0; k < 9; ++k) tD[k] = 0.0;
    if (i == j) {
        if (!s->ewald) {
            tD[0] = tD[4] = tD[8] = preDii / s->coord[4 * i + 3];
        } else if (s->ewald_method == 0) {
            /* diff_tensor_calc_ewald_smith_diag (diff_tensor.c:245-263) */
            double aw = s->coord[4 * i + 3];
            double il = s->inv_L[0];
            double sc3;
            int l;
            tile_smith(s, preDii, preDij, i, i, tD);
            sc3 = s->ewald_alpha * aw * il;
            sc3 = sc3 * sc3 * sc3 * M1_SQRTPI_REF / 3;
            sc3 = 0.75f * il * 1.5f * s->ewald_alpha * aw * M1_SQRTPI_REF * il + 0.5f * aw * aw * il * il * il * sc3;
            sc3 *= preDii;
            for (k = 0; k < 3; ++k) {
                tD[k * 4] = preDii / aw - sc3 + tD[k * 4];
                for (l = 0; l < k; ++l) tD[l + 3 * k] = tD[k + 3 * l] = 0;
            }
        } else {
            /* diff_tensor_calc_ewald_beenakker_diag (diff_tensor.c:404-422) */
            double aw = s->coord[4 * i + 3];
            double ewald_alpha = SQRTPI * s->inv_L[0];
            double alpha3 = ewald_alpha * ewald_alpha * ewald_alpha;
            double sc3;
            int l;
            tile_beenakker(s, preDii, preDij, i, i, tD);
            sc3 = -6 * ewald_alpha / SQRTPI + 40 * alpha3 * aw * aw / (3 * SQRTPI);
            sc3 *= preDii;
            for (k = 0; k < 3; ++k) {
                tD[k * 4] = preDii / aw + sc3 + tD[k * 4];
                for (l = 0; l < k; ++l) tD[l + 3 * k] = tD[k + 3 * l] = 0;
            }
        }
    } else if (!s->ewald) {
        tile_free(s, preDii, preDij, i, j, tD);
    } else if (s->ewald_method == 0) {
        tile_smith(s, preDii, preDij, i, j, tD);
    } else {
        tile_beenakker(s, preDii, preDij, i, j, tD);
    }
}

void orc_D(const orc_system* s, double* D)
{
    int n3 = 3 * s->n;
    int i;
    memset(D, 0, sizeof(double) * (size_t)n3 * n3);
    if (!s->hydro) {
        /* compute_D returns at once without hydrodynamics (diff_tensor.c:477);
         * the tensor is diag_D (single_point_print, main_loop.c:161-175) */
        double preDii, preDij;
        orc_prefactors(s, &preDii, &preDij);
        for (i = 0; i < n3; ++i) D[(size_t)i * n3 + i] = preDii / s->coord[4 * (i / 3) + 3];
        return;
    }
#pragma omp parallel for schedule(dynamic)
    for (i = 0; i < s->n; ++i) {
        int j, k, l;
        double tD[9];
        for (j = 0; j <= i; ++j) {
            orc_tile(s, i, j, tD);
            /* insert9 (diff_tensor.c:425-435): tile (i, j) goes to rows 3j+k,
             * columns 3i+l of the upper triangle; mirror it below */
            for (k = 0; k < 3; ++k)
                for (l = 0; l < 3; ++l) {
                    D[(size_t)(3 * j + k) * n3 + 3 * i + l] = tD[k + 3 * l];
                    D[(size_t)(3 * i + l) * n3 + 3 * j + k] = tD[k + 3 * l];
                }
        }
    }
}

int orc_cholesky(int n, double* A, int lda)
{
    /* right-looking unblocked Cholesky in the column order of the NR choldc
     * that myblas.c:63-89 restates (L stored below the diagonal) */
    int i, j, k;
    for (j = 0; j < n; ++j) {
        double d = A[(size_t)j * lda + j];
        for (k = 0; k < j; ++k) d -= A[(size_t)j * lda + k] * A[(size_t)j * lda + k];
        if (d <= 0.0) return j + 1;
        d = sqrt(d);
        A[(size_t)j * lda + j] = d;
#pragma omp parallel for if (n - j > 256)
        for (i = j + 1; i < n; ++i) {
            double sum = A[(size_t)i * lda + j];
            int kk;
            for (kk = 0; kk < j; ++kk) sum -= A[(size_t)i * lda + kk] * A[(size_t)j * lda + kk];
            A[(size_t)i * lda + j] = sum / d;
        }
    }
    return 0;
}

void orc_trmv_lower(int n, const double* L, int lda, const double* x, double* y)
{
    int i;
#pragma omp parallel for if (n > 512)
    for (i = 0; i < n; ++i) {
        double sum = 0.0;
        int j;
        for (j = 0; j <= i; ++j) sum += L[(size_t)i * lda + j] * x[j];
        y[i] = sum;
    }
}

void orc_symv_upper(int n, const double* A, int lda, const double* x, double* y)
{
    int i;
#pragma omp parallel for if (n > 512)
    for (i = 0; i < n; ++i) {
        double sum = 0.0;
        int j;
        for (j = 0; j < n; ++j)
            sum += (i <= j ? A[(size_t)i * lda + j] : A[(size_t)j * lda + i]) * x[j];
        y[i] = sum;
    }
}

void orc_df(const orc_system* s, const double* D, const double* F, double dt, double* Rf)
{
    int n3 = 3 * s->n, i;
    double pre = dt / (KB * s->T);
    double preDii, preDij;
    orc_prefactors(s, &preDii, &preDij);
    if (!s->hydro) {
        /* diff_equation.c:138-146 */
        for (i = 0; i < n3; ++i) Rf[i] = pre * (preDii / s->coord[4 * (i / 3) + 3]) * F[i];
        return;
    }
    if (D) {
        orc_symv_upper(n3, D, n3, F, Rf);
    } else {
        /* compute_Rf_geyer_in_fly (diff_equation.c:55-117) */
        memset(Rf, 0, sizeof(double) * n3);
        for (i = 0; i < s->n; ++i) {
            int k, j, l;
            double tD[9];
            for (k = 0; k < i; ++k) {
                orc_tile(s, i, k, tD);
                for (j = 0; j < 3; ++j)
                    for (l = 0; l < 3; ++l) {
                        Rf[i * 3 + j] += F[k * 3 + l] * tD[j * 3 + l];
                        Rf[k * 3 + l] += F[i * 3 + j] * tD[j * 3 + l];
                    }
            }
            orc_tile(s, i, i, tD);
            Rf[i * 3] += F[i * 3] * tD[0];
            Rf[i * 3 + 1] += F[i * 3 + 1] * tD[4];
            Rf[i * 3 + 2] += F[i * 3 + 2] * tD[8];
        }
    }
    for (i = 0; i < n3; ++i) Rf[i] *= pre;
}

void orc_tea(const orc_system* s, const double* D, const double* gauss, double dt,
             double* Rs, double* eps_out, double* beta_out)
{
    int n3 = 3 * s->n, i;
    double preDii, preDij, eps = 0.0, a, beta;
    double* X = (double*)malloc(sizeof(double) * n3);
    double* C = (double*)calloc(n3, sizeof(double));
    double* Feff = (double*)calloc(n3, sizeof(double));
    double* diag = (double*)malloc(sizeof(double) * n3);
    double* inv_diag = (double*)malloc(sizeof(double) * n3);
    orc_prefactors(s, &preDii, &preDij);
    /* diag_D / inv_diag_D (diff_decl.c:94-99): free-space self mobility */
    for (i = 0; i < n3; ++i) {
        diag[i] = preDii / s->coord[4 * (i / 3) + 3];
        inv_diag[i] = 1 / diag[i];
    }
    for (i = 0; i < n3; ++i) X[i] = gauss[i] * sqrt(2 * dt * inv_diag[i]);
    if (!D) {
        for (i = 0; i < s->n; ++i) {
            int k, j, l;
            double tD[9];
            for (k = 0; k < i; ++k) {
                orc_tile(s, i, k, tD);
                for (j = 0; j < 3; ++j)
                    for (l = 0; l < 3; ++l) {
                        C[i * 3 + j] += tD[j * 3 + l] * tD[j * 3 + l] * inv_diag[k * 3 + l];
                        C[k * 3 + l] += tD[j * 3 + l] * tD[j * 3 + l] * inv_diag[i * 3 + j];
                        Feff[i * 3 + j] += X[k * 3 + l] * tD[j * 3 + l];
                        Feff[k * 3 + l] += X[i * 3 + j] * tD[j * 3 + l];
                        eps += tD[j * 3 + l];
                    }
            }
        }
    } else {
        for (i = 0; i < n3; ++i) {
            int k;
            for (k = 0; k < i; ++k) {
                double d = D[(size_t)k * n3 + i];
                C[i] += d * d * inv_diag[k];
                C[k] += d * d * inv_diag[i];
                Feff[i] += X[k] * d;
                Feff[k] += X[i] * d;
                eps += d;
            }
        }
    }
    /* diff_rand.c:197-228 */
    eps /= n3;
    eps /= (n3 - 1);
    eps *= 2;
    if (eps > 1.0) eps = 1.0;
    a = (3 * s->n - 1) * eps * eps - (3 * s->n - 2) * eps;
    if ((a < 0.0 ? -a : a) < 0.0000001f)
        beta = 0.5;
    else
        beta = (1 - sqrt(1 - a)) / a;
    for (i = 0; i < n3; ++i) {
        double c = C[i] * (beta * beta * inv_diag[i]);
        c = 1 / (1 + c);
        c = sqrt(c);
        Rs[i] = c * (beta * Feff[i] + diag[i] * X[i]);
    }
    if (eps_out) *eps_out = eps;
    if (beta_out) *beta_out = beta;
    free(X);
    free(C);
    free(Feff);
    free(diag);
    free(inv_diag);
}

/* ------------------------------------------------------------------ forces */

static int bad(double v) { return isnan(v) || isinf(v); }

static void v2_norms(const orc_system* s, int p1, int p2, double* e, double* r_norm, double* r_sq)
{
    double inv;
    dist_vec(s, s->coord + 4 * p1, s->coord + 4 * p2, e);
    *r_sq = e[0] * e[0] + e[1] * e[1] + e[2] * e[2];
    *r_norm = sqrt(*r_sq);
    inv = 1 / *r_norm;
    e[0] *= inv;
    e[1] *= inv;
    e[2] *= inv;
}

static int bonded_pair(const orc_system* s, int i, int j)
{
    /* are_conn (bond.c:87-92) is live only when a 1-2 scale differs from 1
     * (alloc_connections, bond.c:113-130) */
    int k;
    if (!(s->n_bond && ((s->elec && s->bond_c_scale != 1) || (s->alpha_lj != 0.0 && s->bond_lj_scale != 1))))
        return 0;
    for (k = 0; k < s->n_bond; ++k) {
        int a = s->bond_pairs[2 * k], b = s->bond_pairs[2 * k + 1];
        if ((a == i && b == j) || (a == j && b == i)) return 1;
    }
    return 0;
}

static int lj_force(const orc_system* s, double r_norm, const double* e, double* F1, double* F2,
                    const double* lj1, const double* lj2, double scale, double* E)
{
    /* LJ_force / LJ_force_scale (LJ.c:37-93) */
    double sigma_ij = lj1[0] + lj2[0];
    double epsilon_ij = sqrt(lj1[1] * lj2[1]);
    double s6 = sigma_ij / r_norm;
    double Fm, en = 0;
    s6 *= s6;
    s6 *= s6 * s6;
    if (scale == 1.0) {
        en = s->alpha_lj * epsilon_ij * (s6 * (s6 - s->lj_6_term));
        Fm = s->alpha_lj * epsilon_ij * 6 * (s6 * (2 * s6 - s->lj_6_term)) / r_norm;
    } else {
        en = scale * s->alpha_lj * epsilon_ij * (s6 * (s6 - s->lj_6_term));
        Fm = scale;
        Fm *= s->alpha_lj * epsilon_ij * 6 * (s6 * (2 * s6 - s->lj_6_term)) / r_norm;
    }
    if (E) E[ORC_E_LJ] += en;
    F1[0] -= e[0] * Fm;
    F1[1] -= e[1] * Fm;
    F1[2] -= e[2] * Fm;
    F2[0] += e[0] * Fm;
    F2[1] += e[1] * Fm;
    F2[2] += e[2] * Fm;
    return (sigma_ij > r_norm) || bad(Fm) || bad(e[0]) || bad(e[1]) || bad(e[2]) || (E ? bad(E[ORC_E_LJ]) : 0);
}

static int electro_force(const orc_system* s, double r_norm, double r_sq, const double* e, double* F1,
                         double* F2, double Q1, double Q2, double scale, double* E)
{
    /* electro_force / electro_force_scale (electro.c:36-78) */
    double Fm = (s->gamma_c / s->epsilon_c) * Q1 * Q2 * (1 + s->kappa_c * r_norm);
    Fm *= exp(-s->kappa_c * r_norm) / r_sq;
    if (scale != 1.0) Fm *= scale;
    if (E) {
        if (scale != 1.0)
            E[ORC_E_COULOMB] += scale * (s->gamma_c / s->epsilon_c) * Q1 * Q2 * exp(-s->kappa_c * r_norm) / r_norm;
        else
            E[ORC_E_COULOMB] += (s->gamma_c / s->epsilon_c) * Q1 * Q2 * exp(-s->kappa_c * r_norm) / r_norm;
    }
    F1[0] -= e[0] * Fm;
    F1[1] -= e[1] * Fm;
    F1[2] -= e[2] * Fm;
    F2[0] += e[0] * Fm;
    F2[1] += e[1] * Fm;
    F2[2] += e[2] * Fm;
    return bad(Fm) || bad(e[0]) || bad(e[1]) || bad(e[2]) || (E ? bad(E[ORC_E_COULOMB]) : 0);
}

static double lj_range(const orc_system* s, int i, int j)
{
    return s->cutoff_lj > 0.0 ? s->cutoff_lj : 1.122462f * (s->LJ[2 * i] + s->LJ[2 * j]);
}

/* force_single (calc_func.c:370-409) */
static int force_single(const orc_system* s, int i, int j, double* F, double* E, long long* counts)
{
    double r_norm, r_sq, e[3];
    int rep = 0, conn = -1;
    const double* LJ = s->LJ;
    v2_norms(s, i, j, e, &r_norm, &r_sq);
    /* the 1-2 connection only matters inside a cut-off: looked up there (a
     * scan of the bond list, so not for every pair) */
    if ((s->elec && r_norm <= s->cutoff_c) || (s->alpha_lj != 0.0 && r_norm <= lj_range(s, i, j)))
        conn = bonded_pair(s, i, j);
    if (s->elec && r_norm <= s->cutoff_c) {
        if (counts) counts[0]++;
        if (!conn)
            electro_force(s, r_norm, r_sq, e, F + 3 * i, F + 3 * j, s->Q[i], s->Q[j], 1.0, E);
        else if (s->bond_c_scale != 0.0)
            electro_force(s, r_norm, r_sq, e, F + 3 * i, F + 3 * j, s->Q[i], s->Q[j], s->bond_c_scale, E);
    }
    if (s->alpha_lj != 0.0 && r_norm <= lj_range(s, i, j)) {
        if (counts) counts[1]++;
        if (!conn)
            rep = lj_force(s, r_norm, e, F + 3 * i, F + 3 * j, LJ + 2 * i, LJ + 2 * j, 1.0, E);
        else if (s->bond_lj_scale != 0.0)
            rep = lj_force(s, r_norm, e, F + 3 * i, F + 3 * j, LJ + 2 * i, LJ + 2 * j, s->bond_lj_scale, E);
        else
            rep = (LJ[2 * i] + LJ[2 * j]) * (LJ[2 * i] + LJ[2 * j]) > r_sq;
    } else {
        rep = (LJ[2 * i] + LJ[2 * j]) * (LJ[2 * i] + LJ[2 * j]) > r_sq;
    }
    return s->check_overlap && rep;
}

static void v3_norms(const orc_system* s, int p1, int p2, int p3, double* e1, double* e2)
{
    /* get_v3_norms (math_help.c:103-123) */
    double nrm1, nrm2;
    dist_vec(s, s->coord + 4 * p1, s->coord + 4 * p2, e1);
    dist_vec(s, s->coord + 4 * p3, s->coord + 4 * p2, e2);
    nrm1 = 1.0f / sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
    nrm2 = 1.0f / sqrt(e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2]);
    e1[0] *= nrm1;
    e1[1] *= nrm1;
    e1[2] *= nrm1;
    e2[0] *= nrm2;
    e2[1] *= nrm2;
    e2[2] *= nrm2;
}

static double cos_vs(const double* a, const double* b)
{
    double c = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
    if (c <= -1.0) c = -1.0;
    if (c >= 1.0) c = 1.0;
    return c;
}

static int bond_calc(const orc_system* s, int pos, double* F, double* E)
{
    /* bond.c:43-85 (an over-stretched bond is fatal there; here it is
     * reported through the return value 2) */
    double r_norm, r_sq, e[3];
    double r_0 = s->bond_parms[3 * pos], r_max = s->bond_parms[3 * pos + 1], H = s->bond_parms[3 * pos + 2];
    double Ff = 0, dist_rmax;
    int a = s->bond_pairs[2 * pos], b = s->bond_pairs[2 * pos + 1];
    double *F1 = F + 3 * a, *F2 = F + 3 * b;
    v2_norms(s, a, b, e, &r_norm, &r_sq);
    if (!(r_norm < r_max)) return 2;
    if (E)
        E[ORC_E_BOND] += -0.5 * H * (r_max * r_max * log((r_max * r_max - r_sq) / (r_max * r_max - r_0 * r_0)) +
                                      r_0 * r_max * log((r_max + r_norm) * (r_max - r_0) / ((r_max - r_norm) * (r_max + r_0))));
    dist_rmax = 1 - r_sq / (r_max * r_max);
    Ff = H * (r_0 - r_norm) / dist_rmax;
    F1[0] -= Ff * e[0];
    F1[1] -= Ff * e[1];
    F1[2] -= Ff * e[2];
    F2[0] += Ff * e[0];
    F2[1] += Ff * e[1];
    F2[2] += Ff * e[2];
    return bad(Ff) || bad(e[0]) || bad(e[1]) || bad(e[2]) || (E ? bad(E[ORC_E_BOND]) : 0);
}

static int angle_calc(const orc_system* s, int pos, double* F, double* E)
{
    /* angle.c:38-86 */
    double phi_0 = s->angle_parms[2 * pos], k_phi = s->angle_parms[2 * pos + 1];
    int p1 = s->angle_pairs[3 * pos], p2 = s->angle_pairs[3 * pos + 1], p3 = s->angle_pairs[3 * pos + 2];
    double Fi[3], Fk[3], e1[3], e2[3], cos_phi, phi;
    int k;
    v3_norms(s, p1, p2, p3, e1, e2);
    cos_phi = cos_vs(e1, e2);
    if (cos_phi >= 1 - 0.000001 || cos_phi <= -1 + 0.000001) return 0;
    phi = acos(cos_phi);
    k_phi *= (phi - phi_0);
    if (E) E[ORC_E_ANGLE] += 0.5f * k_phi * (phi - phi_0);
    k_phi /= sqrt(1 - cos_phi * cos_phi);
    for (k = 0; k < 3; ++k) {
        Fi[k] = -k_phi * (e2[k] - e1[k] * cos_phi);
        Fk[k] = -k_phi * (e1[k] - e2[k] * cos_phi);
    }
    for (k = 0; k < 3; ++k) {
        F[3 * p1 + k] += Fi[k];
        F[3 * p2 + k] += -Fi[k] - Fk[k];
        F[3 * p3 + k] += Fk[k];
    }
    return bad(Fk[0]) || bad(Fk[1]) || bad(Fk[2]) || bad(Fi[0]) || bad(Fi[1]) || bad(Fi[2]) ||
           (E ? bad(E[ORC_E_ANGLE]) : 0);
}

static int angle_cos_calc(const orc_system* s, int pos, double* F, double* E)
{
    /* angle_cos.c:36-81 */
    double phi_0 = s->angle_cos_parms[2 * pos], k_phi = s->angle_cos_parms[2 * pos + 1];
    int p1 = s->angle_cos_pairs[3 * pos], p2 = s->angle_cos_pairs[3 * pos + 1], p3 = s->angle_cos_pairs[3 * pos + 2];
    double Fi[3], Fk[3], e1[3], e2[3], cos_phi;
    int k;
    v3_norms(s, p1, p2, p3, e1, e2);
    cos_phi = cos_vs(e1, e2);
    k_phi *= (cos_phi - phi_0);
    if (E) E[ORC_E_ANGLE_COS] += 0.5f * k_phi * (cos_phi - phi_0);
    for (k = 0; k < 3; ++k) {
        Fi[k] = k_phi * (e2[k] - e1[k] * cos_phi);
        Fk[k] = k_phi * (e1[k] - e2[k] * cos_phi);
    }
    for (k = 0; k < 3; ++k) {
        F[3 * p1 + k] += Fi[k];
        F[3 * p2 + k] += -Fi[k] - Fk[k];
        F[3 * p3 + k] += Fk[k];
    }
    return bad(Fk[0]) || bad(Fk[1]) || bad(Fk[2]) || bad(Fi[0]) || bad(Fi[1]) || bad(Fi[2]) ||
           (E ? bad(E[ORC_E_ANGLE_COS]) : 0);
}

static double delta_cos(int m, double c)
{
    /* get_delta_cos (dihe.c:146-159) */
    switch (m) {
    case 1: return 1;
    case 2: return 4 * c;
    case 3: return 12 * c * c - 3;
    case 4: return c * (32 * c * c - 16);
    case 5: return c * c * (80 * c * c - 60) + 5;
    case 6: return c * (192 * c * c * (c * c - 1) + 36);
    default: return 0;
    }
}

static double m_cos(int m, double c)
{
    /* get_m_cos (dihe.c:161-174) */
    switch (m) {
    case 1: return c;
    case 2: return 2 * c * c - 1;
    case 3: return 4 * c * c * c - 3 * c;
    case 4: return 8 * c * c * (c * c - 1) + 1;
    case 5: return c * (c * c * (16 * c * c - 20) + 5);
    case 6: return c * c * (c * c * (32 * c * c - 48) + 18) - 1;
    default: return 1;
    }
}

static int dihe_calc(const orc_system* s, int pos, double* F, double* E)
{
    /* dihe.c:42-144 */
    const int* q = s->dihe_pairs + 4 * pos;
    const double *ri = s->coord + 4 * q[0], *rj = s->coord + 4 * q[1], *rk = s->coord + 4 * q[2], *rl = s->coord + 4 * q[3];
    double rim[3], rln[3], rkj[3], rij[3], rkl[3], Fi[3], Fj[3], Fk[3], Fl[3];
    double inv_nrim, inv_nrln, sijkj, sklkj, nkjsq, cos_theta, dc, tmp;
    double mkcd = s->dihe_parms[2 * pos];
    int m = (int)s->dihe_parms[2 * pos + 1], k;
    dist_vec(s, rk, rj, rkj);
    nkjsq = rkj[0] * rkj[0] + rkj[1] * rkj[1] + rkj[2] * rkj[2];
    dist_vec(s, ri, rj, rij);
    dist_vec(s, rk, rl, rkl);
    sijkj = (rij[0] * rkj[0] + rij[1] * rkj[1] + rij[2] * rkj[2]) / nkjsq;
    sklkj = (rkl[0] * rkj[0] + rkl[1] * rkj[1] + rkl[2] * rkj[2]) / nkjsq;
    for (k = 0; k < 3; ++k) rim[k] = -rij[k] + sijkj * rkj[k];
    tmp = sqrt(rim[0] * rim[0] + rim[1] * rim[1] + rim[2] * rim[2]);
    if ((tmp < 0 ? -tmp : tmp) < 0.000001) return 0;
    inv_nrim = 1.0f / tmp;
    for (k = 0; k < 3; ++k) rln[k] = rkl[k] - sklkj * rkj[k];
    tmp = sqrt(rln[0] * rln[0] + rln[1] * rln[1] + rln[2] * rln[2]);
    if ((tmp < 0 ? -tmp : tmp) < 0.000001) return 0;
    inv_nrln = 1.0f / tmp;
    cos_theta = (rim[0] * rln[0] + rim[1] * rln[1] + rim[2] * rln[2]) * inv_nrln * inv_nrim;
    if (cos_theta < -1) cos_theta = -1;
    if (cos_theta > 1) cos_theta = 1;
    if (E) {
        double am = mkcd < 0 ? -mkcd : mkcd;
        E[ORC_E_DIHE] += am * (1 + am * m_cos(m, cos_theta));
    }
    dc = delta_cos(m, cos_theta);
    tmp = mkcd * dc * inv_nrim;
    for (k = 0; k < 3; ++k) Fi[k] = tmp * (rln[k] * inv_nrln - rim[k] * inv_nrim * cos_theta);
    tmp = mkcd * dc * inv_nrln;
    for (k = 0; k < 3; ++k) Fl[k] = tmp * (rim[k] * inv_nrim - rln[k] * inv_nrln * cos_theta);
    for (k = 0; k < 3; ++k) Fj[k] = (sijkj - 1) * Fi[k] - sklkj * Fl[k];
    for (k = 0; k < 3; ++k) Fk[k] = -Fi[k] - Fj[k] - Fl[k];
    for (k = 0; k < 3; ++k) {
        F[3 * q[0] + k] += Fi[k];
        F[3 * q[1] + k] += Fj[k];
        F[3 * q[2] + k] += Fk[k];
        F[3 * q[3] + k] += Fl[k];
    }
    for (k = 0; k < 3; ++k)
        if (bad(Fi[k]) || bad(Fj[k]) || bad(Fk[k]) || bad(Fl[k])) return 1;
    return E ? bad(E[ORC_E_DIHE]) : 0;
}

static void cross(const double* a, const double* b, double* o)
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

static void grad_dihedral(const double* p1, const double* p2, const double* p3, const double* p4,
                          double* out_phi, double* g)
{
    /* measureAndCalcGradDihedral (dihe_angle.c:95-255) */
    double K1 = 1, r12[3], r23[3], r34[3], A[3], B[3], C[3], rAinv, rBinv, rCinv;
    double cos_phi, sin_phi, f1[3], f2[3], f3[3];
    int k;
    for (k = 0; k < 3; ++k) {
        r12[k] = p2[k] - p1[k];
        r23[k] = p3[k] - p2[k];
        r34[k] = p4[k] - p3[k];
    }
    cross(r12, r23, A);
    cross(r23, r34, B);
    cross(r23, A, C);
    rAinv = 1.0f / sqrt(A[0] * A[0] + A[1] * A[1] + A[2] * A[2]);
    rBinv = 1.0f / sqrt(B[0] * B[0] + B[1] * B[1] + B[2] * B[2]);
    rCinv = 1.0f / sqrt(C[0] * C[0] + C[1] * C[1] + C[2] * C[2]);
    cos_phi = (A[0] * B[0] + A[1] * B[1] + A[2] * B[2]) * (rAinv * rBinv);
    sin_phi = (C[0] * B[0] + C[1] * B[1] + C[2] * B[2]) * (rCinv * rBinv);
    if (cos_phi < -1) cos_phi = -1;
    if (cos_phi > 1) cos_phi = 1;
    if (sin_phi < -1) sin_phi = -1;
    if (sin_phi > 1) sin_phi = 1;
    *out_phi = -atan2(sin_phi, cos_phi);
    for (k = 0; k < 3; ++k) B[k] *= rBinv;
    if ((sin_phi < 0 ? -sin_phi : sin_phi) > 0.1f) {
        double dcosdA[3], dcosdB[3];
        for (k = 0; k < 3; ++k) A[k] *= rAinv;
        for (k = 0; k < 3; ++k) {
            dcosdA[k] = rAinv * (cos_phi * A[k] - B[k]);
            dcosdB[k] = rBinv * (cos_phi * B[k] - A[k]);
        }
        K1 = K1 / sin_phi;
        f1[0] = K1 * (r23[1] * dcosdA[2] - r23[2] * dcosdA[1]);
        f1[1] = K1 * (r23[2] * dcosdA[0] - r23[0] * dcosdA[2]);
        f1[2] = K1 * (r23[0] * dcosdA[1] - r23[1] * dcosdA[0]);
        f3[0] = K1 * (r23[2] * dcosdB[1] - r23[1] * dcosdB[2]);
        f3[1] = K1 * (r23[0] * dcosdB[2] - r23[2] * dcosdB[0]);
        f3[2] = K1 * (r23[1] * dcosdB[0] - r23[0] * dcosdB[1]);
        f2[0] = K1 * (r12[2] * dcosdA[1] - r12[1] * dcosdA[2] + r34[1] * dcosdB[2] - r34[2] * dcosdB[1]);
        f2[1] = K1 * (r12[0] * dcosdA[2] - r12[2] * dcosdA[0] + r34[2] * dcosdB[0] - r34[0] * dcosdB[2]);
        f2[2] = K1 * (r12[1] * dcosdA[0] - r12[0] * dcosdA[1] + r34[0] * dcosdB[1] - r34[1] * dcosdB[0]);
    } else {
        double dsindC[3], dsindB[3];
        for (k = 0; k < 3; ++k) C[k] *= rCinv;
        for (k = 0; k < 3; ++k) {
            dsindC[k] = rCinv * (sin_phi * C[k] - B[k]);
            dsindB[k] = rBinv * (sin_phi * B[k] - C[k]);
        }
        K1 = -K1 / cos_phi;
        f1[0] = K1 * ((r23[1] * r23[1] + r23[2] * r23[2]) * dsindC[0] - r23[0] * r23[1] * dsindC[1] - r23[0] * r23[2] * dsindC[2]);
        f1[1] = K1 * ((r23[2] * r23[2] + r23[0] * r23[0]) * dsindC[1] - r23[1] * r23[2] * dsindC[2] - r23[1] * r23[0] * dsindC[0]);
        f1[2] = K1 * ((r23[0] * r23[0] + r23[1] * r23[1]) * dsindC[2] - r23[2] * r23[0] * dsindC[0] - r23[2] * r23[1] * dsindC[1]);
        cross(dsindB, r23, f3);
        for (k = 0; k < 3; ++k) f3[k] *= K1;
        f2[0] = K1 * (-(r23[1] * r12[1] + r23[2] * r12[2]) * dsindC[0] + (2.0f * r23[0] * r12[1] - r12[0] * r23[1]) * dsindC[1] +
                      (2.0f * r23[0] * r12[2] - r12[0] * r23[2]) * dsindC[2] + dsindB[2] * r34[1] - dsindB[1] * r34[2]);
        f2[1] = K1 * (-(r23[2] * r12[2] + r23[0] * r12[0]) * dsindC[1] + (2.0f * r23[1] * r12[2] - r12[1] * r23[2]) * dsindC[2] +
                      (2.0f * r23[1] * r12[0] - r12[1] * r23[0]) * dsindC[0] + dsindB[0] * r34[2] - dsindB[2] * r34[0]);
        f2[2] = K1 * (-(r23[0] * r12[0] + r23[1] * r12[1]) * dsindC[2] + (2.0f * r23[2] * r12[0] - r12[2] * r23[0]) * dsindC[0] +
                      (2.0f * r23[2] * r12[1] - r12[2] * r23[1]) * dsindC[1] + dsindB[1] * r34[0] - dsindB[0] * r34[1]);
    }
    for (k = 0; k < 3; ++k) {
        g[k] = f1[k];
        g[3 + k] = f2[k] - f1[k];
        g[6 + k] = f3[k] - f2[k];
        g[9 + k] = -f3[k];
    }
}

static int dihe_angle_calc(const orc_system* s, int pos, double* F, double* E)
{
    /* dihe_angle.c:43-93 */
    const int* q = s->dihe_angle_pairs + 4 * pos;
    double oD[12], theta = 0, tmp;
    double k_theta = s->dihe_angle_parms[2 * pos], theta_0 = s->dihe_angle_parms[2 * pos + 1];
    int k, r = 0;
    grad_dihedral(s->coord + 4 * q[0], s->coord + 4 * q[1], s->coord + 4 * q[2], s->coord + 4 * q[3], &theta, oD);
    tmp = theta - theta_0;
    if (tmp < -M_PIF) tmp += 2 * M_PIF;
    if (tmp > M_PIF) tmp -= 2 * M_PIF;
    k_theta *= -tmp;
    if (E) E[ORC_E_DIHE_ANGLE] -= 0.5f * k_theta * tmp;
    for (k = 0; k < 4; ++k) {
        F[3 * q[k]] += k_theta * oD[3 * k];
        F[3 * q[k] + 1] += k_theta * oD[3 * k + 1];
        F[3 * q[k] + 2] += k_theta * oD[3 * k + 2];
    }
    for (k = 0; k < 12; ++k) r |= bad(oD[k]);
    return r || bad(k_theta) || (E ? bad(E[ORC_E_DIHE_ANGLE]) : 0);
}

/* electro_ext_force (electro_ext.c:38-51): Q * E_factor * E_magn on E_dir1,
 * times cos(E_freq t) for AC and RF, plus the sin part on E_dir2 for RF */
static int electro_ext_force(const orc_system* s, double Q, double* F)
{
    int pos = s->e_dir1, pos2 = 0;
    switch (s->e_type) {
        case 0: F[pos] += Q * s->e_factor * s->e_magn; break;
        case 1: F[pos] += Q * s->e_factor * s->e_magn * cos(s->e_freq * s->t); break;
        case 2:
            pos2 = s->e_dir2;
            F[pos] += Q * s->e_factor * s->e_magn * cos(s->e_freq * s->t);
            F[pos2] += Q * s->e_factor * s->e_magn * sin(s->e_freq * s->t);
            break;
    }
    return isnan(F[pos]) || isinf(F[pos]) || (s->e_type == 2 && (isnan(F[pos2]) || isinf(F[pos2])));
}

/* sboundary_ext (sboundary.c:36-73): -A x / (r R^n), R = sphere_radius - r,
 * beyond the cutoff radius; 1 (retry) within 1e-6 of the wall */
static int sboundary_ext(const orc_system* s, const double* c, double* F)
{
    double r = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    if (r >= s->sboundary_cutoff) {
        double R = s->sphere_radius - r;
        if (R >= 0.000001) {
            double inr = 1.0f / r, inR = 1.0f / R;
            int i;
            for (i = 1; i <= s->sboundary_n; i *= 2) {
                if (s->sboundary_n & i) inr *= inR;
                inR *= inR;
            }
            F[0] -= s->sboundary_A * c[0] * inr;
            F[1] -= s->sboundary_A * c[1] * inr;
            F[2] -= s->sboundary_A * c[2] * inr;
            return 0;
        }
        return 1;
    }
    return 0;
}

int orc_forces(const orc_system* s, double* F, double* E, long long counts[2])
{
    int i, j, rep = 0, r;
    memset(F, 0, sizeof(double) * 3 * s->n);
    if (E) memset(E, 0, sizeof(double) * ORC_E_LAST + sizeof(double));
    if (counts) counts[0] = counts[1] = 0;
    /* bonded_inter order (pre_func.c:97-159) */
    for (i = 0; i < s->n_angle_cos; ++i) rep |= angle_cos_calc(s, i, F, E);
    for (i = 0; i < s->n_angle; ++i) rep |= angle_calc(s, i, F, E);
    for (i = 0; i < s->n_bond; ++i) {
        r = bond_calc(s, i, F, E);
        if (r == 2) return 2;
        rep |= r;
    }
    for (i = 0; i < s->n_dihe; ++i) rep |= dihe_calc(s, i, F, E);
    for (i = 0; i < s->n_dihe_angle; ++i) rep |= dihe_angle_calc(s, i, F, E);
    if (s->e_ext)
        for (i = 0; i < s->n; ++i)
            if (s->Q[i] != 0.0) rep |= electro_ext_force(s, s->Q[i], F + 3 * i);
    if (s->sboundary && s->bc == 2)
        for (i = 0; i < s->n; ++i) rep |= sboundary_ext(s, s->coord + 4 * i, F + 3 * i);
    /* brute_force_val (calc_func.c:188-228) */
    if (s->elec || s->alpha_lj != 0.0) {
        for (i = 0; i < s->n; ++i)
            for (j = i + 1; j < s->n; ++j) rep |= force_single(s, i, j, F, E, counts);
    } else if (s->check_overlap) {
        for (i = 0; i < s->n; ++i)
            for (j = i + 1; j < s->n; ++j) {
                double e[3], rr, r_sq;
                v2_norms(s, i, j, e, &rr, &r_sq);
                rep |= (s->LJ[2 * i] + s->LJ[2 * j]) * (s->LJ[2 * i] + s->LJ[2 * j]) > r_sq;
            }
    }
    return rep ? 1 : 0;
}

int orc_run_steps(orc_system* s, double* coord, double* F, double dt, int K, const double* gauss,
                  int refresh, double* traj)
{
    int n3 = 3 * s->n, step, i, rep = 0;
    double* D = NULL;
    double* L = NULL;
    double* Rf = (double*)malloc(sizeof(double) * n3);
    double* Rs = (double*)malloc(sizeof(double) * n3);
    double* X = (double*)malloc(sizeof(double) * n3);
    double preDii, preDij;
    s->coord = coord;
    orc_prefactors(s, &preDii, &preDij);
    if (s->hydro == 1) {
        D = (double*)malloc(sizeof(double) * (size_t)n3 * n3);
        L = (double*)malloc(sizeof(double) * (size_t)n3 * n3);
    }
    if (refresh < 1) refresh = 1;
    for (step = 0; step < K; ++step) {
        const double* xi = gauss + (size_t)step * n3;
        if (s->hydro == 1) {
            if (step % refresh == 0) {
                orc_D(s, D);
                memcpy(L, D, sizeof(double) * (size_t)n3 * n3);
                if (orc_cholesky(n3, L, n3)) {
                    rep = -1;
                    break;
                }
            }
            orc_df(s, D, F, dt, Rf);
            for (i = 0; i < n3; ++i) X[i] = xi[i] * sqrt(2 * dt);
            orc_trmv_lower(n3, L, n3, X, Rs);
        } else if (s->hydro == 2) {
            orc_df(s, NULL, F, dt, Rf);
            orc_tea(s, NULL, xi, dt, Rs, NULL, NULL);
        } else {
            orc_df(s, NULL, F, dt, Rf);
            for (i = 0; i < n3; ++i) Rs[i] = xi[i] * sqrt(preDii / coord[4 * (i / 3) + 3] * 2 * dt);
        }
        /* diff_equation.c:254-283 */
        for (i = 0; i < s->n; ++i) {
            int k;
            double tmp[3] = {0, 0, 0};
            if (s->flow) {
                const double* G = s->vel_grad;
                const double* c = coord + 4 * i;
                for (k = 0; k < 3; ++k) tmp[k] = dt * (G[3 * k] * c[0] + G[3 * k + 1] * c[1] + G[3 * k + 2] * c[2]);
            }
            for (k = 0; k < 3; ++k)
                coord[4 * i + k] = s->flow ? Rf[3 * i + k] + Rs[3 * i + k] + coord[4 * i + k] + tmp[k]
                                           : Rf[3 * i + k] + Rs[3 * i + k] + coord[4 * i + k];
            if (s->bc == 1)
                for (k = 0; k < 3; ++k)
                    coord[4 * i + k] -= s->box[k] * floor(coord[4 * i + k] * s->inv_L[k] + 0.5f);
        }
        /* forces at curr_time + curr_dt, then curr_time += dt (diff_comp.c:161, 216) */
        s->t = s->t + dt;
        rep |= orc_forces(s, F, NULL, NULL);
        if (traj) memcpy(traj + (size_t)step * 4 * s->n, coord, sizeof(double) * 4 * s->n);
    }
    free(D);
    free(L);
    free(Rf);
    free(Rs);
    free(X);
    return rep;
}

/* K IGT predictor-corrector steps without retries (comp_step_IGT_const,
 * diff_comp.c:76-107; compute_hydro_IGT and compute_hydro_IGT_second_phase,
 * diff_equation.c:288-374). Predictor: the Ermak-McCammon step of
 * compute_hydro_ermak (diff_equation.c:216-286) into r'. Forces F' at r'.
 * Rf0 = (D(r)F + D(r')F')/2 * dt/kT; the stored tensor is averaged,
 * D = (D(r) + D(r'))/2, over the off-diagonal 3x3 blocks (the diagonal
 * blocks do not depend on the positions); corrector: r += Rf0 + L X2 with
 * L = chol(D) and fresh Gaussians, then forces. gauss: K*2*3N (the
 * predictor's 3N, then the corrector's, per step). Hydro none or cholesky.
 * Returns the OR of overlap flags (1: forces at r', 2: forces after the
 * step), or -1 on a failed Cholesky. */
int orc_run_igt_steps(orc_system* s, double* coord, double* F, double dt, int K, const double* gauss,
                      double* traj)
{
    int n3 = 3 * s->n, step, i, k, rep = 0;
    double *D = NULL, *Dp = NULL, *L = NULL;
    double* Rf = (double*)malloc(sizeof(double) * n3);
    double* Rf2 = (double*)malloc(sizeof(double) * n3);
    double* Rs = (double*)malloc(sizeof(double) * n3);
    double* X = (double*)malloc(sizeof(double) * n3);
    double* Fp = (double*)malloc(sizeof(double) * n3);
    double* cp = (double*)malloc(sizeof(double) * 4 * s->n);
    double* FS = (double*)calloc(n3, sizeof(double));
    double preDii, preDij;
    orc_prefactors(s, &preDii, &preDij);
    if (s->hydro == 1) {
        D = (double*)malloc(sizeof(double) * (size_t)n3 * n3);
        Dp = (double*)malloc(sizeof(double) * (size_t)n3 * n3);
        L = (double*)malloc(sizeof(double) * (size_t)n3 * n3);
    }
    for (step = 0; step < K && rep >= 0; ++step) {
        const double* x1 = gauss + (size_t)step * 2 * n3;
        const double* x2 = x1 + n3;
        s->coord = coord;
        /* predictor */
        if (s->hydro == 1) {
            orc_D(s, D);
            orc_df(s, D, F, dt, Rf);
            memcpy(L, D, sizeof(double) * (size_t)n3 * n3);
            if (orc_cholesky(n3, L, n3)) {
                rep = -1;
                break;
            }
            for (i = 0; i < n3; ++i) X[i] = x1[i] * sqrt(2 * dt);
            orc_trmv_lower(n3, L, n3, X, Rs);
        } else {
            orc_df(s, NULL, F, dt, Rf);
            for (i = 0; i < n3; ++i) Rs[i] = x1[i] * sqrt(preDii / coord[4 * (i / 3) + 3] * 2 * dt);
        }
        for (i = 0; i < s->n; ++i) {
            if (s->flow) {
                /* diff_equation.c:265-283: tmp = dt G r, FS = tmp + dt G r' */
                const double* G = s->vel_grad;
                const double* c = coord + 4 * i;
                double tmp[3];
                for (k = 0; k < 3; ++k) tmp[k] = dt * (G[3 * k] * c[0] + G[3 * k + 1] * c[1] + G[3 * k + 2] * c[2]);
                for (k = 0; k < 3; ++k) cp[4 * i + k] = Rf[3 * i + k] + Rs[3 * i + k] + coord[4 * i + k] + tmp[k];
                for (k = 0; k < 3; ++k)
                    FS[3 * i + k] = tmp[k] + dt * (G[3 * k] * cp[4 * i] + G[3 * k + 1] * cp[4 * i + 1] +
                                                   G[3 * k + 2] * cp[4 * i + 2]);
            } else {
                for (k = 0; k < 3; ++k) cp[4 * i + k] = Rf[3 * i + k] + Rs[3 * i + k] + coord[4 * i + k];
            }
            cp[4 * i + 3] = coord[4 * i + 3];
            if (s->bc == 1)
                for (k = 0; k < 3; ++k) cp[4 * i + k] -= s->box[k] * floor(cp[4 * i + k] * s->inv_L[k] + 0.5f);
        }
        /* forces and D(r') F' at the predicted positions, at curr_time +
         * curr_dt like the forces after the step (diff_equation.c:314, 327) */
        const double t0 = s->t;
        s->t = t0 + dt;
        s->coord = cp;
        if (orc_forces(s, Fp, NULL, NULL)) rep |= 1;
        if (s->hydro == 1) {
            orc_D(s, Dp);
            orc_df(s, Dp, Fp, dt, Rf2);
        } else {
            orc_df(s, NULL, Fp, dt, Rf2);
        }
        s->coord = coord;
        for (i = 0; i < n3; ++i) Rf[i] = 0.5 * (Rf[i] + Rf2[i]);
        /* corrector */
        if (s->hydro == 1) {
            int a, b;
            for (a = 0; a < n3; ++a)
                for (b = 0; b < n3; ++b)
                    L[(size_t)a * n3 + b] = a / 3 != b / 3 ? (D[(size_t)a * n3 + b] + Dp[(size_t)a * n3 + b]) / 2
                                                           : D[(size_t)a * n3 + b];
            if (orc_cholesky(n3, L, n3)) {
                rep = -1;
                break;
            }
            for (i = 0; i < n3; ++i) X[i] = x2[i] * sqrt(2 * dt);
            orc_trmv_lower(n3, L, n3, X, Rs);
        } else {
            for (i = 0; i < n3; ++i) Rs[i] = x2[i] * sqrt(preDii / coord[4 * (i / 3) + 3] * 2 * dt);
        }
        for (i = 0; i < s->n; ++i) {
            for (k = 0; k < 3; ++k)
                coord[4 * i + k] += s->flow ? Rf[3 * i + k] + Rs[3 * i + k] + 0.5 * FS[3 * i + k]
                                            : Rf[3 * i + k] + Rs[3 * i + k];
            if (s->bc == 1)
                for (k = 0; k < 3; ++k) coord[4 * i + k] -= s->box[k] * floor(coord[4 * i + k] * s->inv_L[k] + 0.5f);
        }
        if (orc_forces(s, F, NULL, NULL)) rep |= 2;
        if (traj) memcpy(traj + (size_t)step * 4 * s->n, coord, sizeof(double) * 4 * s->n);
    }
    s->coord = coord;
    free(D);
    free(Dp);
    free(L);
    free(Rf);
    free(Rf2);
    free(Rs);
    free(X);
    free(Fp);
    free(cp);
    free(FS);
    return rep;
}

/* ---- elastic-collision overlap removal (ermak_newton) ------------------ */

#define ORC_NEWTON_EPSILON 0.000001 /* data.h:217 (double build) */
#define ORC_NEWTON_OFFSET 0.0001    /* data.h:218 */

/* comp_time (newton.c:57-138), one thread: the earliest time at which an
 * approaching pair (i < j) comes within LJ[2i] + LJ[2j] + NEWTON_OFFSET, and
 * the pairs that reach it, in (i, j) order. The list-size check reads the
 * pair count of the previous call (*npairs on entry), as the reference's
 * global size_pairs. Returns the time (DBL_MAX if no pair approaches). */
static double newton_comp_time(const orc_system* s, const double* coord, const double* vel, int* pairs, int* npairs)
{
    const int prev = *npairs;
    int cnt = 0, i, j;
    double tmin = DBL_MAX;
    for (i = 0; i < s->n; ++i)
        for (j = i + 1; j < s->n; ++j) {
            double r[3], v[3], rv, l;
            dist_vec(s, coord + 4 * j, coord + 4 * i, r);
            l = s->LJ[2 * j] + s->LJ[2 * i] + ORC_NEWTON_OFFSET;
            v[0] = vel[3 * i] - vel[3 * j];
            v[1] = vel[3 * i + 1] - vel[3 * j + 1];
            v[2] = vel[3 * i + 2] - vel[3 * j + 2];
            rv = r[0] * v[0] + r[1] * v[1] + r[2] * v[2];
            if (rv < 0) {
                double vv = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
                double delta = rv * rv - vv * ((r[0] * r[0] + r[1] * r[1] + r[2] * r[2]) - l * l);
                if (delta > 0) {
                    double t2, inv_vv = 1 / vv;
                    delta = sqrt(delta);
                    t2 = -(rv + delta) * inv_vv;
                    if (t2 < 0) t2 = 0;
                    if (t2 <= tmin) {
                        cnt = (t2 < tmin) ? 0 : cnt;
                        if (prev + 1 < 2 * s->n) {
                            pairs[cnt] = i;
                            pairs[cnt + 1] = j;
                            cnt += 2;
                        }
                        tmin = t2;
                    }
                }
            }
        }
    *npairs = cnt;
    return tmin;
}

/* newton_moves (newton.c:140-200): ballistic moves with velocities vel to
 * just before the earliest contact, elastic collisions of the pairs that
 * reach it (restitution e_collision, masses), until dt has elapsed.
 * Returns 1 if a move leaves the sphere (bc 2, iscorrect), 0 otherwise, -2
 * when *count exceeds move_attempts ("Ermak Newton error"). */
static int newton_moves(const orc_system* s, double* coord, double* vel, const double* masses, double e_collision,
                        double dt, int move_attempts, int* count, int* pairs, int* npairs)
{
    double elapsed = 0.0;
    int ret = 0, i, j;
    while (elapsed < dt - 2 * ORC_NEWTON_EPSILON) {
        double next;
        ret = 0;
        next = newton_comp_time(s, coord, vel, pairs, npairs);
        if (next < 0 || next > dt - elapsed) next = dt - elapsed;
        next = (next > ORC_NEWTON_EPSILON) ? next - ORC_NEWTON_EPSILON : 0;
        elapsed += next;
        if (next > 0.0) {
            for (j = 0; j < s->n; ++j) {
                int k;
                for (k = 0; k < 3; ++k) coord[4 * j + k] += vel[3 * j + k] * next;
                if (s->bc == 1)
                    for (k = 0; k < 3; ++k) coord[4 * j + k] -= s->box[k] * floor(coord[4 * j + k] * s->inv_L[k] + 0.5f);
            }
            if (s->bc == 2) {
                /* iscorrect (trans.c:130-145) */
                double sr = s->sphere_radius * s->sphere_radius;
                for (j = 0; j < s->n && !ret; ++j) {
                    const double* c = coord + 4 * j;
                    ret = c[0] * c[0] + c[1] * c[1] + c[2] * c[2] > sr;
                }
            }
        }
        if (ret) break;
        for (i = 0; i < *npairs / 2; ++i) {
            int p1 = pairs[2 * i], p2 = pairs[2 * i + 1], k;
            double e[3], v[3], ev, rr, inv, m1 = masses[p1], m2 = masses[p2];
            /* get_v2_norms(p2, p1) (math_help.c:40-55) */
            dist_vec(s, coord + 4 * p2, coord + 4 * p1, e);
            rr = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
            inv = 1 / rr;
            e[0] *= inv;
            e[1] *= inv;
            e[2] *= inv;
            for (k = 0; k < 3; ++k) v[k] = vel[3 * p1 + k] - vel[3 * p2 + k];
            ev = e[0] * v[0] + e[1] * v[1] + e[2] * v[2];
            ev *= (1 + e_collision) / (m1 + m2);
            for (k = 0; k < 3; ++k) vel[3 * p1 + k] -= m2 * ev * e[k];
            for (k = 0; k < 3; ++k) vel[3 * p2 + k] += m1 * ev * e[k];
        }
        ++(*count);
        if (*count > move_attempts) return -2;
    }
    return ret;
}

/* one Ermak-McCammon move from coord with forces F (compute_hydro_ermak,
 * diff_equation.c:216-286; the tensor and its factor at coord, refresh 1) */
static int ermak_move(orc_system* s, double* coord, const double* F, double dt, const double* xi, double* D,
                      double* L, double* Rf, double* Rs, double* X, double preDii)
{
    int n3 = 3 * s->n, i, k;
    s->coord = coord;
    if (s->hydro == 1) {
        orc_D(s, D);
        memcpy(L, D, sizeof(double) * (size_t)n3 * n3);
        if (orc_cholesky(n3, L, n3)) return -1;
        orc_df(s, D, F, dt, Rf);
        for (i = 0; i < n3; ++i) X[i] = xi[i] * sqrt(2 * dt);
        orc_trmv_lower(n3, L, n3, X, Rs);
    } else if (s->hydro == 2) {
        orc_df(s, NULL, F, dt, Rf);
        orc_tea(s, NULL, xi, dt, Rs, NULL, NULL);
    } else {
        orc_df(s, NULL, F, dt, Rf);
        for (i = 0; i < n3; ++i) Rs[i] = xi[i] * sqrt(preDii / coord[4 * (i / 3) + 3] * 2 * dt);
    }
    for (i = 0; i < s->n; ++i) {
        double tmp[3] = {0, 0, 0};
        if (s->flow) {
            const double* G = s->vel_grad;
            const double* c = coord + 4 * i;
            for (k = 0; k < 3; ++k) tmp[k] = dt * (G[3 * k] * c[0] + G[3 * k + 1] * c[1] + G[3 * k + 2] * c[2]);
        }
        for (k = 0; k < 3; ++k)
            coord[4 * i + k] = s->flow ? Rf[3 * i + k] + Rs[3 * i + k] + coord[4 * i + k] + tmp[k]
                                       : Rf[3 * i + k] + Rs[3 * i + k] + coord[4 * i + k];
        if (s->bc == 1)
            for (k = 0; k < 3; ++k) coord[4 * i + k] -= s->box[k] * floor(coord[4 * i + k] * s->inv_L[k] + 0.5f);
    }
    return 0;
}

int orc_run_newton_steps(orc_system* s, double* coord, double* F, double dt, int K, const double* gauss,
                         int n_gauss, const double* masses, double e_collision, int move_attempts, double* traj,
                         int* used, int* rounds)
{
    int n3 = 3 * s->n, step, rc = 0, g = 0, count_total = 0;
    double *D = NULL, *L = NULL, preDii, preDij;
    double* Rf = (double*)malloc(sizeof(double) * n3);
    double* Rs = (double*)malloc(sizeof(double) * n3);
    double* X = (double*)malloc(sizeof(double) * n3);
    double* vel = (double*)malloc(sizeof(double) * n3);
    double* save = (double*)malloc(sizeof(double) * 4 * s->n);
    double* Fsave = (double*)malloc(sizeof(double) * n3);
    int* pairs = (int*)malloc(sizeof(int) * 2 * s->n);
    int npairs = 0;   /* the reference's global size_pairs */
    orc_prefactors(s, &preDii, &preDij);
    if (s->hydro == 1) {
        D = (double*)malloc(sizeof(double) * (size_t)n3 * n3);
        L = (double*)malloc(sizeof(double) * (size_t)n3 * n3);
    }
    for (step = 0; step < K && rc >= 0; ++step) {
        /* comp_step_ermak_newton (diff_comp.c:181-210) */
        const double t0 = s->t;
        int count = 0, ret = 1, i;
        memcpy(save, coord, sizeof(double) * 4 * s->n);
        memcpy(Fsave, F, sizeof(double) * n3);
        while (ret) {
            if (g >= n_gauss) {
                rc = -3;
                break;
            }
            if (ermak_move(s, coord, F, dt, gauss + (size_t)g * n3, D, L, Rf, Rs, X, preDii)) {
                rc = -1;
                break;
            }
            ++g;
            s->t = t0 + dt;
            ret = orc_forces(s, F, NULL, NULL);
            if (ret) {
                /* newton_init_vel (newton.c:202-213), load_coord, newton_moves */
                double inv_t = 1.0 / dt;
                for (i = 0; i < s->n; ++i) {
                    dist_vec(s, save + 4 * i, coord + 4 * i, vel + 3 * i);
                    vel[3 * i] *= inv_t;
                    vel[3 * i + 1] *= inv_t;
                    vel[3 * i + 2] *= inv_t;
                }
                memcpy(coord, save, sizeof(double) * 4 * s->n);
                ret = newton_moves(s, coord, vel, masses, e_collision, dt, move_attempts, &count, pairs, &npairs);
                if (ret == -2) {
                    rc = -2;
                    break;
                }
                ret = ret || orc_forces(s, F, NULL, NULL);
                if (ret) {
                    memcpy(coord, save, sizeof(double) * 4 * s->n);
                    memcpy(F, Fsave, sizeof(double) * n3);
                    s->t = t0;
                }
            }
        }
        count_total += count;
        if (traj) memcpy(traj + (size_t)step * 4 * s->n, coord, sizeof(double) * 4 * s->n);
    }
    s->coord = coord;
    if (used) *used = g;
    if (rounds) *rounds = count_total;
    free(D);
    free(L);
    free(Rf);
    free(Rs);
    free(X);
    free(vel);
    free(save);
    free(Fsave);
    free(pairs);
    return rc;
}
