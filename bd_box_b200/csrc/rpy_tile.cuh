// RPY diffusion-tensor tiles, shared by the stored-D build and the
// matrix-free D.F / TEA kernels.
//
// A tile is the symmetric 3x3 block D_ij, kept as 6 values
// {xx, yy, zz, xy, xz, yz}.
//  * rpy_free: diff_tensor_calc_pos (diff_alg/diff_tensor.c:45-92), the
//    free-space Rotne-Prager-Yamakawa tensor with the overlap form for
//    r < a_i + a_j.
//  * rpy_ewald_tab: diff_tensor_calc_ewald_beenakker (diff_tensor.c:265-401)
//    with its self term (:404-422): real-space images r + L m and
//    reciprocal vectors over the same sphere |m|^2 <= R^2, overlap
//    correction on the raw (not minimum-image) separation, alpha = sqrt(pi)/L
//    (init_tensor, :546-559). Constants that the reference forms from the
//    float literal M_PIF are formed the same way on the host.
//  * rpy_smith_tab: diff_tensor_calc_ewald_smith (diff_tensor.c:102-243) with
//    its self term (:245-263): Oseen (O) and sigma^2 (Q) sums over the
//    images r/L + m and the reciprocal vectors of the same sphere, in units
//    of L, alpha = ewald_alpha, preO = 0.75/L, preQ = sigma^2/(2 L^3).
#pragma once

#include "bdb_common.cuh"

namespace bdb {

struct EwaldConst {
    double L, inv_L, alpha, alpha2, alpha3, inv_alpha2, preQ;
    double two_pif;      // 2*M_PIF evaluated in float
    double four_pif2;    // 4*M_PIF*M_PIF evaluated in float
    double six_pif;      // 6*M_PIF evaluated in float
    int R, rr_sq;
    // lattice tables (device memory, built by ewald_tables on the host):
    // rk[12 k ..]: h, f, g, A_k, B_k, then 2(1 - e_a^2) for a = x, y, z and
    // -2 e_a e_b for xy, xz, yz, over one half of the reciprocal sphere
    // (k and -k contribute alike); img[m]: the real-space image offsets L m
    const double* rk = nullptr;
    const double4* img = nullptr;
    int nk = 0, nimg = 0;
    float rcut_sq = 0.f;   // mixed precision: real-space images beyond this are dropped
    // Smith (rpy_smith_tab): rk rows are h, f, g, then the identity, e e^T
    // and sigma^2 e e^T coefficients (k and -k together), then the six
    // products e_a e_b (xx, yy, zz, xy, xz, yz)
    int smith = 0;
    double s_alpha = 0, s_alpha2 = 0, s_alpha3 = 0;
    float s_rcut_sq = 0.f;   // mixed precision: (4.45/alpha)^2 in units of L^2, erfc(4.45) ~ 3e-10
};

// 1/sqrt(pi) as the reference's double build spells it (data.h:228)
#define BDB_M1_SQRTPI 0.5641895835

inline EwaldConst make_ewald(double L, double inv_L, int R)
{
    EwaldConst e;
    e.L = L;
    e.inv_L = inv_L;
    e.alpha = BDB_SQRTPI * inv_L;
    e.alpha2 = e.alpha * e.alpha;
    e.alpha3 = e.alpha * e.alpha2;
    e.inv_alpha2 = 1.0f / e.alpha2;
    e.preQ = inv_L * inv_L * inv_L;
    volatile float pif = BDB_M_PIF;
    volatile float two = 2 * pif;
    volatile float four = 4 * pif;
    volatile float four2 = four * pif;
    volatile float six = 6 * pif;
    e.two_pif = two;
    e.four_pif2 = four2;
    e.six_pif = six;
    e.R = R;
    e.rr_sq = R * R;
    return e;
}

inline EwaldConst make_ewald_smith(double L, double inv_L, int R, double alpha)
{
    EwaldConst e = make_ewald(L, inv_L, R);
    e.smith = 1;
    e.s_alpha = alpha;
    e.s_alpha2 = alpha * alpha;
    e.s_alpha3 = alpha * e.s_alpha2;
    e.s_rcut_sq = (float)((4.45 / alpha) * (4.45 / alpha));
    return e;
}

// diff_tensor_calc_pos(i, j): sigma_i is bead j's radius, sigma_j bead i's,
// e = (r_i - r_j)/|r_i - r_j|.
template <typename T>
__device__ __forceinline__ void rpy_free(const double4& pi, const double4& pj, T preDii, T preDij, T* t)
{
    const T si = (T)pj.w, sj = (T)pi.w;
    T e0 = (T)(pi.x - pj.x), e1 = (T)(pi.y - pj.y), e2 = (T)(pi.z - pj.z);
    const T r_sq = e0 * e0 + e1 * e1 + e2 * e2;
    const T r = sqrt(r_sq);
    const T inv = (T)1 / r;
    e0 *= inv;
    e1 *= inv;
    e2 *= inv;
    if (r < si + sj) {
        const T sigma = (si + sj) / 2;
        const T pre = preDii / sigma;
        const T q = r / (32 * sigma);
        const T part1 = 1 - 9 * q;
        const T q3 = 3 * q;
        t[0] = (part1 + q3 * e0 * e0) * pre;
        t[1] = (part1 + q3 * e1 * e1) * pre;
        t[2] = (part1 + q3 * e2 * e2) * pre;
        t[3] = pre * q3 * e0 * e1;
        t[4] = pre * q3 * e0 * e2;
        t[5] = pre * q3 * e1 * e2;
    } else {
        const T pre = preDij / r;
        const T sigm_r = (si * si + sj * sj) / r_sq;
        const T a = 1 + sigm_r / 3;
        const T b = 1 - sigm_r;
        t[0] = (a + e0 * e0 * b) * pre;
        t[1] = (a + e1 * e1 * b) * pre;
        t[2] = (a + e2 * e2 * b) * pre;
        t[3] = pre * e0 * e1 * b;
        t[4] = pre * e0 * e2 * b;
        t[5] = pre * e1 * e2 * b;
    }
}

// diff_tensor_calc_ewald_beenakker(i, j) (+ _diag for i == j) from the
// lattice tables: each reciprocal vector once for the pair k, -k, with its
// k-only factors precomputed. The FP64 path keeps every real-space image
// and the reference's cos(2 pi_f k.r). With MIXED the real-space images are
// summed in FP32 (images beyond rcut dropped) and the reciprocal phases
// taken as FP32 cosines of the same argument, both accumulated in FP64.
template <bool MIXED>
__device__ __forceinline__ void rpy_ewald_tab(const double4& pi, const double4& pj, bool self, double preDii,
                                              double preDij, const EwaldConst& ec, double* t)
{
    const double sigma_i = pj.w, sigma_j = pi.w;
    const double r0 = pj.x - pi.x, r1 = pj.y - pi.y, r2 = pj.z - pi.z;
    const double sigma_sq = 0.5 * (sigma_i * sigma_i + sigma_j * sigma_j);
    double O[6] = {0, 0, 0, 0, 0, 0}, Qr[6] = {0, 0, 0, 0, 0, 0};
    for (int k = 0; k < 6; ++k) t[k] = 0;
    const double rr = r0 * r0 + r1 * r1 + r2 * r2;
    if (!self && rr < (sigma_i + sigma_j) * (sigma_i + sigma_j)) {
        const double r = sqrt(rr), inv = 1 / r;
        const double e[3] = {r0 * inv, r1 * inv, r2 * inv};
        const double sigma = (sigma_i + sigma_j) / 2;
        const double pre = preDii / sigma;
        const double part1 = 1 - (9 * r / (32 * sigma));
        const double pre2 = preDij / r;
        const double sigm_r = (sigma_i * sigma_i + sigma_j * sigma_j) / rr;
        const double p1 = 1 + sigm_r / 3;
        const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
        for (int k = 0; k < 3; ++k)
            t[k] += pre * (part1 + 3 * e[k] * e[k] * r / (32 * sigma)) - pre2 * (p1 + e[k] * e[k] * (1 - sigm_r));
        for (int k = 3; k < 6; ++k)
            t[k] += pre * 3 * e[ia[k]] * e[ib[k]] * r / (32 * sigma) - pre2 * e[ia[k]] * e[ib[k]] * (1 - sigm_r);
    }
    // real space
    if (MIXED) {
        const float a = (float)ec.alpha, a2 = (float)ec.alpha2, a3 = (float)ec.alpha3;
        const float s2 = (float)sigma_sq;
        const float a5s = 20.f * a2 * a3 * s2, a5s16 = 16.f * a2 * a3 * s2, a7s = 4.f * a3 * a2 * a2 * s2;
        const float c0 = 14.f * a3 * s2 - 4.5f * a, c0b = -2.f * a3 * s2 + 1.5f * a;
        const float isp = (float)(1.0 / BDB_SQRTPI);
        const float fx = (float)r0, fy = (float)r1, fz = (float)r2;
        float o[6] = {0, 0, 0, 0, 0, 0};
        for (int m = 0; m < ec.nimg; ++m) {
            const double4 off = ec.img[m];
            const float x = fx + (float)off.x, y = fy + (float)off.y, z = fz + (float)off.z;
            const float r_sq = x * x + y * y + z * z;
            if (r_sq == 0.f || r_sq > ec.rcut_sq) continue;
            const float inv_r = rsqrtf(r_sq), inv_r2 = inv_r * inv_r, inv_r3 = inv_r * inv_r2, r = r_sq * inv_r;
            const float ex = __expf(-a2 * r_sq) * isp;
            const float ec_ = erfcf(r * a);
            const float sc = (a * s2 * inv_r2 + c0 - a5s * r_sq + 3.f * a3 * r_sq + a7s * r_sq * r_sq) * ex +
                             ec_ * (0.75f * inv_r + 0.5f * s2 * inv_r3);
            const float sc2 = (-3.f * a * s2 * inv_r2 + c0b + a5s16 * r_sq - 3.f * a3 * r_sq - a7s * r_sq * r_sq) * ex +
                              ec_ * (0.75f * inv_r - 1.5f * s2 * inv_r3);
            const float e0 = x * inv_r, e1 = y * inv_r, e2 = z * inv_r;
            o[0] += sc + sc2 * e0 * e0;
            o[1] += sc + sc2 * e1 * e1;
            o[2] += sc + sc2 * e2 * e2;
            o[3] += sc2 * e0 * e1;
            o[4] += sc2 * e0 * e2;
            o[5] += sc2 * e1 * e2;
        }
        for (int k = 0; k < 6; ++k) O[k] = o[k];
    } else {
        const double a = ec.alpha, a2 = ec.alpha2, a3 = ec.alpha3;
        for (int m = 0; m < ec.nimg; ++m) {
            const double4 off = ec.img[m];
            const double x = r0 + off.x, y = r1 + off.y, z = r2 + off.z;
            const double r_sq = x * x + y * y + z * z;
            if (r_sq == 0.0) continue;
            const double r = sqrt(r_sq);
            const double inv_r = 1 / r, inv_r2 = 1 / r_sq, inv_r3 = inv_r * inv_r2;
            const double e[3] = {x * inv_r, y * inv_r, z * inv_r};
            const double ex = exp(-a2 * r_sq);
            const double ec_ = erfc(r * a);
            double sc = a * sigma_sq * inv_r2 + 14 * a3 * sigma_sq - 4.5 * a - 20 * a2 * a3 * sigma_sq * r_sq +
                        3 * a3 * r_sq + 4 * a3 * a2 * a2 * sigma_sq * r_sq * r_sq;
            sc = sc * ex / BDB_SQRTPI + ec_ * (0.75 * inv_r + 0.5 * sigma_sq * inv_r3);
            double sc2 = -3 * a * sigma_sq * inv_r2 - 2 * a3 * sigma_sq + 1.5 * a + 16 * a2 * a3 * sigma_sq * r_sq -
                         3 * a3 * r_sq - 4 * a3 * a2 * a2 * sigma_sq * r_sq * r_sq;
            sc2 = sc2 * ex / BDB_SQRTPI + ec_ * (0.75 * inv_r - 1.5 * sigma_sq * inv_r3);
            O[0] += sc + sc2 * e[0] * e[0];
            O[1] += sc + sc2 * e[1] * e[1];
            O[2] += sc + sc2 * e[2] * e[2];
            O[3] += sc2 * e[0] * e[1];
            O[4] += sc2 * e[0] * e[2];
            O[5] += sc2 * e[1] * e[2];
        }
    }
    // reciprocal space
    const double v0 = r0 * ec.inv_L, v1 = r1 * ec.inv_L, v2 = r2 * ec.inv_L;
    for (int k = 0; k < ec.nk; ++k) {
        const double* q = ec.rk + 12 * k;
        const double ph = v0 * q[0] + v1 * q[1] + v2 * q[2];
        double cs;
        if (MIXED) {
            // cos(2 pi_f ph), pi_f the float pi of the reference's constants
            cs = (double)cospif((float)(ph * (ec.two_pif / BDB_PI_D)));
        } else {
            cs = cos(ec.two_pif * ph);
        }
        const double sc = (q[3] - sigma_sq * q[4]) * cs;
        for (int c = 0; c < 6; ++c) Qr[c] += sc * q[5 + c];
    }
    for (int k = 0; k < 6; ++k) t[k] += preDii * (O[k] + ec.preQ * Qr[k]);
    if (self) {
        const double aw = pi.w;
        const double a = ec.alpha, a3 = ec.alpha3;
        const double sc3 = (-6 * a / BDB_SQRTPI + 40 * a3 * aw * aw / (3 * BDB_SQRTPI)) * preDii;
        for (int k = 0; k < 3; ++k) t[k] = preDii / aw + sc3 + t[k];
        t[3] = t[4] = t[5] = 0;
    }
}

// diff_tensor_calc_ewald_smith(i, j) (+ _diag for i == j) from the lattice
// tables. The FP64 path keeps every real-space image; with MIXED the
// real-space images are summed in FP32 (images beyond 4.45/alpha dropped,
// 2.5 L at the default alpha = sqrt(pi): erfc there is below 3e-10) and the
// reciprocal phases taken as FP32 cosines of the same argument, both
// accumulated in FP64.
template <bool MIXED>
__device__ __forceinline__ void rpy_smith_tab(const double4& pi, const double4& pj, bool self, double preDii,
                                              double preDij, const EwaldConst& ec, double* t)
{
    const double sigma_i = pj.w, sigma_j = pi.w;
    // dist_vec(coord_j, coord_i): v = r_i - r_j, no minimum image
    const double r0 = pi.x - pj.x, r1 = pi.y - pj.y, r2 = pi.z - pj.z;
    const double sigma_sq = 0.5 * (sigma_i * sigma_i + sigma_j * sigma_j);
    const double preO = 0.75 * ec.inv_L;
    const double preQ = 0.5 * sigma_sq * ec.inv_L * ec.inv_L * ec.inv_L;
    for (int k = 0; k < 6; ++k) t[k] = 0;
    const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
    const double rr = r0 * r0 + r1 * r1 + r2 * r2;
    if (!self && rr < (sigma_i + sigma_j) * (sigma_i + sigma_j)) {
        const double r = sqrt(rr), inv = 1 / r;
        const double e[3] = {r0 * inv, r1 * inv, r2 * inv};
        const double sigma = (sigma_i + sigma_j) / 2;
        const double pre = preDii / sigma;
        const double part1 = 1 - (9 * r / (32 * sigma));
        const double pre2 = preDij / r;
        const double sigm_r = (sigma_i * sigma_i + sigma_j * sigma_j) / rr;
        const double p1 = 1 + sigm_r / 3;
        for (int k = 0; k < 3; ++k)
            t[k] += pre * (part1 + 3 * e[k] * e[k] * r / (32 * sigma)) - pre2 * (p1 + e[k] * e[k] * (1 - sigm_r));
        for (int k = 3; k < 6; ++k)
            t[k] += pre * 3 * e[ia[k]] * e[ib[k]] * r / (32 * sigma) - pre2 * e[ia[k]] * e[ib[k]] * (1 - sigm_r);
    }
    const double v0 = r0 * ec.inv_L, v1 = r1 * ec.inv_L, v2 = r2 * ec.inv_L;
    const double a = ec.s_alpha, a2 = ec.s_alpha2, a3 = ec.s_alpha3;
    double O[6] = {0, 0, 0, 0, 0, 0}, Q[6] = {0, 0, 0, 0, 0, 0};
    // real space: images v + m (m from the image table, stored as L m)
    if (MIXED) {
        const float fa = (float)a, fa2 = (float)a2, fa3 = (float)a3, isp = (float)BDB_M1_SQRTPI;
        const float fx = (float)v0, fy = (float)v1, fz = (float)v2;
        float o[6] = {0, 0, 0, 0, 0, 0}, qq[6] = {0, 0, 0, 0, 0, 0};
        for (int m = 0; m < ec.nimg; ++m) {
            const double4 off = ec.img[m];
            const float x = fx + (float)rint(off.x * ec.inv_L), y = fy + (float)rint(off.y * ec.inv_L),
                        z = fz + (float)rint(off.z * ec.inv_L);
            const float r_sq = x * x + y * y + z * z;
            if (r_sq == 0.f || r_sq > ec.s_rcut_sq) continue;
            const float inv_r = rsqrtf(r_sq), r = r_sq * inv_r, inv_r3 = inv_r * inv_r * inv_r;
            const float e0 = x * inv_r, e1 = y * inv_r, e2 = z * inv_r;
            const float er = erfcf(r * fa), ex = __expf(-fa2 * r_sq);
            const float so = er * inv_r, so2 = so + 2.f * fa * isp * ex;
            const float sq = inv_r3 * (er + 2.f * fa * r * isp * ex);
            const float sq2 = -3.f * sq - 4.f * fa3 * isp * ex;
            o[0] += so + so2 * e0 * e0;
            o[1] += so + so2 * e1 * e1;
            o[2] += so + so2 * e2 * e2;
            o[3] += so2 * e0 * e1;
            o[4] += so2 * e0 * e2;
            o[5] += so2 * e1 * e2;
            qq[0] += sq + sq2 * e0 * e0;
            qq[1] += sq + sq2 * e1 * e1;
            qq[2] += sq + sq2 * e2 * e2;
            qq[3] += sq2 * e0 * e1;
            qq[4] += sq2 * e0 * e2;
            qq[5] += sq2 * e1 * e2;
        }
        for (int k = 0; k < 6; ++k) {
            O[k] = o[k];
            Q[k] = qq[k];
        }
    }
    for (int m = 0; !MIXED && m < ec.nimg; ++m) {
        const double4 off = ec.img[m];
        const double x = v0 + rint(off.x * ec.inv_L), y = v1 + rint(off.y * ec.inv_L), z = v2 + rint(off.z * ec.inv_L);
        const double r_sq = x * x + y * y + z * z;
        if (r_sq == 0.0) continue;
        const double r = sqrt(r_sq);
        const double inv_r = 1 / r, inv_r3 = 1 / (r * r_sq);
        const double e[3] = {x * inv_r, y * inv_r, z * inv_r};
        const double er = erfc(r * a), ex = exp(-a2 * r_sq);
        const double so = er * inv_r, so2 = so + 2 * a * BDB_M1_SQRTPI * ex;
        const double sq = inv_r3 * (er + 2 * a * r * BDB_M1_SQRTPI * ex);
        const double sq2 = -3 * sq - 4 * a3 * BDB_M1_SQRTPI * ex;
        for (int k = 0; k < 3; ++k) {
            O[k] += so + so2 * e[k] * e[k];
            Q[k] += sq + sq2 * e[k] * e[k];
        }
        for (int k = 3; k < 6; ++k) {
            O[k] += so2 * e[ia[k]] * e[ib[k]];
            Q[k] += sq2 * e[ia[k]] * e[ib[k]];
        }
    }
    // reciprocal space: one row per pair k, -k
    double Rc[6] = {0, 0, 0, 0, 0, 0};
    for (int k = 0; k < ec.nk; ++k) {
        const double* q = ec.rk + 12 * k;
        const double ph = v0 * q[0] + v1 * q[1] + v2 * q[2];
        // cos(2 pi_f ph), pi_f the float pi of the reference's constants
        const double cs = MIXED ? (double)cospif((float)(ph * (ec.two_pif / BDB_PI_D))) : cos(ec.two_pif * ph);
        const double ci = q[3] * cs, ce = (q[4] + sigma_sq * q[5]) * cs;
        for (int c = 0; c < 3; ++c) Rc[c] += ci + ce * q[6 + c];
        for (int c = 3; c < 6; ++c) Rc[c] += ce * q[6 + c];
    }
    for (int k = 0; k < 6; ++k) t[k] += preDii * (preO * O[k] + preQ * Q[k] + Rc[k]);
    if (self) {
        const double aw = pi.w, il = ec.inv_L;
        double sc3 = a * aw * il;
        sc3 = sc3 * sc3 * sc3 * BDB_M1_SQRTPI / 3;
        sc3 = 0.75 * il * 1.5 * a * aw * BDB_M1_SQRTPI * il + 0.5 * aw * aw * il * il * il * sc3;
        sc3 *= preDii;
        for (int k = 0; k < 3; ++k) t[k] = preDii / aw - sc3 + t[k];
        t[3] = t[4] = t[5] = 0;
    }
}

}  // namespace bdb
