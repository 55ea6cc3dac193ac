// Hand-written adjoint of the Ermak-McCammon step with Cholesky noise.
//
// One step (diff_equation.c:216-286 with compute_r's Cholesky branch,
// diff_rand.c:64-85) maps x to
//     x' = x + c D(x) F(x; theta) + B(x) X,   c = dt/(kB T), B = chol(D),
// with X = sqrt(2 dt) xi the step's fixed noise. Given lambda' = dL/dx', the
// adjoint step returns
//     lambda = lambda' + c [ (dD/dx : F)^T lambda' + (dF/dx)^T (D lambda') ]
//                     + (d(B X)/dx)^T lambda'
//     theta_bar += c (D lambda')^T dF/dtheta.
// * D is a sum of pair tiles T(x_i - x_j) (free-space RPY with the overlap
//   form; the diagonal tiles do not depend on x), so every x-derivative of a
//   contraction <G, D> is a pair sum of grad_r <G_ij, T(r)> (k_tile_grad).
// * The forces are conservative, dF/dx is symmetric, and its product with
//   u = D lambda' is a pair sum over bonds, LJ and Debye-Hueckel pairs with
//   the forward pass's cutoffs and bonded scaling (k_force_jvp), which also
//   accumulates u^T dF/dtheta for the four force-field scale factors.
// * The Cholesky factor's derivative dB = B Phi(B^-1 dD B^-T), Phi = lower
//   triangle with half the diagonal, gives
//     lambda'^T dB X = <Dbar, dD>,  Dbar = B^-T Phi(v X^T) B^-1,  v = B^T lambda',
//   formed with two blocked triangular solves (k_gemm_tn, k_trinv64).
// The forward pass is recomputed from checkpoints every `checkpoint` steps.
// Precision follows the system's: FP64 throughout for an FP64 system; for a
// mixed-precision system (FP32 tensor, FP16-split Cholesky) the forward steps
// are the mixed path's, and the backward's O(n^3) part -- Phi(v X^T), the
// two blocked triangular solves and their transposes -- runs in FP32 on its
// FP32 factor, while the O(N^2) tile gradients and force products keep FP64
// arithmetic and FP64 sums.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "bdb_common.cuh"

namespace bdb {

// ---------------------------------------------------------------- tiles

// T(r) = A(r) I + Bc(r) e e^T (rpy_free); the gradient of <G, T(r)> with
// respect to r = x_i - x_j needs A', Bc and Bc'. si is bead j's radius, sj
// bead i's.
__device__ __forceinline__ void tile_grad(const double* r, double si, double sj, double preDii, double preDij,
                                          const double* G, double* g)
{
    const double r_sq = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    const double rn = sqrt(r_sq);
    const double e[3] = {r[0] / rn, r[1] / rn, r[2] / rn};
    double Bc, dA, dB;
    if (rn < si + sj) {
        const double sigma = (si + sj) / 2;
        const double pre = preDii / sigma;
        Bc = pre * 3 * rn / (32 * sigma);
        dA = -9 * pre / (32 * sigma);
        dB = 3 * pre / (32 * sigma);
    } else {
        const double S = si * si + sj * sj;
        Bc = preDij / rn - preDij * S / (rn * r_sq);
        dA = -preDij / r_sq - preDij * S / (r_sq * r_sq);
        dB = -preDij / r_sq + 3 * preDij * S / (r_sq * r_sq);
    }
    const double tr = G[0] + G[4] + G[8];
    double Ge[3], GTe[3];
    for (int a = 0; a < 3; ++a) {
        Ge[a] = G[3 * a] * e[0] + G[3 * a + 1] * e[1] + G[3 * a + 2] * e[2];
        GTe[a] = G[a] * e[0] + G[3 + a] * e[1] + G[6 + a] * e[2];
    }
    const double eGe = e[0] * Ge[0] + e[1] * Ge[1] + e[2] * Ge[2];
    for (int a = 0; a < 3; ++a)
        g[a] = (dA * tr + dB * eGe) * e[a] + Bc / rn * (Ge[a] + GTe[a] - 2 * eGe * e[a]);
}

// grad_i += sum_{j != i} grad_r <G_ij, T(x_i - x_j)> with
//   G_ij = c (lam_i F_j^T + lam_j F_i^T) + S_ij,
// S the (symmetric) noise weight matrix Z + Z^T (3x3 tile ij, row-major, ld),
// or none. One warp per bead, lanes over j, fixed-order reduction.
template <typename T>
__global__ void k_tile_grad(int n, const double4* __restrict__ pos, double preDii, double preDij, double c,
                            const double* __restrict__ lam, const double* __restrict__ F,
                            const T* __restrict__ S, int ld, double* __restrict__ grad)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (i >= n) return;
    const double4 pi = pos[i];
    double li[3], fi[3];
    for (int a = 0; a < 3; ++a) {
        li[a] = lam[3 * i + a];
        fi[a] = F[3 * i + a];
    }
    double acc[3] = {0, 0, 0};
    for (int j = lane; j < n; j += 32) {
        if (j == i) continue;
        const double4 pj = pos[j];
        const double r[3] = {pi.x - pj.x, pi.y - pj.y, pi.z - pj.z};
        double G[9];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                G[3 * a + b] = c * (li[a] * F[3 * j + b] + lam[3 * j + a] * fi[b]) +
                               (S ? (double)S[(size_t)(3 * i + a) * ld + 3 * j + b] : 0.0);
        double g[3];
        tile_grad(r, pj.w, pi.w, preDii, preDij, G, g);
        acc[0] += g[0];
        acc[1] += g[1];
        acc[2] += g[2];
    }
    for (int o = 16; o > 0; o >>= 1)
        for (int a = 0; a < 3; ++a) acc[a] += __shfl_xor_sync(0xffffffffu, acc[a], o);
    if (lane == 0)
        for (int a = 0; a < 3; ++a) grad[3 * i + a] += acc[a];
}

// ---------------------------------------------------------------- forces

struct AdjForce {
    int elec;
    double epsilon_c, kappa_c, gamma_c, cutoff_c;
    double alpha_lj, cutoff_lj, lj6;
    double bond_lj_scale, bond_c_scale;
    int conn_live;
};

__device__ __forceinline__ bool adj_conn(const int* conn_ptr, const int* conn_list, int i, int j)
{
    for (int k = conn_ptr[i]; k < conn_ptr[i + 1]; ++k)
        if (conn_list[k] == j) return true;
    return false;
}

// the pair force on bead i is Fm(r) d / r with d = x_i - x_j; add the
// directional derivative along du = u_i - u_j and the parameter terms
__device__ __forceinline__ void pair_jvp(double Fm, double dFm, const double* d, double rn, const double* du,
                                         double* jvp)
{
    const double phi = Fm / rn;
    const double k2 = (dFm * rn - Fm) / (rn * rn * rn);
    const double dd = d[0] * du[0] + d[1] * du[1] + d[2] * du[2];
    for (int a = 0; a < 3; ++a) jvp[a] += phi * du[a] + k2 * dd * d[a];
}

// grad_i += c (dF/dx u)_i and ppart[4 i + k] = c u_i . dF_i/ds_k for the
// scale factors s = (LJ epsilon, LJ sigma, bond H, Debye length), following
// force_single (calc_func.c:370-409), LJ_force (LJ.c:37-64), electro_force
// (electro.c:36-56) and bond_calc (bond.c:43-85). One warp per bead: lanes
// over all other beads (the forward pass's cutoffs and 1-2 scaling decide
// which pairs act), then the bead's bonds.
__global__ void k_force_jvp(int n, AdjForce fp, const double4* __restrict__ pos, const double* __restrict__ Q,
                            const double2* __restrict__ LJ, const int* __restrict__ conn_ptr,
                            const int* __restrict__ conn_list, const int* __restrict__ bptr,
                            const int* __restrict__ blist, const int* __restrict__ bond_pairs,
                            const double* __restrict__ bond_parms, const double* __restrict__ u, double c,
                            double* __restrict__ grad, double* __restrict__ ppart)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (i >= n) return;
    const double4 pi = pos[i];
    const double ui[3] = {u[3 * i], u[3 * i + 1], u[3 * i + 2]};
    double jvp[3] = {0, 0, 0}, pp[4] = {0, 0, 0, 0};
    for (int j = lane; j < n; j += 32) {
        if (j == i) continue;
        const int a = min(i, j), b = max(i, j);
        const double4 pj = pos[j];
        const double d[3] = {pi.x - pj.x, pi.y - pj.y, pi.z - pj.z};
        const double r_sq = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        const double rn = sqrt(r_sq);
        const double2 la = LJ[a], lb = LJ[b];
        const double sig = la.x + lb.x;
        const double lj_lim = fp.cutoff_lj > 0.0 ? fp.cutoff_lj : (double)1.122462f * sig;
        const bool elec_in = fp.elec && rn <= fp.cutoff_c;
        const bool lj_in = fp.alpha_lj != 0.0 && rn <= lj_lim;
        if (!elec_in && !lj_in) continue;
        const bool conn = fp.conn_live && adj_conn(conn_ptr, conn_list, a, b);
        double Fm = 0, dFm = 0;
        const double du[3] = {ui[0] - u[3 * j], ui[1] - u[3 * j + 1], ui[2] - u[3 * j + 2]};
        const double ud = (ui[0] * d[0] + ui[1] * d[1] + ui[2] * d[2]) / rn;
        if (elec_in && (!conn || fp.bond_c_scale != 0.0)) {
            const double scale = conn ? fp.bond_c_scale : 1.0;
            const double gq = scale * fp.gamma_c / fp.epsilon_c * Q[a] * Q[b];
            const double kap = fp.kappa_c;
            const double ex = exp(-kap * rn);
            Fm += gq * (1 + kap * rn) * ex / r_sq;
            dFm += gq * ex * (-kap * kap / rn - 2 * (1 + kap * rn) / (r_sq * rn));
            pp[3] += ud * gq * kap * kap * ex;   // kappa -> kappa / s
        }
        if (lj_in && (!conn || fp.bond_lj_scale != 0.0)) {
            const double scale = conn ? fp.bond_lj_scale : 1.0;
            const double K = scale * fp.alpha_lj * sqrt(la.y * lb.y) * 6;
            double s6 = sig / rn;
            s6 *= s6;
            s6 *= s6 * s6;
            const double F = K * s6 * (2 * s6 - fp.lj6) / rn;
            Fm += F;
            dFm += K * s6 * (6 * fp.lj6 - 24 * s6) / r_sq - F / rn;
            pp[0] += ud * F;
            pp[1] += ud * K * s6 * (24 * s6 - 6 * fp.lj6) / rn;
        }
        pair_jvp(Fm, dFm, d, rn, du, jvp);
    }
    for (int k = bptr[i] + lane; k < bptr[i + 1]; k += 32) {
        const int t = blist[k];
        const int j = bond_pairs[2 * t] == i ? bond_pairs[2 * t + 1] : bond_pairs[2 * t];
        const double r0 = bond_parms[3 * t], rmax = bond_parms[3 * t + 1], H = bond_parms[3 * t + 2];
        const double4 pj = pos[j];
        const double d[3] = {pi.x - pj.x, pi.y - pj.y, pi.z - pj.z};
        const double r_sq = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        const double rn = sqrt(r_sq);
        const double q = 1 - r_sq / (rmax * rmax);
        const double Ff = H * (r0 - rn) / q;
        const double dFf = (-H * q + H * (r0 - rn) * 2 * rn / (rmax * rmax)) / (q * q);
        const double du[3] = {ui[0] - u[3 * j], ui[1] - u[3 * j + 1], ui[2] - u[3 * j + 2]};
        pair_jvp(Ff, dFf, d, rn, du, jvp);
        pp[2] += (ui[0] * d[0] + ui[1] * d[1] + ui[2] * d[2]) / rn * Ff;
    }
    for (int o = 16; o > 0; o >>= 1) {
        for (int a = 0; a < 3; ++a) jvp[a] += __shfl_xor_sync(0xffffffffu, jvp[a], o);
        for (int k = 0; k < 4; ++k) pp[k] += __shfl_xor_sync(0xffffffffu, pp[k], o);
    }
    if (lane == 0) {
        for (int a = 0; a < 3; ++a) grad[3 * i + a] += c * jvp[a];
        for (int k = 0; k < 4; ++k) ppart[4 * i + k] = c * pp[k];
    }
}

// ---------------------------------------------------------------- dense

// One pass over the stored matrix M (strict upper: D, lower with diagonal:
// B = chol(D)) for u = D lam (with dD the diagonal) and v = B^T lam. A CTA
// covers 64 columns x 256 rows; thread (row group g, column q) walks 64 rows.
// Partial sums: colp[rb][q] = (lower, upper) column sums of row block rb,
// rowp[cb][p] = upper row sums of column block cb; k_mv2_finish adds them
// in a fixed order.
static constexpr int MV2_COLS = 64, MV2_ROWS = 256;

template <typename TM>
__global__ void __launch_bounds__(256) k_mv2(const TM* __restrict__ M, int n, int ld,
                                             const double* __restrict__ lam, double* __restrict__ colp,
                                             double* __restrict__ rowp)
{
    __shared__ double cl[4][MV2_COLS], cu[4][MV2_COLS];
    __shared__ double rs[MV2_ROWS][MV2_COLS / 16 + 1];
    const int q = threadIdx.x & 63, g = threadIdx.x >> 6;
    const int cb = blockIdx.x, rb = blockIdx.y;
    const int col = cb * MV2_COLS + q;
    double sl = 0, su = 0;
    for (int k = 0; k < 64; ++k) {
        const int row = rb * MV2_ROWS + g * 64 + k;
        double rsum = 0;
        if (row < n && col < n) {
            const double m = (double)M[(size_t)row * ld + col];
            const double lr = lam[row];
            if (col <= row) {
                sl += m * lr;
            } else {
                su += m * lr;
                rsum = m * lam[col];
            }
        }
        // row sum of the upper part over this CTA's 64 columns: 16 lanes per
        // partial, then 4 partials in a fixed order
        for (int o = 8; o > 0; o >>= 1) rsum += __shfl_xor_sync(0xffffffffu, rsum, o, 16);
        if ((q & 15) == 0) rs[g * 64 + k][q >> 4] = rsum;
    }
    cl[g][q] = sl;
    cu[g][q] = su;
    __syncthreads();
    if (g == 0 && col < n) {
        colp[((size_t)rb * n + col) * 2] = cl[0][q] + cl[1][q] + cl[2][q] + cl[3][q];
        colp[((size_t)rb * n + col) * 2 + 1] = cu[0][q] + cu[1][q] + cu[2][q] + cu[3][q];
    }
    for (int r = threadIdx.x; r < MV2_ROWS; r += blockDim.x) {
        const int row = rb * MV2_ROWS + r;
        if (row < n) rowp[(size_t)cb * n + row] = rs[r][0] + rs[r][1] + rs[r][2] + rs[r][3];
    }
}

__global__ void k_mv2_finish(int n, int nrb, int ncb, const double* __restrict__ colp,
                             const double* __restrict__ rowp, const double* __restrict__ dD,
                             const double* __restrict__ lam, double* __restrict__ u, double* __restrict__ v)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    double sl = 0, su = 0, sr = 0;
    for (int rb = 0; rb < nrb; ++rb) {
        sl += colp[((size_t)rb * n + a) * 2];
        su += colp[((size_t)rb * n + a) * 2 + 1];
    }
    for (int cb = 0; cb < ncb; ++cb) sr += rowp[(size_t)cb * n + a];
    u[a] = dD[a] * lam[a] + su + sr;
    v[a] = sl;
}

// R = Phi(v X^T): lower triangle, half the diagonal
template <typename T>
__global__ void k_phi(int n, const double* __restrict__ v, const double* __restrict__ X, T* __restrict__ R)
{
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)n * n) return;
    const int a = (int)(idx / n), b = (int)(idx % n);
    R[idx] = (T)(a > b ? v[a] * X[b] : (a == b ? 0.5 * v[a] * X[a] : 0.0));
}

// out = in^T (n x n, row-major), or out = in + in^T when sym
template <typename T>
__global__ void k_transpose(int n, const T* __restrict__ in, T* __restrict__ out, int sym)
{
    __shared__ T t[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += 8) {
        const int r = by + k, c = bx + threadIdx.x;
        if (r < n && c < n) t[k][threadIdx.x] = in[(size_t)r * n + c];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += 8) {
        const int r = bx + k, c = by + threadIdx.x;
        if (r < n && c < n) {
            const T tv = t[threadIdx.x][k];
            out[(size_t)r * n + c] = sym ? in[(size_t)r * n + c] + tv : tv;
        }
    }
}

// inverses of the 64x64 diagonal blocks of the lower-triangular B (ld):
// Winv[k] row-major 64x64, column c by forward substitution (thread c),
// accumulated in FP64 over the column's entries as stored (T)
template <typename TM, typename T>
__global__ void k_trinv64(const TM* __restrict__ B, int ld, T* __restrict__ Winv)
{
    __shared__ double Bs[64][65];
    const int k = blockIdx.x, c = threadIdx.x;
    const size_t o = (size_t)k * 64;
    for (int r = 0; r < 64; ++r) Bs[r][c] = c <= r ? (double)B[(o + r) * ld + o + c] : 0.0;
    __syncthreads();
    T* W = Winv + (size_t)k * 64 * 64;
    for (int i = 0; i < 64; ++i) {
        double w;
        if (i < c) {
            w = 0.0;
        } else {
            double s = i == c ? 1.0 : 0.0;
            for (int m = c; m < i; ++m) s -= Bs[i][m] * (double)W[m * 64 + c];
            w = s / Bs[i][i];
        }
        W[i * 64 + c] = (T)w;
    }
}

// C[M x N] = alpha A^T B + beta C in T (FP64 or FP32) arithmetic; A is
// K x M (lda, elements TA), B K x N (ldb), C M x N (ldc), all row-major; M,
// N multiples of 64, K of 16. 64x64 tiles, 256 threads with 4x4 outputs
// each (rows ty + 16 i, columns tx + 16 j).
template <typename T, typename TA>
__global__ void __launch_bounds__(256) k_gemm_tn(int M, int N, int K, T alpha, const TA* __restrict__ A, int lda,
                                                 const T* __restrict__ B, int ldb, T beta, T* __restrict__ C, int ldc)
{
    __shared__ T As[16][64 + 2], Bs[16][64 + 2];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    T acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += 16) {
        for (int e = threadIdx.x; e < 16 * 64; e += 256) {
            const int kk = e >> 6, mm = e & 63;
            As[kk][mm] = (T)A[(size_t)(k0 + kk) * lda + m0 + mm];
            Bs[kk][mm] = B[(size_t)(k0 + kk) * ldb + n0 + mm];
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            T a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                a[i] = As[kk][ty + 16 * i];
                b[i] = Bs[kk][tx + 16 * i];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * b[j];
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            T* cp = C + (size_t)(m0 + ty + 16 * i) * ldc + n0 + tx + 16 * j;
            *cp = beta == (T)0 ? alpha * acc[i][j] : alpha * acc[i][j] + beta * *cp;
        }
}

template <typename T, typename TA>
static void gemm_tn(cudaStream_t st, int M, int N, int K, T alpha, const TA* A, int lda, const T* B, int ldb, T beta,
                    T* C, int ldc)
{
    dim3 grid(N / 64, M / 64);
    k_gemm_tn<T, TA><<<grid, 256, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
}

// Y = B^-T R for the lower-triangular B (ld ldb, n x n, n a multiple of 64),
// right-looking from the last 64-row block; R (n x n) is overwritten.
// Winv: inverses of B's diagonal blocks (k_trinv64).
template <typename T, typename TM>
static int trsm_lt(bdb_system* s, int n, const TM* B, int ldb, const T* Winv, T* R, T* Y)
{
    const int nb = n / 64;
    for (int k = nb - 1; k >= 0; --k) {
        T* Yk = Y + (size_t)k * 64 * n;
        // Y_k = Winv_k^T R_k
        gemm_tn<T, T>(s->stream, 64, n, 64, (T)1, Winv + (size_t)k * 64 * 64, 64, R + (size_t)k * 64 * n, n, (T)0, Yk, n);
        // R_0..k-1 -= B[k, 0:k]^T Y_k
        if (k > 0)
            gemm_tn<T, TM>(s->stream, 64 * k, n, 64, (T)-1, B + (size_t)k * 64 * ldb, ldb, Yk, n, (T)1, R, n);
        s->launches += 1 + (k > 0);
    }
    BDB_CUDA(cudaGetLastError());
    return BDB_OK;
}

// ---------------------------------------------------------------- driver

template <typename T>
struct Scratch {
    T* p = nullptr;
    ~Scratch()
    {
        if (p) cudaFree(p);
    }
    int alloc(size_t n)
    {
        return cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * std::max<size_t>(n, 1)) == cudaSuccess ? 0 : 1;
    }
};

// u = D lam and v = B^T lam from the stored matrix M (D upper, B lower),
// then S = Z + Z^T with Z^T = Dbar = B^-T Phi(v X^T) B^-1 into R (T, np x
// np); Y is scratch of the same size
template <typename T, typename TM>
static int adjoint_linalg(bdb_system* s, const TM* M, int np, int n3, int nrb, int ncb, const double* lam,
                          double* colp, double* rowp, double* u, double* v, const double* Xp, T* R, T* Y, T* Winv)
{
    cudaStream_t st = s->stream;
    k_mv2<TM><<<dim3(ncb, nrb), 256, 0, st>>>(M, n3, np, lam, colp, rowp);
    k_mv2_finish<<<(n3 + 255) / 256, 256, 0, st>>>(n3, nrb, ncb, colp, rowp, s->dD.p, lam, u, v);
    k_phi<T><<<(unsigned)(((size_t)np * np + 255) / 256), 256, 0, st>>>(np, v, Xp, R);
    k_trinv64<TM, T><<<np / 64, 64, 0, st>>>(M, np, Winv);
    int rc = trsm_lt<T, TM>(s, np, M, np, Winv, R, Y);
    if (rc) return rc;
    k_transpose<T><<<dim3(np / 32, np / 32), dim3(32, 8), 0, st>>>(np, Y, R, 0);
    if ((rc = trsm_lt<T, TM>(s, np, M, np, Winv, R, Y))) return rc;
    k_transpose<T><<<dim3(np / 32, np / 32), dim3(32, 8), 0, st>>>(np, Y, R, 1);
    s->launches += 6;
    return BDB_OK;
}

static int set_counter(bdb_system* s, unsigned long long v)
{
    const unsigned long long c[2] = {v, 0ull};
    BDB_CUDA(cudaMemcpyAsync(s->ctr.p, c, sizeof(c), cudaMemcpyHostToDevice, s->stream));
    return BDB_OK;
}

static int set_positions(bdb_system* s, const double4* src)
{
    BDB_CUDA(cudaMemcpyAsync(s->pos.p, src, sizeof(double4) * s->n, cudaMemcpyDeviceToDevice, s->stream));
    BDB_CUDA(cudaMemsetAsync(s->cells_built.p, 0, sizeof(int) * s->segs.size(), s->stream));
    s->have_forces = false;
    s->factor_valid = false;
    return BDB_OK;
}

}  // namespace bdb

using namespace bdb;

extern "C" int bdb_adjoint(bdb_system* s, int K, int checkpoint, int npairs, const int* pairs,
                           const double* targets, double* loss, double* grad_coord, double* grad_params)
{
    if (!s || K < 1 || checkpoint < 1 || npairs < 1 || !pairs || !targets || !loss || !grad_coord || !grad_params)
        return fail(BDB_ERR_ARG, "bad arguments");
    if (s->p.hydro != BDB_HYDRO_CHOLESKY || s->p.refresh != 1 || s->p.noise != BDB_NOISE_PHILOX || s->p.bc != 0 ||
        s->segs.size() != 1)
        return fail(BDB_ERR_UNSUPPORTED,
                    "the adjoint needs one free-space system, hydro cholesky, refresh 1 and device noise");
    const bool mixed = s->p.precision == BDB_PREC_MIXED;
    if (s->p.e_ext && s->p.e_type != 0)
        return fail(BDB_ERR_UNSUPPORTED, "the adjoint takes a constant (DC) external field only");
    if (s->n_angle || s->n_angle_cos || s->n_dihe || s->n_dihe_angle)
        return fail(BDB_ERR_UNSUPPORTED, "the adjoint covers bonds, LJ and Debye-Hueckel terms only");
    for (int p = 0; p < 2 * npairs; ++p)
        if (pairs[p] < 0 || pairs[p] >= s->n) return fail(BDB_ERR_ARG, "loss pair references a missing bead");
    const int n = s->n, n3 = s->n3, np = s->npad;
    const double c = s->p.dt / (BDB_KB * s->p.T);
    cudaStream_t st = s->stream;
    int rc;
    if ((rc = ensure_matrix(s))) return rc;
    // bead -> bond list (host CSR, fixed order)
    std::vector<int> bp_h(2 * std::max(1, s->n_bond)), bptr(n + 1, 0), blist;
    if (s->n_bond)
        BDB_CUDA(d2h(s, bp_h.data(), s->bond_pairs.p, sizeof(int) * 2 * s->n_bond));
    for (int t = 0; t < s->n_bond; ++t) {
        bptr[bp_h[2 * t] + 1]++;
        bptr[bp_h[2 * t + 1] + 1]++;
    }
    for (int i = 0; i < n; ++i) bptr[i + 1] += bptr[i];
    blist.resize(std::max(1, bptr[n]));
    {
        std::vector<int> fill(bptr.begin(), bptr.end() - 1);
        for (int t = 0; t < s->n_bond; ++t) {
            blist[fill[bp_h[2 * t]]++] = t;
            blist[fill[bp_h[2 * t + 1]]++] = t;
        }
    }
    const int nck = (K + checkpoint - 1) / checkpoint;
    const int nrb = (n3 + MV2_ROWS - 1) / MV2_ROWS, ncb = (n3 + MV2_COLS - 1) / MV2_COLS;
    Scratch<double> R, Y, Winv, lam, lam2, u, v, Xp, colp, rowp, ppart;
    Scratch<double4> ckpt, seg, xK;
    Scratch<int> d_bptr, d_blist;
    if (R.alloc((size_t)np * np) || Y.alloc((size_t)np * np) || Winv.alloc((size_t)np * 64) || lam.alloc(np) ||
        lam2.alloc(np) || u.alloc(np) || v.alloc(np) || Xp.alloc(np) || colp.alloc((size_t)nrb * n3 * 2) ||
        rowp.alloc((size_t)ncb * n3) || ppart.alloc(4 * (size_t)n) || ckpt.alloc((size_t)nck * n) ||
        seg.alloc((size_t)checkpoint * n) || xK.alloc(n) || d_bptr.alloc(n + 1) || d_blist.alloc(blist.size()))
        return fail(BDB_ERR_NOMEM, "adjoint scratch allocation failed");
    BDB_CUDA(h2d(s, d_bptr.p, bptr.data(), sizeof(int) * (n + 1)));
    BDB_CUDA(h2d(s, d_blist.p, blist.data(), sizeof(int) * blist.size()));
    BDB_CUDA(cudaMemsetAsync(u.p, 0, sizeof(double) * np, st));
    BDB_CUDA(cudaMemsetAsync(v.p, 0, sizeof(double) * np, st));
    BDB_CUDA(cudaMemsetAsync(Xp.p, 0, sizeof(double) * np, st));
    BDB_CUDA(cudaMemsetAsync(lam.p, 0, sizeof(double) * np, st));
    BDB_CUDA(cudaMemsetAsync(lam2.p, 0, sizeof(double) * np, st));
    unsigned long long base = 0;
    BDB_CUDA(cudaMemcpyAsync(&base, s->ctr.p, sizeof(base), cudaMemcpyDeviceToHost, st));
    BDB_CUDA(cudaStreamSynchronize(st));
    BDB_CUDA(cudaMemsetAsync(s->status.p, 0, sizeof(unsigned), st));

    // forward, keeping the positions at every checkpoint
    for (int k = 0; k < K; ++k) {
        if (k % checkpoint == 0)
            BDB_CUDA(cudaMemcpyAsync(ckpt.p + (size_t)(k / checkpoint) * n, s->pos.p, sizeof(double4) * n,
                                     cudaMemcpyDeviceToDevice, st));
        if ((rc = engine_step(s))) return rc;
    }
    BDB_CUDA(cudaMemcpyAsync(xK.p, s->pos.p, sizeof(double4) * n, cudaMemcpyDeviceToDevice, st));

    // loss = mean over pairs of (|x_b - x_a| - target)^2 and its gradient
    std::vector<double4> xh(n);
    BDB_CUDA(cudaMemcpyAsync(xh.data(), s->pos.p, sizeof(double4) * n, cudaMemcpyDeviceToHost, st));
    BDB_CUDA(cudaStreamSynchronize(st));
    std::vector<double> lh(np, 0.0);
    double L = 0;
    for (int p = 0; p < npairs; ++p) {
        const int a = pairs[2 * p], b = pairs[2 * p + 1];
        const double d[3] = {xh[b].x - xh[a].x, xh[b].y - xh[a].y, xh[b].z - xh[a].z};
        const double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        const double dev = r - targets[p];
        L += dev * dev / npairs;
        for (int k = 0; k < 3; ++k) {
            const double g = 2 * dev / npairs * d[k] / r;
            lh[3 * b + k] += g;
            lh[3 * a + k] -= g;
        }
    }
    BDB_CUDA(cudaMemcpyAsync(lam.p, lh.data(), sizeof(double) * n3, cudaMemcpyHostToDevice, st));
    std::vector<double> gp(4, 0.0);
    AdjForce fp;
    fp.elec = s->p.elec;
    fp.epsilon_c = s->p.epsilon_c;
    fp.kappa_c = s->p.kappa_c;
    fp.gamma_c = s->p.gamma_c;
    fp.cutoff_c = s->p.cutoff_c;
    fp.alpha_lj = s->p.alpha_lj;
    fp.cutoff_lj = s->p.cutoff_lj;
    fp.lj6 = s->p.lj_6_term;
    fp.bond_lj_scale = s->p.bond_lj_scale;
    fp.bond_c_scale = s->p.bond_c_scale;
    fp.conn_live = s->conn_live;
    std::vector<double> pph(4 * (size_t)n);
    const int warps_blocks = (n * 32 + 255) / 256;

    // backward, one checkpoint segment at a time (recomputed forward)
    for (int sg = nck - 1; sg >= 0; --sg) {
        const int k0 = sg * checkpoint, k1 = std::min(K, k0 + checkpoint);
        if ((rc = set_positions(s, ckpt.p + (size_t)sg * n)) || (rc = set_counter(s, base + k0))) return rc;
        for (int k = k0; k < k1; ++k) {
            BDB_CUDA(cudaMemcpyAsync(seg.p + (size_t)(k - k0) * n, s->pos.p, sizeof(double4) * n,
                                     cudaMemcpyDeviceToDevice, st));
            if ((rc = engine_step(s))) return rc;
        }
        for (int k = k1 - 1; k >= k0; --k) {
            // the forward quantities of step k: F(x_k), D(x_k), B(x_k), X_k
            if ((rc = set_positions(s, seg.p + (size_t)(k - k0) * n)) || (rc = set_counter(s, base + k))) return rc;
            if ((rc = forces_run(s, false, false)) || (rc = tensor_build(s)) || (rc = factor_run(s)) ||
                (rc = noise_fill(s, nullptr)))
                return rc;
            BDB_CUDA(cudaMemcpyAsync(Xp.p, s->X.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, st));
            // u = D lam, v = B^T lam; S = Z + Z^T with Z^T = Dbar = B^-T Phi(v X^T) B^-1
            if (mixed)
                rc = adjoint_linalg<float, float>(s, s->M32.p, np, n3, nrb, ncb, lam.p, colp.p, rowp.p, u.p, v.p, Xp.p,
                                                  reinterpret_cast<float*>(R.p), reinterpret_cast<float*>(Y.p),
                                                  reinterpret_cast<float*>(Winv.p));
            else
                rc = adjoint_linalg<double, double>(s, s->M64.p, np, n3, nrb, ncb, lam.p, colp.p, rowp.p, u.p, v.p,
                                                    Xp.p, R.p, Y.p, Winv.p);
            if (rc) return rc;
            // lam_k = lam + c (dD/dx : F)^T lam + (d(BX)/dx)^T lam + c (dF/dx) u
            BDB_CUDA(cudaMemcpyAsync(lam2.p, lam.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, st));
            if (mixed)
                k_tile_grad<float><<<warps_blocks, 256, 0, st>>>(n, s->pos.p, s->preDii, s->preDij, c, lam.p, s->F.p,
                                                                reinterpret_cast<const float*>(R.p), np, lam2.p);
            else
                k_tile_grad<double><<<warps_blocks, 256, 0, st>>>(n, s->pos.p, s->preDii, s->preDij, c, lam.p, s->F.p,
                                                                 R.p, np, lam2.p);
            k_force_jvp<<<warps_blocks, 256, 0, st>>>(n, fp, s->pos.p, s->Q.p, s->LJ.p, s->conn_ptr.p,
                                                     s->conn_list.p, d_bptr.p, d_blist.p, s->bond_pairs.p,
                                                     s->bond_parms.p, u.p, c, lam2.p, ppart.p);
            BDB_CUDA(cudaGetLastError());
            s->launches += 3;
            BDB_CUDA(cudaMemcpyAsync(pph.data(), ppart.p, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, st));
            BDB_CUDA(cudaStreamSynchronize(st));
            for (int i = 0; i < n; ++i)
                for (int q = 0; q < 4; ++q) gp[q] += pph[4 * (size_t)i + q];
            std::swap(lam.p, lam2.p);
        }
    }
    BDB_CUDA(cudaMemcpyAsync(grad_coord, lam.p, sizeof(double) * n3, cudaMemcpyDeviceToHost, st));
    if ((rc = set_positions(s, xK.p)) || (rc = set_counter(s, base + K))) return rc;
    unsigned stw = 0;
    BDB_CUDA(cudaMemcpyAsync(&stw, s->status.p, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    BDB_CUDA(cudaStreamSynchronize(st));
    if (stw & ST_NOT_SPD) return fail(BDB_ERR_NOT_SPD, "Cholesky decomposition error: non-positive pivot");
    if (stw & ST_BOND) return fail(BDB_ERR_BOND, "Overstretched bond (bond.c:73-78)");
    for (int q = 0; q < 4; ++q) grad_params[q] = gp[q];
    *loss = L;
    return BDB_OK;
}
