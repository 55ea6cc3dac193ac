// One pass over the stored matrix M (upper triangle: D, lower triangle
// including the diagonal: its Cholesky factor L) computes both per-step
// products of the Cholesky path:
//   Rf = D F   (dsymv "U", diff_alg/diff_equation.c:152-159)
//   Rs = L X   (my_dtrmv, myblas.c:94-118)
// HBM-bound: every element of M is read once per step.
//
// Work item = one warp on (strip of 32 rows) x (column segment). A lane
// owns 4 consecutive columns of every 128-column tile (one 16-byte load of
// FP32 or two of FP64 per row). For each tile the 32 per-row lane partials
// go through a per-warp shared-memory transpose, after which lane q adds
// row q's sum. The transposed part of D F (left of the diagonal)
// accumulates per column over the strip's 32 rows and is written as one
// partial per (strip, column); k_mv_finish adds all partials in a fixed
// order and applies the position update, so results are deterministic.
// Products are accumulated in FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "bdb_common.cuh"

namespace bdb {

static constexpr int STRIP = 32;
static constexpr int WARPS = 4;

__device__ __forceinline__ void load4(const float* p, double* o)
{
    const float4 v = __ldcs(reinterpret_cast<const float4*>(p));
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
    o[3] = v.w;
}

__device__ __forceinline__ void load4(const double* p, double* o)
{
    const double2 a = __ldcs(reinterpret_cast<const double2*>(p));
    const double2 b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
    o[0] = a.x;
    o[1] = a.y;
    o[2] = b.x;
    o[3] = b.y;
}

// rowp: [nseg][n3][2] row partials (Rs, Rf right part); colp: [nstrip][n3]
template <typename T>
__global__ void __launch_bounds__(32 * WARPS)
k_strip_mv(const T* __restrict__ M, int n3, int npad, int nseg, int seg_cols,
           const double* __restrict__ F, const double* __restrict__ X, double* __restrict__ rowp,
           double* __restrict__ colp)
{
    __shared__ double sF[WARPS][STRIP];
    __shared__ double red[WARPS][32][STRIP + 1];   // [lane][row] partials of one tile
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int item = blockIdx.x * WARPS + warp;
    const int nstrip = (n3 + STRIP - 1) / STRIP;
    if (item >= nstrip * nseg) return;
    const int strip = item / nseg, seg = item % nseg;
    const int r0 = strip * STRIP;
    const int nrow = min(STRIP, n3 - r0);
    const int c_beg = seg * seg_cols, c_end = min(n3, c_beg + seg_cols);
    sF[warp][lane] = lane < nrow ? F[r0 + lane] : 0.0;
    __syncwarp();
    double (*rd)[STRIP + 1] = red[warp];
    double rs_acc = 0, rf_acc = 0;
    for (int c0 = c_beg; c0 < c_end; c0 += 128) {
        const int c = c0 + 4 * lane;
        double x[4], f[4], pc[4] = {0, 0, 0, 0};
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const bool ok = c + v < c_end;
            x[v] = ok ? X[c + v] : 0.0;
            f[v] = ok ? F[c + v] : 0.0;
        }
        const bool lower = c0 + 127 < r0;
        const bool upper = c0 > r0 + STRIP - 1;
        // warp-uniform choice: every lane of an interior tile has 4 columns
        if ((lower || upper) && nrow == STRIP && c0 + 127 < c_end) {
            // interior tile: 8 rows of loads in flight at a time
            const double* w = lower ? x : f;
            double (*dst)[STRIP + 1] = rd;
#pragma unroll 8
            for (int q = 0; q < STRIP; ++q) {
                double m[4];
                load4(M + (size_t)(r0 + q) * npad + c, m);
                dst[lane][q] = m[0] * w[0] + m[1] * w[1] + m[2] * w[2] + m[3] * w[3];
                if (upper) {
                    const double fq = sF[warp][q];
                    pc[0] += m[0] * fq;
                    pc[1] += m[1] * fq;
                    pc[2] += m[2] * fq;
                    pc[3] += m[3] * fq;
                }
            }
            __syncwarp();
            double sum = 0;
#pragma unroll 8
            for (int l = 0; l < 32; ++l) sum += dst[l][lane];
            if (lower) rs_acc += sum; else rf_acc += sum;
            __syncwarp();
        } else {
            // edge tile or tile crossing the diagonal: per element, the L
            // part (columns <= row) first, then the D part
            for (int part = 0; part < 2; ++part) {
                for (int q = 0; q < STRIP; ++q) {
                    const int r = r0 + q;
                    double m[4] = {0, 0, 0, 0};
                    if (q < nrow)
                        for (int v = 0; v < 4; ++v)
                            if (c + v < c_end) m[v] = (double)M[(size_t)r * npad + c + v];
                    double a = 0;
                    const double fq = sF[warp][q];
#pragma unroll
                    for (int v = 0; v < 4; ++v) {
                        if (part == 0 && c + v <= r) a += m[v] * x[v];
                        if (part == 1 && c + v > r) {
                            a += m[v] * f[v];
                            pc[v] += m[v] * fq;
                        }
                    }
                    rd[lane][q] = a;
                }
                __syncwarp();
                double sa = 0;
                for (int l = 0; l < 32; ++l) sa += rd[l][lane];
                if (part == 0) rs_acc += sa; else rf_acc += sa;
                __syncwarp();
            }
        }
        if (!lower) {
#pragma unroll
            for (int v = 0; v < 4; ++v)
                if (c + v < c_end && c + v > r0) colp[(size_t)strip * n3 + c + v] = pc[v];
        }
    }
    if (lane < nrow) {
        rowp[((size_t)seg * n3 + r0 + lane) * 2] = rs_acc;
        rowp[((size_t)seg * n3 + r0 + lane) * 2 + 1] = rf_acc;
    }
}

// Rs = sum of row partials; Rf = pre * (row partials + dD F + column partials
// of the strips above). A block covers 32 rows; its 8 thread rows take every
// 8th strip (4 independent sums each) and are combined in a fixed order.
static constexpr int FIN_ROWS = 32, FIN_GROUPS = 8;

__global__ void __launch_bounds__(FIN_ROWS * FIN_GROUPS)
k_mv_finish(int n3, int nseg, const double* __restrict__ rowp, const double* __restrict__ colp,
            const double* __restrict__ dD, const double* __restrict__ F, double pre, double* __restrict__ Rf,
            double* __restrict__ Rs, int want_rs)
{
    __shared__ double part[FIN_GROUPS][FIN_ROWS + 1];
    const int tx = threadIdx.x % FIN_ROWS, ty = threadIdx.x / FIN_ROWS;
    const int r = blockIdx.x * FIN_ROWS + tx;
    double c[4] = {0, 0, 0, 0};
    if (r < n3) {
        const int nst = (r + STRIP - 1) / STRIP;   // strips st with st * STRIP < r
        int st = ty, q = 0;
        for (; st < nst; st += FIN_GROUPS, q = (q + 1) & 3) c[q] += colp[(size_t)st * n3 + r];
    }
    part[ty][tx] = (c[0] + c[1]) + (c[2] + c[3]);
    __syncthreads();
    if (ty == 0 && r < n3) {
        double s = 0, f = 0;
        for (int g = 0; g < nseg; ++g) {
            s += rowp[((size_t)g * n3 + r) * 2];
            f += rowp[((size_t)g * n3 + r) * 2 + 1];
        }
        f += dD[r] * F[r];
        for (int g = 0; g < FIN_GROUPS; ++g) f += part[g][tx];
        Rf[r] = f * pre;
        if (want_rs) Rs[r] = s;
    }
}

static void mv_finish(cudaStream_t st, int n3, int nseg, const double* rowp, const double* colp, const double* dD,
                      const double* F, double pre, double* Rf, double* Rs, int want_rs)
{
    k_mv_finish<<<(n3 + FIN_ROWS - 1) / FIN_ROWS, FIN_ROWS * FIN_GROUPS, 0, st>>>(n3, nseg, rowp, colp, dD, F, pre, Rf,
                                                                                Rs, want_rs);
}

// column segmentation of the strip products: enough warps for the machine
// (warps_per_sm per SM), columns in multiples of 128
static void mv_split(int n3, int warps_per_sm, int sms, int* nseg_out, int* seg_cols_out)
{
    const int nstrip = (n3 + STRIP - 1) / STRIP;
    int nseg = std::max(1, (sms * warps_per_sm + nstrip - 1) / nstrip);
    const int seg_cols = ((n3 + nseg - 1) / nseg + 127) / 128 * 128;
    nseg = (n3 + seg_cols - 1) / seg_cols;
    *nseg_out = nseg;
    *seg_cols_out = seg_cols;
}

static void mv_launch(bdb_system* s, int nseg, int seg_cols, const double* X, double* rowp, double* colp)
{
    const int n3 = s->n3;
    const int nstrip = (n3 + STRIP - 1) / STRIP;
    const int blocks = (nstrip * nseg + WARPS - 1) / WARPS;
    if (s->p.precision == BDB_PREC_FP64)
        k_strip_mv<double><<<blocks, 32 * WARPS, 0, s->stream>>>(s->M64.p, n3, s->npad, nseg, seg_cols, s->F.p, X,
                                                                 rowp, colp);
    else
        k_strip_mv<float><<<blocks, 32 * WARPS, 0, s->stream>>>(s->M32.p, n3, s->npad, nseg, seg_cols, s->F.p, X,
                                                                rowp, colp);
}

// Autotuning of the segmentation: 8, 16 or 32 warps per SM, each timed
// twice after a warm-up; runs at the first product of a system with
// autotuning on (before any graph capture).
static int mv_tune(bdb_system* s, const double* X, double* part)
{
    const int cands[3] = {8, 16, 32};
    float best_ms = 1e30f;
    int best = s->mv_warps;
    cudaEvent_t e0, e1;
    BDB_CUDA(cudaEventCreate(&e0));
    BDB_CUDA(cudaEventCreate(&e1));
    for (int w : cands) {
        int nseg, seg_cols;
        mv_split(s->n3, w, s->sm_count, &nseg, &seg_cols);
        double* rowp = part;
        double* colp = part + (size_t)nseg * s->n3 * 2;
        mv_launch(s, nseg, seg_cols, X, rowp, colp);
        BDB_CUDA(cudaEventRecord(e0, s->stream));
        mv_launch(s, nseg, seg_cols, X, rowp, colp);
        mv_launch(s, nseg, seg_cols, X, rowp, colp);
        BDB_CUDA(cudaEventRecord(e1, s->stream));
        BDB_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        BDB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        s->launches += 3;
        if (ms < best_ms) {
            best_ms = ms;
            best = w;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    s->mv_warps = best;
    s->mv_tuned = true;
    return BDB_OK;
}

int stored_matvec(bdb_system* s, bool want_rs)
{
    const int n3 = s->n3;
    const int nstrip = (n3 + STRIP - 1) / STRIP;
    // room for the largest segmentation any tuning candidate can pick
    int nseg_max, cols_max;
    mv_split(n3, 32, s->sm_count, &nseg_max, &cols_max);
    const size_t need = (size_t)std::max(nseg_max, 1) * n3 * 2 + (size_t)nstrip * n3;
    if (s->part.n < need) {
        if (s->part.alloc(need)) return BDB_ERR_NOMEM;
    }
    const double* X = want_rs ? s->X.p : s->F.p;   // any valid vector when Rs is not wanted
    if (s->autotune && !s->mv_tuned) {
        int rc = mv_tune(s, X, s->part.p);
        if (rc) return rc;
    }
    int nseg, seg_cols;
    mv_split(n3, s->mv_warps, s->sm_count, &nseg, &seg_cols);
    double* rowp = s->part.p;
    double* colp = s->part.p + (size_t)nseg * n3 * 2;
    mv_launch(s, nseg, seg_cols, X, rowp, colp);
    BDB_CUDA(cudaGetLastError());
    s->launches += 2;
    const double pre = s->p.dt / (BDB_KB * s->p.T);
    mv_finish(s->stream, n3, nseg, rowp, colp, s->dD.p, s->F.p, pre, s->Rf.p, s->Rs.p, want_rs);
    BDB_CUDA(cudaGetLastError());
    return BDB_OK;
}

// ---------------------------------------------------------------------------
// No-allocation entry point: the same two products on caller-owned device
// buffers, with the partial sums kept in a fixed-size array in this file's
// device memory instead of a buffer obtained from cudaMalloc.

static constexpr int NOALLOC_MAX_N3 = 3072;              // 1024 beads
static constexpr int NOALLOC_MAX_SEG = 4;
static constexpr size_t NOALLOC_SCRATCH =
    (size_t)NOALLOC_MAX_SEG * NOALLOC_MAX_N3 * 2 + (size_t)(NOALLOC_MAX_N3 / STRIP) * NOALLOC_MAX_N3;

// Scratch for row and column partial sums (2.5 MB of doubles), one copy on
// every device that loads the library, kept until the process exits.
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_SCRATCH];

static constexpr int NOALLOC_MAX_DEVICES = 64;
static double* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {nullptr};

}  // namespace bdb

using bdb::g_noalloc_scratch;

extern "C" int bdb_stored_matvec_noalloc(const float* M, int n3, int ld, const double* dD, const double* F,
                                         const double* X, double pre, double* Rf, double* Rs, void* stream)
{
    using namespace bdb;
    if (!M || !dD || !F || !X || !Rf || !Rs) return fail(BDB_ERR_ARG, "null device pointer");
    if (n3 <= 0 || n3 > NOALLOC_MAX_N3)
        return fail(BDB_ERR_ARG, "bdb_stored_matvec_noalloc: 3N must be in 1.." + std::to_string(NOALLOC_MAX_N3) +
                                     " (its scratch array has a fixed size), got " + std::to_string(n3));
    if (ld < n3 || ld % 4 != 0 || reinterpret_cast<uintptr_t>(M) % 16 != 0)
        return fail(BDB_ERR_ARG, "bdb_stored_matvec_noalloc: ld must be >= 3N and a multiple of 4, M 16-byte aligned");
    int dev = 0;
    BDB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return fail(BDB_ERR_ARG, "device index out of range");
    if (!g_noalloc_ptr[dev]) {
        // set-up, once per device with that device current: the host-side
        // symbol is only a stand-in, the kernels need its device address
        void* p = nullptr;
        BDB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nstrip = (n3 + STRIP - 1) / STRIP;
    int nseg = std::min(NOALLOC_MAX_SEG, std::max(1, (148 * 16 + nstrip - 1) / nstrip));
    const int seg_cols = ((n3 + nseg - 1) / nseg + 127) / 128 * 128;
    nseg = (n3 + seg_cols - 1) / seg_cols;
    // every partial that k_mv_finish reads is written first by k_strip_mv,
    // so nothing in the scratch has to start at zero
    double* rowp = g_noalloc_ptr[dev];
    double* colp = rowp + (size_t)nseg * n3 * 2;
    const int blocks = (nstrip * nseg + WARPS - 1) / WARPS;
    k_strip_mv<float><<<blocks, 32 * WARPS, 0, st>>>(M, n3, ld, nseg, seg_cols, F, X, rowp, colp);
    BDB_CUDA(cudaGetLastError());
    mv_finish(st, n3, nseg, rowp, colp, dD, F, pre, Rf, Rs, 1);
    BDB_CUDA(cudaGetLastError());
    return BDB_OK;
}
