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

#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "bdb_common.cuh"
#include "philox.cuh"
#include "sm100.cuh"

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

// ---------------------------------------------------------------------------
// FP32 matrix (mixed precision): TMA-fed persistent kernel.
//
// The matrix is cut into tiles of 64 rows x 128 columns (32 KB of FP32),
// numbered strip-major (t = strip * ntc + column tile); CTA k of G takes the
// contiguous range [k T / G, (k+1) T / G) of the T tiles, so every CTA moves
// the same number of bytes; a range touches at most `slots` strips.
//   warp 8      TMA producer: per tile one 2-D box of the matrix (no
//               swizzle: a tile row is 512 contiguous bytes) and the tile's
//               128 entries of X and F (1-D boxes) into a 5-stage ring;
//   warps 0-7   consumers: warp w owns rows 8w..8w+7 of the strip, a lane 4
//               columns of each tile (conflict-free 16-byte shared loads).
//               Row sums stay in registers for the whole strip (16 FP64 per
//               lane) and are reduced across lanes once per strip. For tiles
//               with a D part, each warp's column partials (over its 8 rows)
//               go to one of 4 shared buffers;
//   warp 9      reducer: adds the 8 warps' column partials of a tile in a
//               fixed order and writes one value per (strip, column).
// (Sixteen consumer warps of 4 rows measured slower: 139 vs 130 us per
// product at 3N = 12288.)
// Every hand-over is an mbarrier, so the consumer warps never wait for one
// another and run up to the ring depth ahead of the reducer. Edge boxes are
// zero-filled by the TMA unit (the maps are 3N x 3N and 3N), so no element
// outside the matrix contributes.
static constexpr int MT_ROWS = 64, MT_COLS = 128, MT_STAGES = 5, MT_CW = 8, MT_NB = 4;
static constexpr int MT_RW = MT_ROWS / MT_CW;   // rows per consumer warp
static constexpr int MT_THREADS = 32 * (MT_CW + 2);
static constexpr int MT_BOX_BYTES = MT_ROWS * MT_COLS * 4;
static constexpr int MT_VEC_BYTES = MT_COLS * 8;                         // one FP64 vector box
static constexpr int MT_STAGE_BYTES = MT_BOX_BYTES + 2 * MT_VEC_BYTES;   // matrix box, X box, F box
static constexpr int MT_CPART_DOUBLES = MT_CW * MT_COLS;                 // one column-partial buffer
static constexpr int MT_SMEM = MT_STAGES * MT_STAGE_BYTES + MT_NB * MT_CPART_DOUBLES * 8 + 128;

struct MtBars {
    uint64_t full[MT_STAGES], empty[MT_STAGES], cfull[MT_NB], cempty[MT_NB];
};

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// tile kinds: every column <= every row (L only), every column > every row
// (D only), or crossing the diagonal
__device__ __forceinline__ bool mt_lower(int r0, int c0) { return c0 + MT_COLS - 1 <= r0; }
__device__ __forceinline__ bool mt_upper(int r0, int c0) { return c0 >= r0 + MT_ROWS; }

// rowp: [G][slots][64 rows][2] (Rs, Rf right part); colp: [nstrip][n3]
__global__ void __launch_bounds__(MT_THREADS, 1)
k_strip_mv_tma(const __grid_constant__ CUtensorMap map, const __grid_constant__ CUtensorMap map_x,
               const __grid_constant__ CUtensorMap map_f, int n3, int ntc, long long T, int slots,
               const double* __restrict__ F, double* __restrict__ rowp, double* __restrict__ colp,
               unsigned* __restrict__ status, uint32_t wlim, int gen_x, uint64_t seed,
               const unsigned long long* __restrict__ ctr, double xscale)
{
    {
        uint32_t dyn;
        asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
        if (blockDim.x != MT_THREADS || dyn < (uint32_t)MT_SMEM) {
            if (threadIdx.x == 0) atomicOr(status, ST_LAUNCH);
            return;
        }
    }
    extern __shared__ unsigned char mt_raw[];
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(mt_raw) + 127) & ~uintptr_t(127));
    double* cpart = reinterpret_cast<double*>(sm + MT_STAGES * MT_STAGE_BYTES);   // [MT_NB][MT_CW][MT_COLS]
    __shared__ MtBars bars;
    __shared__ volatile int abort_flag;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t sbase = smem_u32(sm);
    const int G = gridDim.x, k = blockIdx.x;
    const long long t_beg = (long long)k * T / G, t_end = (long long)(k + 1) * T / G;
    const int s_first = (int)(t_beg / ntc);
    if (tid == 0) {
        abort_flag = 0;
        for (int st = 0; st < MT_STAGES; ++st) {
            mbar_init(smem_u32(&bars.full[st]), 1);
            mbar_init(smem_u32(&bars.empty[st]), MT_CW);
        }
        for (int b = 0; b < MT_NB; ++b) {
            mbar_init(smem_u32(&bars.cfull[b]), MT_CW);
            mbar_init(smem_u32(&bars.cempty[b]), 1);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // gen_x (the fused Cholesky step): the noise of this step is normally
    // drawn ahead into X by the previous step's finisher, tagged ctr[2] =
    // stream + 1. Without that tag (the first fused step, or after another
    // writer of X or of the stream index) the producer warp draws it itself.
    bool draw = false;
    uint64_t stream = 0;
    if (gen_x) {
        stream = *reinterpret_cast<const volatile unsigned long long*>(ctr);
        draw = *reinterpret_cast<const volatile unsigned long long*>(ctr + 2) != stream + 1;
    }
    if (warp == MT_CW && draw) {
        // the whole warp computes each tile's 128 entries of X -- the
        // Philox Gaussians k_noise would write, scaled the same way -- into
        // the stage (tiles with an L part only), then lane 0 loads the
        // matrix box and F. Waits and stops are decided by lane 0 and
        // shared, so the lanes never part.
        long long i = 0;
        for (long long t = t_beg; t < t_end; ++t, ++i) {
            if (__shfl_sync(0xffffffffu, lane == 0 ? (int)abort_flag : 0, 0)) break;
            const int st = (int)(i % MT_STAGES);
            bool ok = true;
            if (lane == 0)
                ok = mbar_wait(smem_u32(&bars.empty[st]), (uint32_t)((i / MT_STAGES) & 1) ^ 1u, &abort_flag, wlim);
            if (!__shfl_sync(0xffffffffu, (int)ok, 0)) break;
            __syncwarp();
            const int r0 = (int)(t / ntc) * MT_ROWS, c0 = (int)(t % ntc) * MT_COLS;
            if (!mt_upper(r0, c0)) {
                double2* xs = reinterpret_cast<double2*>(sm + st * MT_STAGE_BYTES + MT_BOX_BYTES);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int m = lane + 32 * h;   // entries c0 + 2m and c0 + 2m + 1
                    const int i0 = c0 + 2 * m;
                    double2 v = make_double2(0.0, 0.0);
                    if (i0 < n3) {
                        double g0, g1;
                        gauss2(seed, stream, (uint32_t)(i0 / 2), g0, g1);
                        v.x = g0 * xscale;
                        v.y = i0 + 1 < n3 ? g1 * xscale : 0.0;
                    }
                    xs[m] = v;
                }
            }
            __syncwarp();
            if (lane == 0) {
                const uint32_t fb = smem_u32(&bars.full[st]);
                const uint32_t dst = sbase + st * MT_STAGE_BYTES;
                mbar_expect_tx(fb, MT_BOX_BYTES + MT_VEC_BYTES);
                tma_load_2d_stream(dst, &map, c0, r0, fb);
                tma_load_1d(dst + MT_BOX_BYTES + MT_VEC_BYTES, &map_f, c0, fb);
            }
        }
        if (lane == 0 && abort_flag) {
            volatile int never = 0;
            for (long long j = i > MT_STAGES ? i - MT_STAGES : 0; j < i; ++j)
                mbar_wait(smem_u32(&bars.full[j % MT_STAGES]), (uint32_t)((j / MT_STAGES) & 1), &never);
        }
    } else if (warp == MT_CW) {
        if (lane == 0) {
            long long i = 0;
            for (long long t = t_beg; t < t_end && !abort_flag; ++t, ++i) {
                const int st = (int)(i % MT_STAGES);
                if (!mbar_wait(smem_u32(&bars.empty[st]), (uint32_t)((i / MT_STAGES) & 1) ^ 1u, &abort_flag, wlim)) break;
                const uint32_t fb = smem_u32(&bars.full[st]);
                const uint32_t dst = sbase + st * MT_STAGE_BYTES;
                const int c0 = (int)(t % ntc) * MT_COLS;
                mbar_expect_tx(fb, MT_STAGE_BYTES);
                // the matrix is read once: evict it first, keep the partials in L2
                tma_load_2d_stream(dst, &map, c0, (int)(t / ntc) * MT_ROWS, fb);
                tma_load_1d(dst + MT_BOX_BYTES, &map_x, c0, fb);
                tma_load_1d(dst + MT_BOX_BYTES + MT_VEC_BYTES, &map_f, c0, fb);
            }
            if (abort_flag) {
                // let the copies still in flight land before the CTA exits
                volatile int never = 0;
                for (long long j = i > MT_STAGES ? i - MT_STAGES : 0; j < i; ++j)
                    mbar_wait(smem_u32(&bars.full[j % MT_STAGES]), (uint32_t)((j / MT_STAGES) & 1), &never);
            }
        }
    } else if (warp == MT_CW + 1) {
        // reducer: the column partials of every tile with a D part, in order
        long long u = 0;
        for (long long t = t_beg; t < t_end; ++t) {
            const int s = (int)(t / ntc), c0 = (int)(t % ntc) * MT_COLS;
            if (mt_lower(s * MT_ROWS, c0)) continue;
            const int b = (int)(u % MT_NB);
            if (!mbar_wait(smem_u32(&bars.cfull[b]), (uint32_t)((u / MT_NB) & 1), &abort_flag, wlim)) break;
            const double2* cp = reinterpret_cast<const double2*>(cpart + (size_t)b * MT_CPART_DOUBLES) + 2 * lane;
            double2 a0 = cp[0], a1 = cp[1];
#pragma unroll
            for (int w = 1; w < MT_CW; ++w) {
                const double2 v0 = cp[w * MT_COLS / 2], v1 = cp[w * MT_COLS / 2 + 1];
                a0.x += v0.x;
                a0.y += v0.y;
                a1.x += v1.x;
                a1.y += v1.y;
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&bars.cempty[b]));
            const int c = c0 + 4 * lane;
            double* o = colp + (size_t)s * n3 + c;
            const double out[4] = {a0.x, a0.y, a1.x, a1.y};
#pragma unroll
            for (int v = 0; v < 4; ++v)
                if (c + v < n3) o[v] = out[v];
            ++u;
        }
    } else {
        double rs[MT_RW], rf[MT_RW], fr[MT_RW];
        int cur = -1;
        long long i = 0, u = 0;
        bool ok = true;
        for (long long t = t_beg; t < t_end; ++t, ++i) {
            const int s = (int)(t / ntc), c0 = (int)(t % ntc) * MT_COLS;
            const int r0 = s * MT_ROWS, rw = r0 + MT_RW * warp;
            if (s != cur) {
                if (cur >= 0 && cur - s_first < slots) {
#pragma unroll
                    for (int q = 0; q < MT_RW; ++q) {
                        const double a = warp_sum(rs[q]), b = warp_sum(rf[q]);
                        if (lane == q) {
                            double* o = rowp + (((size_t)k * slots + (cur - s_first)) * MT_ROWS + MT_RW * warp + q) * 2;
                            o[0] = a;
                            o[1] = b;
                        }
                    }
                }
                cur = s;
#pragma unroll
                for (int q = 0; q < MT_RW; ++q) {
                    rs[q] = 0;
                    rf[q] = 0;
                    fr[q] = rw + q < n3 ? F[rw + q] : 0.0;
                }
            }
            const int c = c0 + 4 * lane;
            const bool lower = mt_lower(r0, c0), upper = mt_upper(r0, c0);
            const int st = (int)(i % MT_STAGES);
            ok = mbar_wait(smem_u32(&bars.full[st]), (uint32_t)((i / MT_STAGES) & 1), &abort_flag, wlim);
            if (!ok) break;
            const unsigned char* stage = sm + st * MT_STAGE_BYTES;
            const float4* tile = reinterpret_cast<const float4*>(stage) + 32 * MT_RW * warp + lane;
            // the tile's X and F entries (zero beyond 3N: the boxes are filled)
            const double2* xs = reinterpret_cast<const double2*>(stage + MT_BOX_BYTES) + 2 * lane;
            const double2* fs = reinterpret_cast<const double2*>(stage + MT_BOX_BYTES + MT_VEC_BYTES) + 2 * lane;
            double x[4] = {0, 0, 0, 0}, f[4] = {0, 0, 0, 0};
            if (!upper) {
                const double2 xa = xs[0], xb = xs[1];
                x[0] = xa.x;
                x[1] = xa.y;
                x[2] = xb.x;
                x[3] = xb.y;
            }
            if (!lower) {
                const double2 fa = fs[0], fb = fs[1];
                f[0] = fa.x;
                f[1] = fa.y;
                f[2] = fb.x;
                f[3] = fb.y;
            }
            double pc[4] = {0, 0, 0, 0};
            if (lower) {
#pragma unroll
                for (int q = 0; q < MT_RW; ++q) {
                    const float4 m = tile[32 * q];
                    rs[q] = fma((double)m.x, x[0], rs[q]);
                    rs[q] = fma((double)m.y, x[1], rs[q]);
                    rs[q] = fma((double)m.z, x[2], rs[q]);
                    rs[q] = fma((double)m.w, x[3], rs[q]);
                }
            } else if (upper) {
#pragma unroll
                for (int q = 0; q < MT_RW; ++q) {
                    const float4 m = tile[32 * q];
                    const double m0 = m.x, m1 = m.y, m2 = m.z, m3 = m.w;
                    rf[q] = fma(m0, f[0], rf[q]);
                    rf[q] = fma(m1, f[1], rf[q]);
                    rf[q] = fma(m2, f[2], rf[q]);
                    rf[q] = fma(m3, f[3], rf[q]);
                    pc[0] = fma(m0, fr[q], pc[0]);
                    pc[1] = fma(m1, fr[q], pc[1]);
                    pc[2] = fma(m2, fr[q], pc[2]);
                    pc[3] = fma(m3, fr[q], pc[3]);
                }
            } else {
                // tile crossing the diagonal: element (r, c) is L for c <= r
#pragma unroll
                for (int q = 0; q < MT_RW; ++q) {
                    const float4 m = tile[32 * q];
                    const double mv[4] = {m.x, m.y, m.z, m.w};
#pragma unroll
                    for (int v = 0; v < 4; ++v) {
                        if (c + v <= rw + q) {
                            rs[q] = fma(mv[v], x[v], rs[q]);
                        } else {
                            rf[q] = fma(mv[v], f[v], rf[q]);
                            pc[v] = fma(mv[v], fr[q], pc[v]);
                        }
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&bars.empty[st]));
            if (!lower) {
                const int b = (int)(u % MT_NB);
                ok = mbar_wait(smem_u32(&bars.cempty[b]), (uint32_t)((u / MT_NB) & 1) ^ 1u, &abort_flag, wlim);
                if (!ok) break;
                double2* cp = reinterpret_cast<double2*>(cpart + (size_t)b * MT_CPART_DOUBLES + warp * MT_COLS) + 2 * lane;
                cp[0] = make_double2(pc[0], pc[1]);
                cp[1] = make_double2(pc[2], pc[3]);
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_u32(&bars.cfull[b]));
                ++u;
            }
        }
        if (ok && cur >= 0 && cur - s_first < slots) {
#pragma unroll
            for (int q = 0; q < MT_RW; ++q) {
                const double a = warp_sum(rs[q]), b = warp_sum(rf[q]);
                if (lane == q) {
                    double* o = rowp + (((size_t)k * slots + (cur - s_first)) * MT_ROWS + MT_RW * warp + q) * 2;
                    o[0] = a;
                    o[1] = b;
                }
            }
        }
    }
    if (abort_flag && tid == 0) atomicOr(status, ST_TIMEOUT);
}

// Rs and Rf for the TMA kernel's partials: row r of strip s gets the row
// partials of the CTAs whose ranges overlap the strip's tiles, in CTA order,
// then dD F and the column partials of the strips above (as k_mv_finish).
__global__ void __launch_bounds__(FIN_ROWS * FIN_GROUPS)
k_mv_finish_tma(int n3, int ntc, long long T, int G, int slots, const double* __restrict__ rowp, const double* __restrict__ colp,
                const double* __restrict__ dD, const double* __restrict__ F, double pre, double* __restrict__ Rf,
                double* __restrict__ Rs, int want_rs, double* __restrict__ pos_d, int periodic, double3 box,
                double3 inv_L, unsigned long long* __restrict__ ctr, uint64_t seed, double xscale,
                double* __restrict__ X)
{
    __shared__ double part[FIN_GROUPS][FIN_ROWS + 1];
    const int tx = threadIdx.x % FIN_ROWS, ty = threadIdx.x / FIN_ROWS;
    const int r = blockIdx.x * FIN_ROWS + tx;
    // 8 independent loads in flight per thread (register accumulators)
    double c[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (r < n3) {
        const int nst = (r + MT_ROWS - 1) / MT_ROWS;   // strips st with st * 64 < r
        for (int base = ty; base < nst; base += 8 * FIN_GROUPS) {
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int st = base + q * FIN_GROUPS;
                if (st < nst) c[q] += colp[(size_t)st * n3 + r];
            }
        }
    }
    part[ty][tx] = ((c[0] + c[1]) + (c[2] + c[3])) + ((c[4] + c[5]) + (c[6] + c[7]));
    __syncthreads();
    if (ty == 0 && r < n3) {
        const int s = r / MT_ROWS;
        const long long ta = (long long)s * ntc, tb = ta + ntc - 1;
        // CTA holding tile t: the largest k with k T / G <= t
        const int ka = (int)(((ta + 1) * G - 1) / T), kb = (int)(((tb + 1) * G - 1) / T);
        double sr = 0, f = 0;
        for (int k = ka; k <= kb; ++k) {
            const int slot = s - (int)(((long long)k * T / G) / ntc);
            const double* o = rowp + (((size_t)k * slots + slot) * MT_ROWS + r % MT_ROWS) * 2;
            sr += o[0];
            f += o[1];
        }
        f += dD[r] * F[r];
        for (int g = 0; g < FIN_GROUPS; ++g) f += part[g][tx];
        Rf[r] = f * pre;
        if (want_rs) Rs[r] = sr;
        if (pos_d) {
            // the position update of k_update (no flow) for this coordinate:
            // the same operations in the same order, so the same bits
            double* pc = pos_d + 4 * (r / 3) + r % 3;
            double v = add(add(f * pre, sr), *pc);
            if (periodic) {
                const double L = (&box.x)[r % 3], iL = (&inv_L.x)[r % 3];
                v = sub(v, mul(L, floor(add(mul(v, iL), 0.5))));
            }
            *pc = v;
        }
    }
    if (ctr) {
        // the next step's noise, drawn ahead (the product of this step is
        // done with X): the Gaussians of stream index + 1, as k_noise would
        // draw them
        const uint64_t next = *reinterpret_cast<volatile unsigned long long*>(ctr) + 1;
        if (ty == 0 && r < n3 && (r & 1) == 0) {
            double g0, g1;
            gauss2(seed, next, (uint32_t)(r / 2), g0, g1);
            X[r] = g0 * xscale;
            if (r + 1 < n3) X[r + 1] = g1 * xscale;
        }
        // the last block advances the Philox stream index, as k_noise does,
        // and tags X as holding its noise
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            const unsigned done = atomicAdd(reinterpret_cast<unsigned*>(ctr + 1), 1u);
            if (done == gridDim.x - 1) {
                const unsigned long long stream = *reinterpret_cast<volatile unsigned long long*>(ctr);
                ctr[1] = 0;
                ctr[0] = stream + 1;
                ctr[2] = stream + 2;
                __threadfence();
            }
        }
    }
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

// (re)encode the tensor maps (the FP32 matrix, X and F) when one of the
// buffers changed (IGT swaps its two matrices), and size the persistent grid
static int mv_tma_setup(bdb_system* s)
{
    const void* src[3] = {s->M32.p, s->X.p, s->F.p};
    if (std::equal(src, src + 3, s->mv_map_src)) return BDB_OK;
    auto enc = get_encode();
    if (!enc) return fail(BDB_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    if (reinterpret_cast<uintptr_t>(s->M32.p) % 16 || s->npad % 4 || reinterpret_cast<uintptr_t>(s->X.p) % 16 ||
        reinterpret_cast<uintptr_t>(s->F.p) % 16)
        return fail(BDB_ERR_ARG, "matvec operands not 16-byte aligned");
    CUtensorMap* maps = reinterpret_cast<CUtensorMap*>(s->mv_map);
    cuuint64_t dims[2] = {(cuuint64_t)s->n3, (cuuint64_t)s->n3};
    cuuint64_t strides[1] = {(cuuint64_t)s->npad * sizeof(float)};
    cuuint32_t box[2] = {MT_COLS, MT_ROWS};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(&maps[0], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, s->M32.p, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    for (int v = 0; v < 2 && r == CUDA_SUCCESS; ++v)
        r = enc(&maps[1 + v], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 1, v ? (void*)s->F.p : (void*)s->X.p, dims, strides,
                box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(BDB_ERR_CUDA, "cuTensorMapEncodeTiled failed (matvec)");
    if (!s->mv_ctas_per_sm) {
        BDB_CUDA(cudaFuncSetAttribute(k_strip_mv_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, MT_SMEM));
        int occ = 0;
        BDB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_strip_mv_tma, MT_THREADS, MT_SMEM));
        s->mv_ctas_per_sm = std::max(1, occ);
    }
    std::copy(src, src + 3, s->mv_map_src);
    return BDB_OK;
}

// grid of the TMA kernel: all resident CTAs, at most one per tile
static int mv_tma_grid(const bdb_system* s, long long T)
{
    return (int)std::min<long long>(T, (long long)s->mv_ctas_per_sm * s->sm_count);
}

// strips a CTA's range of at most ceil(T / G) tiles can touch
static int mv_tma_slots(long long T, int G, int ntc)
{
    const long long len = (T + G - 1) / G;
    return (int)((len + ntc - 1) / ntc) + 1;
}

// fused: the position update inside the finisher, which also draws the
// next step's Philox noise into X (Cholesky scaling sqrt(2 dt)); the
// product uses that X, or draws its own when X does not hold this step's
// noise. The caller has checked that no flow is on.
static int stored_matvec_tma(bdb_system* s, bool want_rs, bool fused = false)
{
    int rc = mv_tma_setup(s);
    if (rc) return rc;
    const int n3 = s->n3;
    const int nstrip = (n3 + MT_ROWS - 1) / MT_ROWS, ntc = (n3 + MT_COLS - 1) / MT_COLS;
    const long long T = (long long)nstrip * ntc;
    const int G = mv_tma_grid(s, T);
    const int slots = mv_tma_slots(T, G, ntc);
    const size_t need = (size_t)G * slots * MT_ROWS * 2 + (size_t)nstrip * n3;
    if (s->part.n < need) {
        if (s->part.alloc(need)) return BDB_ERR_NOMEM;
    }
    double* rowp = s->part.p;
    double* colp = s->part.p + (size_t)G * slots * MT_ROWS * 2;
    const CUtensorMap* maps = reinterpret_cast<const CUtensorMap*>(s->mv_map);
    // X: any valid vector when Rs is not wanted
    k_strip_mv_tma<<<G, MT_THREADS, MT_SMEM, s->stream>>>(maps[0], want_rs ? maps[1] : maps[2], maps[2], n3, ntc, T,
                                                           slots, s->F.p, rowp, colp, s->status.p,
                                                           (uint32_t)s->wait_limit, fused ? 1 : 0, s->p.seed,
                                                           s->ctr.p, sqrt(2 * s->p.dt));
    BDB_CUDA(cudaGetLastError());
    const double pre = s->p.dt / (BDB_KB * s->p.T);
    k_mv_finish_tma<<<(n3 + FIN_ROWS - 1) / FIN_ROWS, FIN_ROWS * FIN_GROUPS, 0, s->stream>>>(
        n3, ntc, T, G, slots, rowp, colp, s->dD.p, s->F.p, pre, s->Rf.p, s->Rs.p, want_rs,
        fused ? reinterpret_cast<double*>(s->pos.p) : nullptr, s->p.bc == 1,
        make_double3(s->p.box[0], s->p.box[1], s->p.box[2]), make_double3(s->inv_L[0], s->inv_L[1], s->inv_L[2]),
        fused ? s->ctr.p : nullptr, s->p.seed, sqrt(2 * s->p.dt), s->X.p);
    BDB_CUDA(cudaGetLastError());
    s->launches += 2;
    return BDB_OK;
}

int stored_matvec_step(bdb_system* s) { return stored_matvec_tma(s, true, true); }

int stored_matvec(bdb_system* s, bool want_rs)
{
    if (s->p.precision != BDB_PREC_FP64) return stored_matvec_tma(s, want_rs);
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

// Set-up of the entry point, per device: the device address of the array
// (the host-side symbol is only a stand-in for it) and the SM count. A
// module's device variables can move when the device's context is destroyed
// and created again (cudaDeviceReset), so each entry remembers the context it
// was made in and is made again in a new one. The mutex orders first calls
// from several host threads.
static constexpr int NOALLOC_MAX_DEVICES = 64;
struct NoallocSlot {
    bool set = false;
    unsigned long long ctx_id = 0;
    double* scratch = nullptr;
    int sms = 0;
};
static NoallocSlot g_noalloc_slot[NOALLOC_MAX_DEVICES];
static std::mutex g_noalloc_mu;

// ID of the calling thread's current context, 0 if it has none yet
static unsigned long long current_context_id()
{
    static PFN_cuCtxGetCurrent_v4000 get_cur = nullptr;
    static PFN_cuCtxGetId_v12000 get_id = nullptr;
    if (!get_cur || !get_id) {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_cur = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(p);
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(p);
        if (!get_cur || !get_id) return 0;
    }
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_cur(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

static int noalloc_setup(int dev, double** scratch, int* sms)
{
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoallocSlot& sl = g_noalloc_slot[dev];
    unsigned long long id = current_context_id();
    if (!sl.set || id == 0 || sl.ctx_id != id) {
        void* p = nullptr;
        BDB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));   // creates the context if there is none
        int m = 0;
        BDB_CUDA(cudaDeviceGetAttribute(&m, cudaDevAttrMultiProcessorCount, dev));
        if (id == 0) id = current_context_id();
        sl.set = id != 0;   // without a context ID, look the address up on every call
        sl.ctx_id = id;
        sl.scratch = static_cast<double*>(p);
        sl.sms = std::max(1, m);
    }
    *scratch = sl.scratch;
    *sms = sl.sms;
    return BDB_OK;
}

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
    // set-up, once per device (again in a new context), with the device
    // current: the kernels need the array's device address
    double* scratch = nullptr;
    int sms = 0;
    int rc = noalloc_setup(dev, &scratch, &sms);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nstrip = (n3 + STRIP - 1) / STRIP;
    // the segmentation of the system path (16 warps per SM), with no more
    // column segments than the row partials' share of the array holds
    int nseg, seg_cols;
    mv_split(n3, 16, sms, &nseg, &seg_cols);
    const int max_seg = (int)((NOALLOC_SCRATCH - (size_t)nstrip * n3) / (2 * (size_t)n3));
    if (nseg > max_seg) {
        seg_cols = ((n3 + max_seg - 1) / max_seg + 127) / 128 * 128;
        nseg = (n3 + seg_cols - 1) / seg_cols;
    }
    // every partial that k_mv_finish reads is written first by k_strip_mv,
    // so nothing in the scratch has to start at zero
    double* rowp = scratch;
    double* colp = rowp + (size_t)nseg * n3 * 2;
    const int blocks = (nstrip * nseg + WARPS - 1) / WARPS;
    k_strip_mv<float><<<blocks, 32 * WARPS, 0, st>>>(M, n3, ld, nseg, seg_cols, F, X, rowp, colp);
    BDB_CUDA(cudaGetLastError());
    mv_finish(st, n3, nseg, rowp, colp, dD, F, pre, Rf, Rs, 1);
    BDB_CUDA(cudaGetLastError());
    return BDB_OK;
}
