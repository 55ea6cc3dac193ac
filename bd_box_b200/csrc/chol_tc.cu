// Mixed-precision blocked Cholesky for sm_100a: FP64 panels, 3xTF32
// trailing updates on the 5th-generation tensor cores (tcgen05).
//
// M is FP32 (lower triangle: the factor, upper: D, never written here).
// Super-panel P covers columns p0 = 128P .. p0+127:
//   k_potrf128  one CTA factors the 128x128 diagonal block in FP64,
//               right-looking by 8 columns with the 8x8 pivot blocks factored
//               in registers by one thread while the others update; L_PP goes
//               to M (FP32), and its inverse W = L_PP^-1 (FP64, blocked
//               forward substitution) transposed to a scratch block;
//   k_trsm128   slabs of 64 rows below the block solve X L_PP^T = A in FP64
//               as the product X = A W^T (no sequential dependency); each row
//               goes to M and its TF32 split L = L_hi + L_lo (L_hi: low 13
//               mantissa bits cleared, exactly TF32; L_lo = L - L_hi) to two
//               panel buffers;
//   k_syrk_tc   C -= L_i L_j^T over all 128x128 tiles ti >= tj > P of the
//               trailing lower triangle, with
//               L_i L_j^T ~= Lhi_i Lhi_j^T + Lhi_i Llo_j^T + Llo_i Lhi_j^T
//               (the dropped lo*lo term is ~2^-22 relative: FP32 accuracy).
//
// k_syrk_tc is persistent (one CTA per SM, static round-robin over tiles)
// and warp-specialised:
//   warp 0    TMA producer: per K chunk of 32 columns, four 128x32 FP32 boxes
//             (A_hi, A_lo, B_hi, B_lo, 128-byte swizzle) into a 3-stage ring;
//   warp 1    MMA issuer: tcgen05.mma.kind::tf32 M=128 N=128 K=8, three per
//             K step, into one of two TMEM accumulators (128 columns each);
//             tcgen05.commit frees a ring stage / publishes an accumulator;
//   warps 2-5 epilogue: tcgen05.ld of the accumulator (warp w reads TMEM
//             lanes 32(w%4)..), hand the accumulator back, then -acc per
//             128x32 box into a 2-box shared-memory ring and a TMA
//             reduce-add into C (lower triangle only on diagonal tiles);
//             C is never loaded.
// The epilogue of tile t overlaps the MMAs of tile t+1 and the loads of the
// tiles after it. Every mbarrier wait is bounded; a time-out sets
// ST_TIMEOUT and a shared abort flag that stops all roles, and the CTA frees
// its tensor memory before returning.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>

#include "bdb_common.cuh"
#include "sm100.cuh"

namespace bdb {

static constexpr int PW = 128;                    // super-panel width = tile size
static constexpr int KC = 32;                     // K columns per TMA box (128 B of FP32)
static constexpr int NCHUNK = PW / KC;            // 4
static constexpr int STAGES = 3;
static constexpr int BOX_BYTES = PW * KC * 4;     // 16 KB
static constexpr int STAGE_BYTES = 4 * BOX_BYTES; // A_hi, A_lo, B_hi, B_lo
static constexpr int C_BOXES = 2;                 // staging ring of 128x32 boxes for the C update
static constexpr int SYRK_SMEM = STAGES * STAGE_BYTES + C_BOXES * BOX_BYTES + 1024;

// C[tile] += smem tile (FP32 add in L2, no load of C by the SM)
__device__ __forceinline__ void tma_reduce_add_2d(const CUtensorMap* map, uint32_t src, int x, int y)
{
    asm volatile("cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y), "r"(src)
                 : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

// wait until at most C_BOXES-1 of this thread's bulk groups still read
// shared memory
__device__ __forceinline__ void bulk_wait_read_ring()
{
    static_assert(C_BOXES == 2, "wait_group count below");
    asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
}

__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// barrier 1 among the 128 epilogue threads only
__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

// barrier 1 with an OR over the 128 epilogue threads: all of them see the
// same answer, so they leave their loop together
__device__ __forceinline__ bool epi_any(bool x)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "bar.red.or.pred p, 1, 128, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)x)
        : "memory");
    return r != 0;
}

// UMMA shared-memory descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO = 64 x 16 B), LBO = 1 (unused for swizzled K-major),
// version 1 (sm_100), layout type 2 (SWIZZLE_128B).
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1u << 16;
    d |= (uint64_t)64u << 32;
    d |= (uint64_t)1u << 46;
    d |= (uint64_t)2u << 61;
    return d;
}

// instruction descriptor: D=F32, A=B=TF32, both K-major, N=128, M=128
__host__ __device__ constexpr uint32_t idesc_tf32_128x128()
{
    return (1u << 4) | (2u << 7) | (2u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tri_index(int idx, int& ti, int& tj)
{
    int i = (int)((sqrtf(8.0f * (float)idx + 1.0f) - 1.0f) * 0.5f);
    while ((i + 1) * (i + 2) / 2 <= idx) ++i;
    while (i * (i + 1) / 2 > idx) --i;
    ti = i;
    tj = idx - i * (i + 1) / 2;
}

// tile t of a launch -> (ti, tj) relative to the first trailing block:
// mode 0 all tiles of the lower triangle, 1 only block column 0,
// 2 all but block column 0
__device__ __forceinline__ void tile_of_mode(int t, int mode, int& ti, int& tj)
{
    if (mode == 1) {
        ti = t;
        tj = 0;
    } else {
        tri_index(t, ti, tj);
        if (mode == 2) {
            ++ti;
            ++tj;
        }
    }
}

__device__ __forceinline__ float tf32_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }

// ------------------------------------------------------------ FP64 panel

// 1/sqrt(x) for x > 0 in FP64: the single-precision estimate (relative
// error ~2^-22) refined by one Newton-Raphson step y <- y (3 - x y^2) / 2,
// which squares the error to ~2^-43: far below the FP32 rounding of the
// factor that leaves this kernel, with half the dependency chain of a
// second step.
__device__ __forceinline__ double rsqrt_nr(double x)
{
    const double y = (double)rsqrtf((float)x);
    return y * (1.5 - 0.5 * x * y * y);
}

// FP64 tensor-core MMA (the only FP64 tensor instruction on sm_100a; the
// tcgen05 kinds have no FP64): D = A B + C for an 8x8 tile, k = 4. Lane l
// holds A[l/4][l%4], B[l%4][l/4] and C/D[l/4][2(l%4) + {0,1}].
__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// 8x8 FP64 tiles in shared memory are kept in MMA fragment order, two
// k-steps per lane (one 16-byte load per operand and tile):
//   A order: entry 2 l + h = T[l/4][4h + l%4]   (A fragments of T, and also
//            the B fragments of T^T)
//   B order: entry 2 l + h = T[4h + l%4][l/4]   (B fragments of T)
__device__ __forceinline__ int apos(int r, int c) { return ((r << 2) + (c & 3)) * 2 + (c >> 2); }
__device__ __forceinline__ int bpos(int r, int c) { return ((c << 2) + (r & 3)) * 2 + (r >> 2); }
// tile (g, n), n <= g, of the lower triangle of 16 x 16 tiles
__device__ __forceinline__ int tix(int g, int n) { return g * (g + 1) / 2 + n; }

// 1/x for x > 0 in FP64: the single-precision hardware estimate refined by
// one Newton-Raphson step q <- q + q (1 - x q) (error ~2^-46).
__device__ __forceinline__ double rcp_nr(double x)
{
    float e;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"((float)x));
    const double q = (double)e;
    return fma(q, fma(-x, q, 1.0), q);
}

// Factor the 8x8 block in Dg ([8][9], lower triangle) in registers by one
// thread: L_kk to the lower triangle of Dg, 1/L_jj to rd. The elimination
// runs on the unscaled Schur complements, a_ik -= (a_ij a_kj) q_j with
// q_j = 1/a_jj, so the dependency chain from one pivot to the next is one
// reciprocal and one FMA (the products a_ij a_kj are formed while q_j is
// computed); the columns are scaled by 1/sqrt(a_jj) at the end.
__device__ __forceinline__ bool pivot8(double* Dg, double* rd)
{
    double a[8][8];
    bool ok = true;
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c <= r; ++c) a[r][c] = Dg[r * 9 + c];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        if (!(a[j][j] > 0.0)) ok = false;
        const double q = rcp_nr(a[j][j]);
#pragma unroll
        for (int r = j + 1; r < 8; ++r)
#pragma unroll
            for (int c = j + 1; c <= r; ++c) a[r][c] = fma(-(a[r][j] * a[c][j]), q, a[r][c]);
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const double r = rsqrt_nr(a[j][j]);
        rd[j] = r;
        Dg[j * 9 + j] = a[j][j] * r;
#pragma unroll
        for (int i = j + 1; i < 8; ++i) Dg[i * 9 + j] = a[i][j] * r;
    }
    return ok;
}

static constexpr int POTRF_THREADS = 512;
static constexpr int NT = PW / 8;                  // 16 row groups of 8 rows
static constexpr int NTILE = NT * (NT + 1) / 2;    // 136 tiles in the lower triangle
static constexpr int POTRF_SMEM = (NTILE * 64 + NT * 64 + 80 + 8 + 2 * 64) * 8;
// factor hand-off to the panel solve: L_PP tiles then the W_kk, A order
static constexpr int PANEL_FAC = (NTILE + NT) * 64;

// row group owned by a warp: warp 0 runs the pivots; warps 4, 8, 12 share
// its scheduler (warp w issues on sub-partition w mod 4) and own the row
// groups with the least update work (1, 2, 3); the other 12 warps own 4..15
__device__ __forceinline__ int row_group_of(int warp)
{
    return (warp & 3) ? 4 + warp - 1 - (warp >> 2) : warp >> 2;
}

// FP64 factorisation L_PP of the 128x128 diagonal block (P, P) and the
// inverses W_kk of its 8x8 diagonal tiles, right-looking over 16 blocks of 8
// columns with the
// trailing matrix held in registers: the warp owning row group g keeps its
// tiles (g, n), n <= g, as DMMA accumulators. Iteration k:
//   warp 0      factors diagonal tile (k, k) (pivot8) and inverts it
//               (lanes 0-7), publishing W_kk, L_kk in shared memory;
//   barrier;
//   owners g>k  solve tile (g, k): L[g][k] = C[g][k] W_kk^T (two DMMAs),
//               published in A order;
//   barrier;
//   warp 0      applies the last update to diagonal tile k+1 itself (two
//               DMMAs on the copy its owner handed over one iteration
//               earlier), then goes on to pivot k+1;
//   owners g>k+1 update their tiles n = k+1..g: C[g][n] -= L[g][k] L[n][k]^T,
//               and the owner of row group k+2 hands its diagonal tile
//               (now updated through column k) to warp 0.
//   The next pivot thus waits for no owner: warp 0's sub-partition carries
//   no bulk update (its other warps own row groups 1-3), while an owner's
//   MMAs queue behind those of the three other owners on its own.
// Finally L_PP goes to M (FP32, lower triangle) and, in FP64 for the panel
// solve, its 136 tiles followed by the 16 W_kk to Wt (A order; PANEL_FAC
// doubles). (Storing each tile as soon as it is final measured slower: the
// stores then compete with the pivot chain.)
__global__ void __launch_bounds__(POTRF_THREADS, 1) k_potrf128(float* __restrict__ M, int npad, int P,
                                                            double* __restrict__ Wt, unsigned* __restrict__ status)
{
    extern __shared__ double sh[];
    double* Lt = sh;                       // [NTILE][64] A order
    double* Wa = Lt + NTILE * 64;          // [NT][64] W_kk in A order
    double* Dg = Wa + NT * 64;             // [8][9] diagonal block being factored
    double* rd = Dg + 80;                  // [8] 1/L_jj of that block
    double* Hd = rd + 8;                   // [2][64] diagonal tiles handed to warp 0 (C layout)
    __shared__ int bad;
    {
        // the warp roles and barrier counts assume this exact launch shape
        uint32_t dyn;
        asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
        if (blockDim.x != POTRF_THREADS || dyn < (uint32_t)POTRF_SMEM) {
            if (threadIdx.x == 0) atomicOr(status, ST_LAUNCH);
            return;
        }
    }
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int fr = lane >> 2, fq = lane & 3;
    const size_t base = (size_t)P * PW;
    const int g = row_group_of(warp);
    if (tid == 0) bad = 0;
    if (warp == 0) {
        // ---------------------------------------------------- pivot warp
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int c = 2 * fq + e;
            Dg[fr * 9 + c] = c <= fr ? (double)M[(base + fr) * npad + base + c] : 0.0;
        }
        for (int k = 0; k < NT; ++k) {
            __syncwarp();
            if (lane == 0 && !pivot8(Dg, rd)) bad = 1;
            __syncwarp();
            if (lane < 8) {
                // column c of W_kk by forward substitution (w[m] = 0 for
                // m < c, so every row sums over all m < i); W_kk and L_kk out
                const int c = lane;
                double lk[8][8], r8[8], w[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    r8[i] = rd[i];
#pragma unroll
                    for (int m = 0; m < i; ++m) lk[i][m] = Dg[i * 9 + m];
                }
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    double v = i == c ? 1.0 : 0.0;
#pragma unroll
                    for (int m = 0; m < i; ++m) v = fma(-lk[i][m], w[m], v);
                    w[i] = i >= c ? v * r8[i] : 0.0;
                }
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const double l = i >= c ? Dg[i * 9 + c] : 0.0;
                    Wa[k * 64 + apos(i, c)] = w[i];
                    Lt[tix(k, k) * 64 + apos(i, c)] = l;
                }
            }
            __syncthreads();   // A: W_kk published
            __syncthreads();   // B: block column k solved
            if (k + 1 < NT) {
                // diagonal tile k+1 = its owner's copy - L[k+1][k] L[k+1][k]^T
                const double2 t = *reinterpret_cast<const double2*>(Hd + ((k + 1) & 1) * 64 + 2 * lane);
                const double2 av = *reinterpret_cast<const double2*>(Lt + tix(k + 1, k) * 64 + 2 * lane);
                double e0 = t.x, e1 = t.y;
                dmma884(e0, e1, -av.x, av.x);
                dmma884(e0, e1, -av.y, av.y);
                Dg[fr * 9 + 2 * fq] = e0;
                Dg[fr * 9 + 2 * fq + 1] = e1;
            }
        }
    } else {
        // -------------------------------------------------- tile owners
        double cacc[NT][2];
#pragma unroll
        for (int n = 0; n < NT; ++n) {
            cacc[n][0] = cacc[n][1] = 0.0;
            if (n <= g) {
                const float2 v =
                    *reinterpret_cast<const float2*>(M + (base + 8 * g + fr) * npad + base + 8 * n + 2 * fq);
                cacc[n][0] = (n < g || 2 * fq <= fr) ? (double)v.x : 0.0;
                cacc[n][1] = (n < g || 2 * fq + 1 <= fr) ? (double)v.y : 0.0;
            }
        }
        if (g == 1)   // row group 1's diagonal tile needs only column 0: warp 0's
            *reinterpret_cast<double2*>(Hd + 64 + 2 * lane) = make_double2(cacc[1][0], cacc[1][1]);
        for (int k = 0; k < NT; ++k) {
            __syncthreads();   // A
            if (g > k) {
                // A fragments of C[g][k] (C layout -> A layout by shuffles)
                double c0 = 0.0, c1 = 0.0;
#pragma unroll
                for (int t = 0; t < NT; ++t)
                    if (t == k) {
                        c0 = cacc[t][0];
                        c1 = cacc[t][1];
                    }
                double x0 = 0.0, x1 = 0.0;
                const double2 wb = *reinterpret_cast<const double2*>(Wa + k * 64 + 2 * lane);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int src = (fr << 2) + 2 * h + (fq >> 1);
                    const double v0 = __shfl_sync(0xffffffffu, c0, src);
                    const double v1 = __shfl_sync(0xffffffffu, c1, src);
                    dmma884(x0, x1, (fq & 1) ? v1 : v0, h ? wb.y : wb.x);
                }
                Lt[tix(g, k) * 64 + apos(fr, 2 * fq)] = x0;
                Lt[tix(g, k) * 64 + apos(fr, 2 * fq + 1)] = x1;
            }
            __syncthreads();   // B
            if (g > k + 1) {
                const double2 av = *reinterpret_cast<const double2*>(Lt + tix(g, k) * 64 + 2 * lane);
                // four tiles per batch: their operand loads first (predicated,
                // no branch), then the MMAs
#pragma unroll
                for (int n0 = 1; n0 < NT; n0 += 4) {
                    double2 bv[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int n = n0 + u;
                        const bool act = n < NT && n > k && n <= g;
                        bv[u] = act ? *reinterpret_cast<const double2*>(Lt + tix(n, k) * 64 + 2 * lane)
                                    : make_double2(0.0, 0.0);
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int n = n0 + u;
                        if (n < NT && n > k && n <= g) {
                            dmma884(cacc[n][0], cacc[n][1], -av.x, bv[u].x);
                            dmma884(cacc[n][0], cacc[n][1], -av.y, bv[u].y);
                        }
                    }
                }
                if (g == k + 2) {
                    // hand the diagonal tile (updated through column k) to
                    // warp 0, which applies column k+1 itself
                    double d0 = 0.0, d1 = 0.0;
#pragma unroll
                    for (int t = 0; t < NT; ++t)
                        if (t == g) {
                            d0 = cacc[t][0];
                            d1 = cacc[t][1];
                        }
                    *reinterpret_cast<double2*>(Hd + (g & 1) * 64 + 2 * lane) = make_double2(d0, d1);
                }
            }
        }
    }
    __syncthreads();
    if (tid == 0 && bad) atomicOr(status, ST_NOT_SPD);
    // L_PP to M (FP32, lower triangle)
#pragma unroll 4
    for (int idx = tid; idx < PW * PW; idx += POTRF_THREADS) {
        const int r = idx / PW, c = idx % PW;
        if (c <= r) M[(base + r) * npad + base + c] = (float)Lt[tix(r >> 3, c >> 3) * 64 + apos(r & 7, c & 7)];
    }
    // L_PP tiles and the W_kk (A order, FP64) for the panel solve
    {
        const double2* src = reinterpret_cast<const double2*>(Lt);
        double2* dst = reinterpret_cast<double2*>(Wt);
#pragma unroll 4
        for (int f = tid; f < PANEL_FAC / 2; f += POTRF_THREADS) dst[f] = src[f];
    }
}

// Rows below block P: X L_PP^T = A by blocked forward substitution in FP64
// on the DMMA path, from the tiles of L_PP and the inverses W_kk of its
// diagonal tiles (k_potrf128). Work unit = one row group of 8 rows, owned by
// one warp, which keeps the unit's 16 tiles C_n (8x8, 32 doubles per lane)
// as DMMA accumulators loaded straight from M. For n = 0..15:
//   X_n = C_n W_nn^T                       (two DMMAs),
//   C_n' -= X_n L_n'n^T for n' > n         (two DMMAs each),
// 272 DMMAs per unit; C_n -> A fragments by shuffles. The CTA copies the
// factor (76 KB) into shared memory once. The grid is persistent: unit u goes
// to warp slot u mod (8 grid), slots ordered so that the first 4 grid slots
// put one warp on every SM sub-partition, the next 4 grid a second one.
// Writes the rows to M and their TF32 split L = L_hi + L_lo (L_hi: low 13
// mantissa bits cleared, exactly TF32; L_lo = L - L_hi) to the panel
// buffers.
static constexpr int TRSM_THREADS = 256;
static constexpr int TRSM_SMEM = PANEL_FAC * 8;

// A fragment of k-step h of an 8x8 tile held as C fragments (lane (r, q)
// holds T[r][2q], T[r][2q+1]; the A fragment is T[r][4h + q])
__device__ __forceinline__ double c2a(double c0, double c1, int h, int fr, int fq)
{
    const int src = (fr << 2) + 2 * h + (fq >> 1);
    const double v0 = __shfl_sync(0xffffffffu, c0, src);
    const double v1 = __shfl_sync(0xffffffffu, c1, src);
    return (fq & 1) ? v1 : v0;
}

__global__ void __launch_bounds__(TRSM_THREADS, 1) k_trsm128(float* __restrict__ M, int npad, int P,
                                                          const double* __restrict__ Lf, float* __restrict__ Lhi,
                                                          float* __restrict__ Llo, unsigned* __restrict__ status)
{
    {
        uint32_t dyn;
        asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
        if (blockDim.x != TRSM_THREADS || dyn < (uint32_t)TRSM_SMEM) {
            if (threadIdx.x == 0) atomicOr(status, ST_LAUNCH);
            return;
        }
    }
    asm volatile("griddepcontrol.launch_dependents;");
    extern __shared__ double sh[];
    const double2* Ls = reinterpret_cast<const double2*>(sh);               // [NTILE][32] pairs
    const double2* Ws = reinterpret_cast<const double2*>(sh + NTILE * 64);  // [NT][32] pairs
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int fr = lane >> 2, fq = lane & 3;
    const size_t base = (size_t)P * PW;
    const size_t row0 = base + PW;
    const int units = (int)(((size_t)npad - row0) / 8);
    {
        // the factor: a plain copy, loads batched ahead of stores
        const double2* src = reinterpret_cast<const double2*>(Lf);
        double2* dst = reinterpret_cast<double2*>(sh);
        constexpr int NC = PANEL_FAC / 2;
        constexpr int PER = (NC + TRSM_THREADS - 1) / TRSM_THREADS;   // 19
        double2 w[PER];
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int f = tid + TRSM_THREADS * k;
            if (f < NC) w[k] = __ldg(src + f);
        }
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int f = tid + TRSM_THREADS * k;
            if (f < NC) dst[f] = w[k];
        }
    }
    __syncthreads();
    const int slot = (warp >> 2) * 4 * gridDim.x + blockIdx.x * 4 + (warp & 3);
    for (int u = slot; u < units; u += TRSM_THREADS / 32 * gridDim.x) {
        const size_t row = row0 + (size_t)8 * u + fr;
        double c[16][2];
#pragma unroll
        for (int n = 0; n < 16; ++n) {
            const float2 v = *reinterpret_cast<const float2*>(M + row * npad + base + 8 * n + 2 * fq);
            c[n][0] = v.x;
            c[n][1] = v.y;
        }
#pragma unroll
        for (int n = 0; n < 16; ++n) {
            double x0 = 0.0, x1 = 0.0;
            const double2 w = Ws[n * 32 + lane];
            dmma884(x0, x1, c2a(c[n][0], c[n][1], 0, fr, fq), w.x);
            dmma884(x0, x1, c2a(c[n][0], c[n][1], 1, fr, fq), w.y);
            const int col = 8 * n + 2 * fq;
            const float o0 = (float)x0, o1 = (float)x1;
            const float h0 = tf32_hi(o0), h1 = tf32_hi(o1);
            *reinterpret_cast<float2*>(M + row * npad + base + col) = make_float2(o0, o1);
            *reinterpret_cast<float2*>(Lhi + row * PW + col) = make_float2(h0, h1);
            *reinterpret_cast<float2*>(Llo + row * PW + col) = make_float2(o0 - h0, o1 - h1);
            if (n < 15) {
                const double xa0 = -c2a(x0, x1, 0, fr, fq), xa1 = -c2a(x0, x1, 1, fr, fq);
#pragma unroll
                for (int n2 = n + 1; n2 < 16; ++n2) {
                    const double2 b = Ls[tix(n2, n) * 32 + lane];
                    dmma884(c[n2][0], c[n2][1], xa0, b.x);
                    dmma884(c[n2][0], c[n2][1], xa1, b.y);
                }
            }
        }
    }
}

// ------------------------------------------------------- tensor-core update

struct SyrkBars {
    uint64_t full[STAGES], empty[STAGES], accfull[2], accempty[2];
};

// Staging slot cc of the C update in shared memory: one 128x32 box, 128
// rows of 128 bytes with the 128-byte swizzle (16-byte chunk j of row r at
// position j ^ (r mod 8)), the layout the TMA reduce reads.
__device__ __forceinline__ float4* c_chunk(unsigned char* cbuf, int cc, int r, int j)
{
    return reinterpret_cast<float4*>(cbuf + cc * BOX_BYTES + r * 128 + ((j ^ (r & 7)) << 4));
}

__global__ void __launch_bounds__(192, 1)
k_syrk_tc(const __grid_constant__ CUtensorMap map_hi, const __grid_constant__ CUtensorMap map_lo,
          const __grid_constant__ CUtensorMap map_c, int t0, int ntiles, int mode, unsigned* __restrict__ status)
{
    {
        uint32_t dyn;
        asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
        if (blockDim.x != 192 || dyn < (uint32_t)SYRK_SMEM) {
            if (threadIdx.x == 0) atomicOr(status, ST_LAUNCH);
            return;
        }
    }
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ SyrkBars bars;
    __shared__ uint32_t tmem_base_sh;
    __shared__ volatile int abort_flag;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t sbase = smem_u32(sm);
    unsigned char* cbuf = sm + STAGES * STAGE_BYTES;
    const uint32_t cbase = sbase + STAGES * STAGE_BYTES;
    if (tid == 0) {
        abort_flag = 0;
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(smem_u32(&bars.full[s]), 1);
            mbar_init(smem_u32(&bars.empty[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&bars.accfull[b]), 1);
            mbar_init(smem_u32(&bars.accempty[b]), 4);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                     "r"(256));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_sh;
    // launched as a programmatic dependent of the previous kernel on the
    // stream: the set-up above overlaps its tail; nothing below may read or
    // write what it produces before this wait (a no-op for a plain launch)
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;");

    if (warp == 0) {
        if (lane == 0) {
            // TMA producer of the four K chunks of A/B (hi and lo) per tile
            uint32_t g = 0;
            for (int t = blockIdx.x; t < ntiles && !abort_flag; t += gridDim.x) {
                int ti, tj;
                tile_of_mode(t, mode, ti, tj);
                const int ra = (t0 + ti) * PW, rb = (t0 + tj) * PW;
                for (int kc = 0; kc < NCHUNK; ++kc, ++g) {
                    const int s = g % STAGES;
                    if (!mbar_wait(smem_u32(&bars.empty[s]), ((g / STAGES) & 1) ^ 1, &abort_flag)) break;
                    const uint32_t st = sbase + s * STAGE_BYTES;
                    const uint32_t fb = smem_u32(&bars.full[s]);
                    mbar_expect_tx(fb, STAGE_BYTES);
                    tma_load_2d(st, &map_hi, kc * KC, ra, fb);
                    tma_load_2d(st + BOX_BYTES, &map_lo, kc * KC, ra, fb);
                    tma_load_2d(st + 2 * BOX_BYTES, &map_hi, kc * KC, rb, fb);
                    tma_load_2d(st + 3 * BOX_BYTES, &map_lo, kc * KC, rb, fb);
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // MMA issuer
            const uint32_t idesc = idesc_tf32_128x128();
            uint32_t g = 0, tl = 0;
            for (int t = blockIdx.x; t < ntiles && !abort_flag; t += gridDim.x, ++tl) {
                const uint32_t b = tl & 1;
                if (!mbar_wait(smem_u32(&bars.accempty[b]), ((tl >> 1) & 1) ^ 1, &abort_flag)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc = tmem + b * 128;
                bool ok = true;
                for (int kc = 0; kc < NCHUNK; ++kc, ++g) {
                    const int s = g % STAGES;
                    if (!mbar_wait(smem_u32(&bars.full[s]), (g / STAGES) & 1, &abort_flag)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t ah = sbase + s * STAGE_BYTES, al = ah + BOX_BYTES;
                    const uint32_t bh = ah + 2 * BOX_BYTES, bl = ah + 3 * BOX_BYTES;
#pragma unroll
                    for (int ks = 0; ks < KC / 8; ++ks) {
                        const uint32_t off = ks * 32;
                        umma_tf32(acc, umma_desc_sw128(ah + off), umma_desc_sw128(bh + off), idesc,
                                  (kc | ks) ? 1u : 0u);
                        umma_tf32(acc, umma_desc_sw128(ah + off), umma_desc_sw128(bl + off), idesc, 1u);
                        umma_tf32(acc, umma_desc_sw128(al + off), umma_desc_sw128(bh + off), idesc, 1u);
                    }
                    umma_commit(smem_u32(&bars.empty[s]));
                }
                if (!ok) break;
                umma_commit(smem_u32(&bars.accfull[b]));
            }
        }
    } else {
        // epilogue warps 2..5: TMEM lane quarter = warp % 4. C is never
        // loaded: each 128x32 box of -acc goes to shared memory and a TMA
        // reduce-add applies it in L2 (C - acc and C + (-acc) are the same
        // IEEE sum). On diagonal tiles the upper triangle (D, kept intact)
        // receives -0.0, which leaves every value as it is.
        const int quarter = warp & 3;
        const int rl = 32 * quarter + lane;   // row inside the tile
        uint32_t tl = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++tl) {
            int ti, tj;
            tile_of_mode(t, mode, ti, tj);
            const bool diag = ti == tj;
            const int ra = (t0 + ti) * PW, rb = (t0 + tj) * PW;
            const uint32_t b = tl & 1;
            // a time-out or abort seen by any epilogue thread stops all of
            // them before the next barrier
            if (epi_any(!mbar_wait(smem_u32(&bars.accfull[b]), (tl >> 1) & 1, &abort_flag))) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
            for (int cc = 0; cc < PW / 32; ++cc) {
                uint32_t v[32];
                const uint32_t taddr = tmem + b * 128 + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(32 * cc);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                    "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, "
                    "%31}, [%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                      "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                      "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                      "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (cc == PW / 32 - 1) {
                    // the accumulator is free once all its columns are read
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                    __syncwarp();
                    if (lane == 0) mbar_arrive(smem_u32(&bars.accempty[b]));
                }
                // the reduce that last used this ring slot must have read it
                if (tid == 64) bulk_wait_read_ring();
                epi_sync();
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int c = 32 * cc + 4 * j;   // column inside the tile
                    float4 d;
                    d.x = (!diag || c <= rl) ? -__uint_as_float(v[4 * j]) : -0.0f;
                    d.y = (!diag || c + 1 <= rl) ? -__uint_as_float(v[4 * j + 1]) : -0.0f;
                    d.z = (!diag || c + 2 <= rl) ? -__uint_as_float(v[4 * j + 2]) : -0.0f;
                    d.w = (!diag || c + 3 <= rl) ? -__uint_as_float(v[4 * j + 3]) : -0.0f;
                    *c_chunk(cbuf, cc % C_BOXES, rl, j) = d;
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                epi_sync();
                if (tid == 64) {
                    tma_reduce_add_2d(&map_c, cbase + (cc % C_BOXES) * BOX_BYTES, rb + cc * KC, ra);
                    bulk_commit();
                }
            }
        }
        if (tid == 64) bulk_wait0();
    }
    if (abort_flag && tid == 0) atomicOr(status, ST_TIMEOUT);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        __syncwarp();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256));
    }
}

// ---------------------------------------------------------------- host side

// row-major FP32 [rows][cols] buffer, boxes of 128 rows x 32 columns
static int make_panel_map(float* buf, int rows, CUtensorMap* map, int cols = PW)
{
    auto enc = get_encode();
    if (!enc) return fail(BDB_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    if (reinterpret_cast<uintptr_t>(buf) % 16) return fail(BDB_ERR_ARG, "panel buffer not 16-byte aligned");
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)cols * sizeof(float)};
    cuuint32_t box[2] = {KC, PW};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, buf, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(BDB_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    return BDB_OK;
}

// scratch layout in panel64: two panel buffers (hi, lo: FP32 [npad][128]
// each), then two FP64 128x128 blocks L_PP^T, for even and odd panels
static void panel_ptrs(bdb_system* s, int par, float** hi, float** lo, double** lkk)
{
    const size_t pan = (size_t)s->npad * PW;
    float* base = reinterpret_cast<float*>(s->panel64.p);
    *hi = base + (size_t)par * 2 * pan;
    *lo = *hi + pan;
    *lkk = reinterpret_cast<double*>(base + 4 * pan) + (size_t)par * PW * PW;
}

static int tc_setup(bdb_system* s)
{
    if (s->tc_map_ok) return BDB_OK;
    const size_t pan = (size_t)s->npad * PW;
    if (s->panel64.alloc(2 * pan + 2 * PW * PW + 64)) return BDB_ERR_NOMEM;
    BDB_CUDA(cudaMemset(s->panel64.p, 0, s->panel64.n * sizeof(double)));
    CUtensorMap* maps = reinterpret_cast<CUtensorMap*>(s->tc_map);   // hi0, lo0, hi1, lo1, M
    for (int par = 0; par < 2; ++par) {
        float *hi, *lo;
        double* lkk;
        panel_ptrs(s, par, &hi, &lo, &lkk);
        int rc = make_panel_map(hi, s->npad, &maps[2 * par]);
        if (rc) return rc;
        rc = make_panel_map(lo, s->npad, &maps[2 * par + 1]);
        if (rc) return rc;
    }
    int rc = make_panel_map(s->M32.p, s->npad, &maps[4], s->npad);
    if (rc) return rc;
    BDB_CUDA(cudaFuncSetAttribute(k_syrk_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, SYRK_SMEM));
    BDB_CUDA(cudaFuncSetAttribute(k_potrf128, cudaFuncAttributeMaxDynamicSharedMemorySize, POTRF_SMEM));
    BDB_CUDA(cudaFuncSetAttribute(k_trsm128, cudaFuncAttributeMaxDynamicSharedMemorySize, TRSM_SMEM));
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    s->sm_count = sms;
    s->tc_map_ok = true;
    return BDB_OK;
}

// k_syrk_tc as a programmatic dependent launch: its CTAs may start while the
// previous kernel on the stream drains and wait in griddepcontrol.wait.
static cudaError_t launch_syrk(bdb_system* s, int grid, cudaStream_t st, const CUtensorMap& hi, const CUtensorMap& lo,
                               const CUtensorMap& c, int t0, int ntiles, int mode)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(192);
    cfg.dynamicSmemBytes = SYRK_SMEM;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_syrk_tc, hi, lo, c, t0, ntiles, mode, s->status.p);
}

// Factorisation with one panel of look-ahead. For panel P the trailing
// update is split: block column P+1 first (main stream), then the FP64
// diagonal factorisation of block P+1 runs on the second stream on an SM
// that the persistent update of the remaining tiles leaves free; the panel
// solve of P+1 follows once both are done. Panel buffers alternate between
// even and odd panels so the two never share one.
int factor_mixed_tc(bdb_system* s)
{
    int rc = tc_setup(s);
    if (rc) return rc;
    const CUtensorMap* maps = reinterpret_cast<const CUtensorMap*>(s->tc_map);
    const int nt = s->npad / PW;
    cudaStream_t st = s->stream, st2 = s->stream2;
    float *hi, *lo;
    double* lkk;
    panel_ptrs(s, 0, &hi, &lo, &lkk);
    phase_mark_on(s, P_POTRF, st);
    k_potrf128<<<1, POTRF_THREADS, POTRF_SMEM, st>>>(s->M32.p, s->npad, 0, lkk, s->status.p);
    phase_mark_on(s, P_POTRF, st);
    s->launches += 1;
    for (int P = 0; P + 1 < nt; ++P) {
        const int par = P & 1;
        panel_ptrs(s, par, &hi, &lo, &lkk);
        const int units = (s->npad - (P + 1) * PW) / 8;
        const int per_cta = TRSM_THREADS / 32;
        phase_mark_on(s, P_TRSM, st);
        k_trsm128<<<std::min(s->sm_count, (units + per_cta - 1) / per_cta), TRSM_THREADS, TRSM_SMEM, st>>>(
            s->M32.p, s->npad, P, lkk, hi, lo, s->status.p);
        phase_mark_on(s, P_TRSM, st);
        const int rem = nt - P - 1;
        // block column P+1 of the trailing matrix
        phase_mark_on(s, P_SYRK_COL, st);
        BDB_CUDA(launch_syrk(s, std::min(s->sm_count, rem), st, maps[2 * par], maps[2 * par + 1], maps[4], P + 1, rem, 1));
        phase_mark_on(s, P_SYRK_COL, st);
        s->launches += 2;
        // diagonal block P+1 on the side stream, beside the rest of the update
        float *hi2, *lo2;
        double* lkk2;
        panel_ptrs(s, par ^ 1, &hi2, &lo2, &lkk2);
        BDB_CUDA(cudaEventRecord(s->la_ev[0], st));
        BDB_CUDA(cudaStreamWaitEvent(st2, s->la_ev[0], 0));
        phase_mark_on(s, P_POTRF, st2);
        k_potrf128<<<1, POTRF_THREADS, POTRF_SMEM, st2>>>(s->M32.p, s->npad, P + 1, lkk2, s->status.p);
        phase_mark_on(s, P_POTRF, st2);
        BDB_CUDA(cudaEventRecord(s->la_ev[1], st2));
        s->launches += 1;
        const int rest = rem * (rem + 1) / 2 - rem;
        if (rest > 0) {
            phase_mark_on(s, P_SYRK_REST, st);
            BDB_CUDA(launch_syrk(s, std::min(s->sm_count - 1, rest), st, maps[2 * par], maps[2 * par + 1], maps[4], P + 1,
                                 rest, 2));
            phase_mark_on(s, P_SYRK_REST, st);
            s->launches += 1;
        }
        BDB_CUDA(cudaStreamWaitEvent(st, s->la_ev[1], 0));
    }
    BDB_CUDA(cudaGetLastError());
    return BDB_OK;
}

}  // namespace bdb
