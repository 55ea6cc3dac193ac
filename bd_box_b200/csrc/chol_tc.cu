// Mixed-precision blocked Cholesky for sm_100a: FP64 panels, FP16-split
// trailing updates on the 5th-generation tensor cores (tcgen05), and the
// plain FP64 path's updates on the FP64 tensor instruction (DMMA).
//
// M is FP32 (lower triangle: the factor, upper: D, never written here) or
// FP64 on the FP64 path. Super-panel P covers columns p0 = 128P .. p0+127:
//   k_potrf128  one CTA factors the 128x128 diagonal block in FP64,
//               right-looking by 8 columns (each 8x8 pivot block factored and
//               inverted by the pivot warp while the other warps solve and
//               update), and
//               hands L_PP and the inverses W_kk of its 8x8 diagonal tiles on
//               to the panel solve;
//   k_trsm128   the rows below, X L_PP^T = A, by blocked forward substitution
//               in FP64 (one warp per 8 rows, DMMA); each row goes to M and,
//               on the mixed path, as an FP16 hi/lo pair of the row scaled
//               by a power of two (k_panel_scale) to two panel buffers;
//   k_syrk_tc   C -= L_i L_j^T for single 128x128 tiles and block columns
//               (the diagonal tile, the next two block columns), and
//   k_syrk_tc2  for 256x256 blocks on CTA pairs (the columns beyond), two
//               panels per pass over C, with
//               L_i L_j^T ~= (Lhi_i Lhi_j^T + Lhi_i Llo_j^T + Llo_i Lhi_j^T)
//                            / scale^2
//               (the dropped lo*lo term is ~2^-22 relative: FP32 accuracy);
//   k_syrk64    the FP64 path's updates on mma.sync.m8n8k4.f64.
//
// The update kernels are persistent and warp-specialised:
//   warp 0    TMA producer: per K chunk of 64 columns, four 128x64 FP16
//             boxes (A_hi, A_lo, B_hi, B_lo, 128-byte swizzle) into a
//             3-stage ring;
//   warp 1    MMA issuer: tcgen05.mma.kind::f16 (K=16), three per K step,
//             into one of two TMEM accumulators; tcgen05.commit frees a ring
//             stage / publishes an accumulator;
//   warps 2-5 epilogue: tcgen05.ld of the accumulator (warp w reads TMEM
//             lanes 32(w%4)..), hand the accumulator back, then
//             -acc / scale^2 per 128x32 box into a 2-box shared-memory ring
//             and a TMA reduce-add into C (lower triangle only on diagonal
//             tiles); C is never loaded.
// The epilogue of tile t overlaps the MMAs of tile t+1 and the loads of the
// tiles after it. Every mbarrier wait is bounded; a time-out sets
// ST_TIMEOUT and a shared abort flag that stops all roles, and the CTA frees
// its tensor memory before returning.
//
// Kernels are chained as programmatic dependents (griddepcontrol): each
// reads its inputs only after griddepcontrol.wait. Where the dependent is a
// small kernel of the panel chain, it is released early so that its launch
// overlaps; where it is a full grid (the next bulk update, the side
// stream's column update), only near the end, since its CTAs would hold the
// free SMs in their wait for as long as the releasing kernel runs.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cuda_fp16.h>

#include <algorithm>

#include "bdb_common.cuh"
#include "sm100.cuh"

namespace bdb {

static constexpr int PW = 128;                    // super-panel width = tile size
static constexpr int KC = 32;                     // FP32 columns of a box of the C update (128 B)
static constexpr int KCP = 64;                    // panel K columns per TMA box (128 B of FP16)
static constexpr int NCHUNK = PW / KCP;           // 2 boxes per panel
static constexpr int KSTEPS = KCP / 16;           // MMA k-steps per box (K = 16 for kind::f16)
static constexpr int STAGES = 3;
static constexpr int BOX_BYTES = PW * KC * 4;     // 16 KB: a C box, and a panel box (PW x KCP x 2 B)
static_assert(PW * KCP * 2 == BOX_BYTES, "panel and C boxes have the same size");
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

// instruction descriptor: D=F32, A=B=F16, both K-major, N=128, M=128
__host__ __device__ constexpr uint32_t idesc_f16_128x128()
{
    return (1u << 4) | (0u << 7) | (0u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
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
// mode 0 all tiles of the lower triangle, 1 only block column 0, 2 only
// block column 1, 3 block columns 2 and beyond, 4 block column 0 below its
// diagonal tile, 5 only block column 2
__device__ __forceinline__ void tile_of_mode(int t, int mode, int& ti, int& tj)
{
    if (mode == 5) {
        ti = t + 2;
        tj = 2;
    } else if (mode == 4) {
        ti = t + 1;
        tj = 0;
    } else if (mode == 1 || mode == 2) {
        tj = mode - 1;
        ti = t + tj;
    } else {
        tri_index(t, ti, tj);
        if (mode == 3) {
            ti += 2;
            tj += 2;
        }
    }
}

// the mixed path's panel operands: x = (hi + lo) / scale with hi and lo in
// FP16 (11 significant bits each, 22 together: the accuracy class of a
// TF32 hi/lo split, at twice the tensor rate and half the bytes). scale is
// a power of two chosen per factorisation from D's largest diagonal entry
// (|L_ij| <= sqrt(D_ii)), so that every entry stays in FP16's normal range
// where it matters; the products are unscaled exactly in the epilogue.
__device__ __forceinline__ void f16_split(float x, float scale, __half& hi, __half& lo)
{
    const float xs = x * scale;
    hi = __float2half_rn(xs);
    lo = __float2half_rn(xs - __half2float(hi));
}

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

// 1/x for x > 0 in FP64: the hardware's FP64 reciprocal estimate (no
// conversions on the pivot chain) refined by one Newton-Raphson step
// q <- q + q (1 - x q), which squares its relative error.
__device__ __forceinline__ double rcp_nr(double x)
{
    double q;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(q) : "d"(x));
    return fma(q, fma(-x, q, 1.0), q);
}

// Factor the 8x8 block in Dg ([8][9], lower triangle) in registers and
// invert the factor; every lane of the pivot warp runs the whole
// factorisation (nothing passes between lanes), lane c (c < 8) returns
// column c of L_kk and of W_kk = L_kk^-1. The elimination runs on the
// unscaled Schur complements with q_j = 1/a_jj: the next pivot
// a_{j+1,j+1} -= a_{j+1,j}^2 q_j first (the square is formed while q_j is
// computed, so one reciprocal and one FMA separate two pivots), then the
// other entries as a_ic -= a_ij (a_cj q_j), one FMA each after the 7-j
// scaled column entries. The columns are scaled by r_j = 1/sqrt(a_jj) at
// the end, and column c of W follows by right-looking forward
// substitution: w_m = acc_m r_m, then acc_i -= L_im w_m for i > m. It is
// one straight-line block, so the substitution fills the latency of the
// reciprocal chain. With kFull (the plain FP64 path) every reciprocal and
// reciprocal square root takes a second Newton step, which brings it to
// FP64 rounding.
template <bool kFull>
__device__ __forceinline__ bool pivot8_inv(const double* Dg, int c, double (&lcol)[8], double (&wcol)[8])
{
    double a[8][8];
    bool ok = true;
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int k = 0; k <= r; ++k) a[r][k] = Dg[r * 9 + k];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        if (!(a[j][j] > 0.0)) ok = false;
        double q = rcp_nr(a[j][j]);
        if (kFull) q = fma(q, fma(-a[j][j], q, 1.0), q);
        if (j + 1 < 8) a[j + 1][j + 1] = fma(-(a[j + 1][j] * a[j + 1][j]), q, a[j + 1][j + 1]);
        double t[8];
#pragma unroll
        for (int k = j + 1; k < 8; ++k) t[k] = a[k][j] * q;
#pragma unroll
        for (int r = j + 1; r < 8; ++r)
#pragma unroll
            for (int k = j + 1; k <= r; ++k)
                if (r != j + 1) a[r][k] = fma(-a[r][j], t[k], a[r][k]);
    }
    double rj[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        double r = rsqrt_nr(a[j][j]);
        if (kFull) r = r * (1.5 - 0.5 * a[j][j] * r * r);
        rj[j] = r;
#pragma unroll
        for (int i = j; i < 8; ++i) a[i][j] *= r;
    }
    double acc[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) acc[i] = i == c ? 1.0 : 0.0;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        wcol[m] = m >= c ? acc[m] * rj[m] : 0.0;
#pragma unroll
        for (int i = m + 1; i < 8; ++i) acc[i] = fma(-a[i][m], wcol[m], acc[i]);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        double l = 0.0;
#pragma unroll
        for (int k = 0; k <= i; ++k)
            if (k == c) l = a[i][k];
        lcol[i] = l;
    }
    return ok;
}

// two consecutive elements of an FP32 or FP64 matrix as doubles, and back
__device__ __forceinline__ double2 ld_pair(const float* p)
{
    const float2 v = *reinterpret_cast<const float2*>(p);
    return make_double2(v.x, v.y);
}
__device__ __forceinline__ double2 ld_pair(const double* p) { return *reinterpret_cast<const double2*>(p); }
__device__ __forceinline__ void st_pair(float* p, double a, double b)
{
    *reinterpret_cast<float2*>(p) = make_float2((float)a, (float)b);
}
__device__ __forceinline__ void st_pair(double* p, double a, double b)
{
    *reinterpret_cast<double2*>(p) = make_double2(a, b);
}

static constexpr int POTRF_THREADS = 512;
static constexpr int NT = PW / 8;                  // 16 row groups of 8 rows
static constexpr int NTILE = NT * (NT + 1) / 2;    // 136 tiles in the lower triangle
// Lt tiles, W_kk, the 8x8 block being factored [8][9], 1/L_jj, and one
// hand-over slot of two tiles per step
static constexpr int POTRF_SMEM = (NTILE * 64 + NT * 64 + 80 + NT * 128) * 8;
// factor hand-off to the panel solve: L_PP tiles then the W_kk, A order
static constexpr int PANEL_FAC = (NTILE + NT) * 64;

// row group owned by a warp: warp 0 runs the pivots; warps 4, 8, 12 share
// its scheduler (warp w issues on sub-partition w mod 4) and own the row
// groups with the least work (1, 2, 3); the other 12 warps own 4..15
__device__ __forceinline__ int row_group_of(int warp)
{
    return (warp & 3) ? 4 + warp - 1 - (warp >> 2) : warp >> 2;
}

// per-step mbarriers of k_potrf128, each completing exactly once
struct PotrfBars {
    uint64_t w[NT];      // W_kk and L_kk published by the pivot warp (32 arrivals)
    uint64_t lcol[NT];   // every tile of block column k solved (32 per solving warp)
    uint64_t hand[NT];   // row group k+2's last two tiles and L[k+2][k] handed over (32 arrivals)
};

// all 32 lanes wait; false on a time-out or an abort seen by this lane
__device__ __forceinline__ bool bar_wait0(uint64_t* b, volatile int* abort_flag, uint32_t limit)
{
    return mbar_wait(smem_u32(b), 0, abort_flag, limit);
}

// A solved off-diagonal tile X (C fragments x0, x1 of lane (fr, fq)) of
// L_PP, tile index t = tix(g, n): to the shared tiles (A order), to the FP64
// hand-off for the panel solve (the same order) and, in M's precision, to M
template <typename T>
__device__ __forceinline__ void put_tile(double* Lt, double* Wt, T* M, size_t row0, size_t col0, int npad, int t,
                                         int fr, int fq, double x0, double x1)
{
    const int p0 = t * 64 + apos(fr, 2 * fq), p1 = t * 64 + apos(fr, 2 * fq + 1);
    Lt[p0] = x0;
    Lt[p1] = x1;
    Wt[p0] = x0;
    Wt[p1] = x1;
    st_pair(M + (row0 + fr) * npad + col0 + 2 * fq, x0, x1);
}

// X = C W^T for an 8x8 tile C held as C fragments (c0, c1) and W in A order
// (pairs at 2 lane): two DMMAs, the A fragments of C by shuffles
__device__ __forceinline__ void solve_tile(double c0, double c1, const double* Wk, int lane, int fr, int fq,
                                           double& x0, double& x1)
{
    x0 = 0.0;
    x1 = 0.0;
    const double2 wb = *reinterpret_cast<const double2*>(Wk + 2 * lane);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int src = (fr << 2) + 2 * h + (fq >> 1);
        const double v0 = __shfl_sync(0xffffffffu, c0, src);
        const double v1 = __shfl_sync(0xffffffffu, c1, src);
        dmma884(x0, x1, (fq & 1) ? v1 : v0, h ? wb.y : wb.x);
    }
}

// FP64 factorisation L_PP of the 128x128 diagonal block (P, P) and the
// inverses W_kk of its 8x8 diagonal tiles, right-looking over 16 blocks of 8
// columns with the trailing matrix in registers: the warp owning row group g
// keeps its tiles (g, n), n <= g, as DMMA accumulators. No CTA-wide barrier
// orders the steps; per-step mbarriers carry exactly what each warp needs:
//   pivot warp, step k: factor tile (k, k) and invert it (pivot8_inv, every
//     lane the whole factorisation) -> publish W_kk; take row group k+1's last two tiles
//     (k+1, k) and (k+1, k+1), handed over through column k-2 together with
//     L[k+1][k-1], and apply column k-1 to them; solve L[k+1][k] = C[k+1][k]
//     W_kk^T -> publish; update tile (k+1, k+1) with it and go on to pivot
//     k+1;
//   owner g, step k < g-1: solve L[g][k] = C[g][k] W_kk^T -> publish; for
//     k < g-2 update tiles n = k+1..g with column k once all of block column
//     k is solved and step k's hand-over is made; at k = g-2 hand the tiles
//     (g, g-1), (g, g) over instead and retire.
// So the pivot chain waits only for one solve of row group k+2, made while
// the pivot warp factors and inverts the next block, and the bulk updates
// of a step start after that hand-over, so that they do not stand in front
// of it on the FP64 pipes (four warps share each). Each solved tile goes to M (FP32) and
// to the FP64 hand-off Wt for the panel solve (A order: the 136 L_PP tiles,
// then the 16 W_kk; PANEL_FAC doubles) as soon as it is final, so nothing
// is left to store at the end. Every wait is bounded: a time-out sets
// ST_TIMEOUT and every warp runs out to the final barrier.
template <typename T>
__global__ void __launch_bounds__(POTRF_THREADS, 1) k_potrf128(T* __restrict__ M, int npad, int P,
                                                            double* __restrict__ Wt, unsigned* __restrict__ status,
                                                            uint32_t wlim)
{
    extern __shared__ double sh[];
    double* Lt = sh;                       // [NTILE][64] A order
    double* Wa = Lt + NTILE * 64;          // [NT][64] W_kk in A order
    double* Dg = Wa + NT * 64;             // [8][9] diagonal block being factored
    double* Hd = Dg + 80;                  // [NT][2][64] hand-over slots (C layout)
    __shared__ PotrfBars bars;
    __shared__ int bad;
    __shared__ volatile int abort_flag;
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
    if (tid < NT) {
        mbar_init(smem_u32(&bars.w[tid]), 32);
        // solvers of block column k: the pivot warp (row group k+1) and the
        // owners of row groups k+2..15
        mbar_init(smem_u32(&bars.lcol[tid]), 32 * (tid < NT - 1 ? NT - 1 - tid : 1));
        mbar_init(smem_u32(&bars.hand[tid]), 32);
    }
    if (tid == 0) {
        bad = 0;
        abort_flag = 0;
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    __syncthreads();
    // launched as a programmatic dependent of the update of this block
    // column: the set-up above overlaps its tail, M is read only after it
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (warp == 0) {
        // ---------------------------------------------------- pivot warp
        // tile (0, 0) to Dg; tiles (1, 0) and (1, 1) (nothing updates them
        // before step 0) as C fragments
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int c = 2 * fq + e;
            Dg[fr * 9 + c] = c <= fr ? (double)M[(base + fr) * npad + base + c] : 0.0;
        }
        double t1[2], t2[2];
        {
            const double2 a = ld_pair(M + (base + 8 + fr) * npad + base + 2 * fq);
            const double2 b = ld_pair(M + (base + 8 + fr) * npad + base + 8 + 2 * fq);
            t1[0] = a.x;
            t1[1] = a.y;
            t2[0] = 2 * fq <= fr ? (double)b.x : 0.0;
            t2[1] = 2 * fq + 1 <= fr ? (double)b.y : 0.0;
        }
        for (int k = 0; k < NT; ++k) {
            // the dependent (block row P+1's solve, 4 CTAs) launches for the
            // last four steps only: launched at the start, its CTAs held 4
            // SMs in their wait for the whole factorisation
            if (k == NT - 4) asm volatile("griddepcontrol.launch_dependents;");
            __syncwarp();
            {
                double lc[8], wc[8];
                if (!pivot8_inv<sizeof(T) == 8>(Dg, lane & 7, lc, wc) && lane == 0) bad = 1;
                if (lane < 8) {
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const int pa = apos(i, lane);
                        Wa[k * 64 + pa] = wc[i];
                        Lt[tix(k, k) * 64 + pa] = lc[i];
                    }
                }
            }
            mbar_arrive(smem_u32(&bars.w[k]));   // release: this lane's writes
            if (k + 1 == NT) break;
            __syncwarp();
            if (k > 0) {
                // tiles (k+1, k) and (k+1, k+1) through column k-2 and
                // L[k+1][k-1] from their owner; column k-1 applied here
                if (!bar_wait0(&bars.hand[k - 1], &abort_flag, wlim)) break;
                const double2 a = *reinterpret_cast<const double2*>(Hd + (size_t)(k - 1) * 128 + 2 * lane);
                const double2 b = *reinterpret_cast<const double2*>(Hd + (size_t)(k - 1) * 128 + 64 + 2 * lane);
                const double2 u = *reinterpret_cast<const double2*>(Lt + tix(k + 1, k - 1) * 64 + 2 * lane);
                const double2 v = *reinterpret_cast<const double2*>(Lt + tix(k, k - 1) * 64 + 2 * lane);
                t1[0] = a.x;
                t1[1] = a.y;
                t2[0] = b.x;
                t2[1] = b.y;
                dmma884(t1[0], t1[1], -u.x, v.x);
                dmma884(t1[0], t1[1], -u.y, v.y);
                dmma884(t2[0], t2[1], -u.x, u.x);
                dmma884(t2[0], t2[1], -u.y, u.y);
            }
            // L[k+1][k] = C[k+1][k] W_kk^T
            double x0, x1;
            solve_tile(t1[0], t1[1], Wa + k * 64, lane, fr, fq, x0, x1);
            Lt[tix(k + 1, k) * 64 + apos(fr, 2 * fq)] = x0;
            Lt[tix(k + 1, k) * 64 + apos(fr, 2 * fq + 1)] = x1;
            __syncwarp();
            mbar_arrive(smem_u32(&bars.lcol[k]));
            // tile (k+1, k+1) -= L[k+1][k] L[k+1][k]^T: the next pivot block
            const double2 av = *reinterpret_cast<const double2*>(Lt + tix(k + 1, k) * 64 + 2 * lane);
            double e0 = t2[0], e1 = t2[1];
            dmma884(e0, e1, -av.x, av.x);
            dmma884(e0, e1, -av.y, av.y);
            Dg[fr * 9 + 2 * fq] = e0;
            Dg[fr * 9 + 2 * fq + 1] = e1;
        }
    } else if (g == 1) {
        // ------------------------------------------------------ store warp
        // (row group 1 needs no owner: the pivot warp takes its tiles). It
        // copies the pivot warp's results to global memory off the pivot
        // chain: L_kk and W_kk once published, L[k+1][k] once block column k
        // is solved; FP64 in A order to Wt, L as FP32 to M
        for (int k = 0; k < NT; ++k) {
            if (!bar_wait0(&bars.w[k], &abort_flag, wlim)) break;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int p = 2 * lane + h, r = p >> 3, c = ((p & 1) << 2) | ((p & 7) >> 1);
                const double l = Lt[tix(k, k) * 64 + p];
                Wt[tix(k, k) * 64 + p] = l;
                Wt[(NTILE + k) * 64 + p] = Wa[k * 64 + p];
                if (c <= r) M[(base + 8 * k + r) * npad + base + 8 * k + c] = (T)l;
            }
            if (k + 1 == NT) break;
            if (!bar_wait0(&bars.lcol[k], &abort_flag, wlim)) break;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int p = 2 * lane + h, r = p >> 3, c = ((p & 1) << 2) | ((p & 7) >> 1);
                const double l = Lt[tix(k + 1, k) * 64 + p];
                Wt[tix(k + 1, k) * 64 + p] = l;
                M[(base + 8 * (k + 1) + r) * npad + base + 8 * k + c] = (T)l;
            }
        }
    } else {
        // -------------------------------------------------- tile owners
        double cacc[NT][2];
#pragma unroll
        for (int n = 0; n < NT; ++n) {
            cacc[n][0] = cacc[n][1] = 0.0;
            if (n <= g) {
                const double2 v = ld_pair(M + (base + 8 * g + fr) * npad + base + 8 * n + 2 * fq);
                cacc[n][0] = (n < g || 2 * fq <= fr) ? v.x : 0.0;
                cacc[n][1] = (n < g || 2 * fq + 1 <= fr) ? v.y : 0.0;
            }
        }
        for (int k = 0; k + 1 < g; ++k) {
            if (!bar_wait0(&bars.w[k], &abort_flag, wlim)) break;
            // L[g][k] = C[g][k] W_kk^T
            double c0 = 0.0, c1 = 0.0;
#pragma unroll
            for (int t = 0; t < NT; ++t)
                if (t == k) {
                    c0 = cacc[t][0];
                    c1 = cacc[t][1];
                }
            double x0, x1;
            solve_tile(c0, c1, Wa + k * 64, lane, fr, fq, x0, x1);
            put_tile(Lt, Wt, M, base + 8 * g, base + 8 * k, npad, tix(g, k), fr, fq, x0, x1);
            if (k + 2 == g) {
                // the last two tiles, (g, g-1) and (g, g), through column
                // k-1, for the pivot warp
#pragma unroll
                for (int t = 0; t < NT; ++t) {
                    if (t == g - 1)
                        *reinterpret_cast<double2*>(Hd + (size_t)k * 128 + 2 * lane) =
                            make_double2(cacc[t][0], cacc[t][1]);
                    if (t == g)
                        *reinterpret_cast<double2*>(Hd + (size_t)k * 128 + 64 + 2 * lane) =
                            make_double2(cacc[t][0], cacc[t][1]);
                }
                __syncwarp();
                mbar_arrive(smem_u32(&bars.lcol[k]));
                mbar_arrive(smem_u32(&bars.hand[k]));
                break;
            }
            __syncwarp();
            mbar_arrive(smem_u32(&bars.lcol[k]));
            const double2 av = *reinterpret_cast<const double2*>(Lt + tix(g, k) * 64 + 2 * lane);
            // the bulk updates of step k wait for its hand-over, so that the
            // solve on the pivot chain does not queue behind them
            if (!bar_wait0(&bars.hand[k], &abort_flag, wlim) || !bar_wait0(&bars.lcol[k], &abort_flag, wlim)) break;
            // C[g][n] -= L[g][k] L[n][k]^T for n = k+1..g, four tiles per
            // batch: their operand loads first (predicated, no branch), then
            // the MMAs
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
        }
    }
    __syncthreads();
    if (tid == 0) {
        if (bad) atomicOr(status, ST_NOT_SPD);
        if (abort_flag) atomicOr(status, ST_TIMEOUT);
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
// Writes the rows to M and, for the mixed path (T = float), their FP16
// split L s = hi + lo (f16_split, s = pscale[0]) to the panel buffers; for
// the FP64 path (T = double) the rows in FP64 to one panel buffer (Lhi, as
// doubles; Llo unused).
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

template <typename T>
__global__ void __launch_bounds__(TRSM_THREADS, 1) k_trsm128(T* __restrict__ M, int npad, int P, int unit0, int units,
                                                          const double* __restrict__ Lf, float* __restrict__ Lhi,
                                                          float* __restrict__ Llo, unsigned* __restrict__ status,
                                                          const float* __restrict__ pscale)
{
    {
        uint32_t dyn;
        asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
        if (blockDim.x != TRSM_THREADS || dyn < (uint32_t)TRSM_SMEM) {
            if (threadIdx.x == 0) atomicOr(status, ST_LAUNCH);
            return;
        }
    }
    // block row P+1 (unit0 = 0) releases its dependent, the chain's one-CTA
    // update, at once; the rows below only as their warps finish, because
    // theirs is the side stream's column update, a grid that would
    // otherwise wait on the free SMs the chain needs while this runs
    if (unit0 == 0) asm volatile("griddepcontrol.launch_dependents;");
    extern __shared__ double sh[];
    const double2* Ls = reinterpret_cast<const double2*>(sh);               // [NTILE][32] pairs
    const double2* Ws = reinterpret_cast<const double2*>(sh + NTILE * 64);  // [NT][32] pairs
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int fr = lane >> 2, fq = lane & 3;
    const size_t base = (size_t)P * PW;
    // units unit0 .. unit0 + units - 1 of 8 rows below the block
    const size_t row0 = base + PW + (size_t)8 * unit0;
    // block row P+1 is launched as a programmatic dependent of the diagonal
    // block's factorisation (a no-op wait for the rows below, a plain
    // launch): nothing is read before this
    asm volatile("griddepcontrol.wait;" ::: "memory");
    {
        // the factor, by asynchronous 16-byte copies (no register staging)
        const char* src = reinterpret_cast<const char*>(Lf);
        const uint32_t dst = smem_u32(sh);
        for (int f = tid; f < PANEL_FAC / 2; f += TRSM_THREADS)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst + 16 * f), "l"(src + 16 * (size_t)f)
                         : "memory");
        asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    const int slot = (warp >> 2) * 4 * gridDim.x + blockIdx.x * 4 + (warp & 3);
    for (int u = slot; u < units; u += TRSM_THREADS / 32 * gridDim.x) {
        const size_t row = row0 + (size_t)8 * u + fr;
        double c[16][2];
#pragma unroll
        for (int n = 0; n < 16; ++n) {
            const double2 v = ld_pair(M + row * npad + base + 8 * n + 2 * fq);
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
            if constexpr (sizeof(T) == 4) {
                const float o0 = (float)x0, o1 = (float)x1;
                *reinterpret_cast<float2*>(M + row * npad + base + col) = make_float2(o0, o1);
                __half2 h, l;
                f16_split(o0, pscale[0], h.x, l.x);
                f16_split(o1, pscale[0], h.y, l.y);
                *reinterpret_cast<__half2*>(reinterpret_cast<__half*>(Lhi) + row * PW + col) = h;
                *reinterpret_cast<__half2*>(reinterpret_cast<__half*>(Llo) + row * PW + col) = l;
            } else {
                st_pair(M + row * npad + base + col, x0, x1);
                // the FP64 panel in k_syrk64's fragment order: within each
                // group of 8 columns, column c at 2 (c mod 4) + (c / 4 mod 2)
                double* pr = reinterpret_cast<double*>(Lhi) + row * PW + 8 * n;
                pr[(((2 * fq) & 3) << 1) | (fq >> 1)] = x0;
                pr[(((2 * fq + 1) & 3) << 1) | (fq >> 1)] = x1;
            }
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
    asm volatile("griddepcontrol.launch_dependents;");
}

// ------------------------------------------------------- tensor-core update

struct SyrkBars {
    uint64_t full[STAGES], empty[STAGES], accfull[2], accempty[2], drain;
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
          const __grid_constant__ CUtensorMap map_c, int t0, int ntiles, int mode, unsigned* __restrict__ status,
          uint32_t wlim, const float* __restrict__ pscale)
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
        mbar_init(smem_u32(&bars.drain), 1);
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
    // The chain's and the side stream's updates (modes 1 and 4) let their
    // dependents launch at once (a one-CTA factorisation; a plain launch).
    // A bulk update's dependent is the next bulk update, a full grid of CTAs
    // that, launched early, would sit on every free SM in its
    // griddepcontrol.wait for as long as this launch runs, SMs the chain
    // needs meanwhile: bulk updates release it only once their last loads
    // are issued (below).
    if (mode == 1 || mode == 4) asm volatile("griddepcontrol.launch_dependents;");

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
                    if (!mbar_wait(smem_u32(&bars.empty[s]), ((g / STAGES) & 1) ^ 1, &abort_flag, wlim)) break;
                    const uint32_t st = sbase + s * STAGE_BYTES;
                    const uint32_t fb = smem_u32(&bars.full[s]);
                    mbar_expect_tx(fb, STAGE_BYTES);
                    tma_load_2d(st, &map_hi, kc * KCP, ra, fb);
                    tma_load_2d(st + BOX_BYTES, &map_lo, kc * KCP, ra, fb);
                    tma_load_2d(st + 2 * BOX_BYTES, &map_hi, kc * KCP, rb, fb);
                    tma_load_2d(st + 3 * BOX_BYTES, &map_lo, kc * KCP, rb, fb);
                }
            }
            if (mode != 1 && mode != 4) asm volatile("griddepcontrol.launch_dependents;");
            if (abort_flag) {
                // the loads still in flight (the last fill of each stage)
                // must land before the CTA exits
                volatile int never = 0;
                for (uint32_t j = g > (uint32_t)STAGES ? g - STAGES : 0; j < g; ++j)
                    mbar_wait(smem_u32(&bars.full[j % STAGES]), (j / STAGES) & 1, &never);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // MMA issuer
            const uint32_t idesc = idesc_f16_128x128();
            uint32_t g = 0, tl = 0;
            for (int t = blockIdx.x; t < ntiles && !abort_flag; t += gridDim.x, ++tl) {
                const uint32_t b = tl & 1;
                if (!mbar_wait(smem_u32(&bars.accempty[b]), ((tl >> 1) & 1) ^ 1, &abort_flag, wlim)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc = tmem + b * 128;
                bool ok = true;
                for (int kc = 0; kc < NCHUNK; ++kc, ++g) {
                    const int s = g % STAGES;
                    if (!mbar_wait(smem_u32(&bars.full[s]), (g / STAGES) & 1, &abort_flag, wlim)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t ah = sbase + s * STAGE_BYTES, al = ah + BOX_BYTES;
                    const uint32_t bh = ah + 2 * BOX_BYTES, bl = ah + 3 * BOX_BYTES;
#pragma unroll
                    for (int ks = 0; ks < KSTEPS; ++ks) {
                        const uint32_t off = ks * 32;   // 16 FP16 of K
                        umma_f16(acc, umma_desc_sw128(ah + off), umma_desc_sw128(bh + off), idesc,
                                 (kc | ks) ? 1u : 0u);
                        umma_f16(acc, umma_desc_sw128(ah + off), umma_desc_sw128(bl + off), idesc, 1u);
                        umma_f16(acc, umma_desc_sw128(al + off), umma_desc_sw128(bh + off), idesc, 1u);
                    }
                    umma_commit(smem_u32(&bars.empty[s]));
                }
                if (!ok) break;
                umma_commit(smem_u32(&bars.accfull[b]));
            }
            if (abort_flag) {
                // every MMA issued so far completes before the tensor
                // memory is freed: commit once more and wait for it
                volatile int never = 0;
                umma_commit(smem_u32(&bars.drain));
                mbar_wait(smem_u32(&bars.drain), 0, &never);
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
        const float is2 = pscale[1];         // 1 / scale^2: the panels' FP16 scaling undone, exactly
        uint32_t tl = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++tl) {
            int ti, tj;
            tile_of_mode(t, mode, ti, tj);
            const bool diag = ti == tj;
            const int ra = (t0 + ti) * PW, rb = (t0 + tj) * PW;
            const uint32_t b = tl & 1;
            // a time-out or abort seen by any epilogue thread stops all of
            // them before the next barrier
            if (epi_any(!mbar_wait(smem_u32(&bars.accfull[b]), (tl >> 1) & 1, &abort_flag, wlim))) break;
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
                    d.x = (!diag || c <= rl) ? -is2 * __uint_as_float(v[4 * j]) : -0.0f;
                    d.y = (!diag || c + 1 <= rl) ? -is2 * __uint_as_float(v[4 * j + 1]) : -0.0f;
                    d.z = (!diag || c + 2 <= rl) ? -is2 * __uint_as_float(v[4 * j + 2]) : -0.0f;
                    d.w = (!diag || c + 3 <= rl) ? -is2 * __uint_as_float(v[4 * j + 3]) : -0.0f;
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

// ------------------------------------------- 2-SM tensor-core bulk update
//
// Block columns 2 and beyond of the trailing update (mode 3, most of the
// factorisation's work) on CTA pairs: a cluster of two CTAs computes a
// 256x256 block (2x2 tiles) of -L_i L_j^T with tcgen05.mma.cta_group::2,
// M = N = 256. CTA r of the pair stages the 128 rows of tile row 2I+r (its
// half of A) and of tile column 2J+r (its half of B) in the same ring as the
// 1-SM kernel, so each SM pulls the same 64 KB per K chunk from L2 for twice
// the MMA work: the operand feed that bounds the 1-SM kernel is halved.
// CTA r's tensor memory holds its 128 rows x 256 columns of the block, two
// buffers (all 512 columns). Protocol: the leader (rank 0) owns the full
// barriers (it expects both CTAs' bytes; each CTA's loads complete on the
// leader's barrier) and the accumulator-empty barriers (both CTAs' epilogue
// warps arrive there); its single MMA thread commits stage release and
// accumulator-full to both CTAs at once. Every wait is bounded; a time-out in
// either CTA stops both. With npan = 2 the block takes the updates of two
// panels at once (K = 256: the second panel's maps continue the K loop), so
// C is read and written once for both.
__host__ __device__ constexpr uint32_t idesc_f16_256x256()
{
    return (1u << 4) | (0u << 7) | (0u << 10) | ((256u >> 3) << 17) | ((256u >> 4) << 24);
}

__device__ __forceinline__ void umma_f16_pair(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                              uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// arrive once on the barrier at offset `bar` of both CTAs of the pair when
// this thread's MMAs so far have completed
__device__ __forceinline__ void umma_commit_pair(uint32_t bar)
{
    asm volatile(
        "{\n\t.reg .b16 m;\n\tmov.b16 m, 3;\n\t"
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], m;\n\t}" ::"r"(
            bar)
        : "memory");
}

// shared::cluster address of `addr` (a shared::cta address of this CTA) in
// CTA `rank` of the cluster
__device__ __forceinline__ uint32_t cluster_addr(uint32_t addr, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}

__device__ __forceinline__ void cluster_sync_all()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// 2-D load into this CTA's shared memory whose completion is counted on the
// pair leader's barrier (cluster address `bar`); the data lands in this
// CTA's shared memory only
__device__ __forceinline__ void tma_load_2d_pair(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

struct PairBars {
    uint64_t full[STAGES], empty[STAGES], accfull[2], accempty[2], drain;
};

// block t of the lower triangle of 256-wide blocks over the trailing tile
// columns c0 .. cols-1 -> tile row and column of its top-left tile
__device__ __forceinline__ void pair_block(int t, int c0, int& ti, int& tj)
{
    int bi, bj;
    tri_index(t, bi, bj);
    ti = c0 + 2 * bi;
    tj = c0 + 2 * bj;
}

__global__ void __launch_bounds__(192, 1)
k_syrk_tc2(const __grid_constant__ CUtensorMap map_hi, const __grid_constant__ CUtensorMap map_lo,
           const __grid_constant__ CUtensorMap map_hi2, const __grid_constant__ CUtensorMap map_lo2,
           const __grid_constant__ CUtensorMap map_c, int t0, int c0, int cols, int npan, unsigned* __restrict__ status,
           uint32_t wlim, const float* __restrict__ pscale)
{
    {
        uint32_t dyn, ncta;
        asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
        asm("mov.u32 %0, %%cluster_nctarank;" : "=r"(ncta));
        if (blockDim.x != 192 || dyn < (uint32_t)SYRK_SMEM || ncta != 2 || npan < 1 || npan > 2) {
            if (threadIdx.x == 0) atomicOr(status, ST_LAUNCH);
            return;
        }
    }
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ PairBars bars;
    __shared__ uint32_t tmem_base_sh;
    __shared__ volatile int abort_flag;
    uint32_t rank, cid, ncl;
    asm("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
    asm("mov.u32 %0, %%clusterid.x;" : "=r"(cid));
    asm("mov.u32 %0, %%nclusterid.x;" : "=r"(ncl));
    const bool leader = rank == 0;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t sbase = smem_u32(sm);
    unsigned char* cbuf = sm + STAGES * STAGE_BYTES;
    const uint32_t cbase = sbase + STAGES * STAGE_BYTES;
    // the other CTA's abort flag: a time-out here stops the pair
    const uint32_t peer_abort = cluster_addr(smem_u32((const void*)&abort_flag), rank ^ 1u);
    auto stop_pair = [&]() {
        abort_flag = 1;
        asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(peer_abort), "r"(1) : "memory");
    };
    if (tid == 0) {
        abort_flag = 0;
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(smem_u32(&bars.full[s]), 1);
            mbar_init(smem_u32(&bars.empty[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&bars.accfull[b]), 1);
            mbar_init(smem_u32(&bars.accempty[b]), 8);   // 4 epilogue warps x 2 CTAs
        }
        mbar_init(smem_u32(&bars.drain), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    // both CTAs' barriers are initialised (and their flags cleared) before
    // either signals the other's
    cluster_sync_all();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_sh;
    // a bulk update: its dependent (the next bulk update) is released only
    // once this CTA's last loads are issued, so that its CTAs do not wait on
    // SMs the chain needs for as long as this launch runs
    asm volatile("griddepcontrol.wait;" ::: "memory");

    const int nb = (cols - c0 + 1) / 2;   // 256-wide block columns
    const int nblocks = nb * (nb + 1) / 2;
    const int nchunk = NCHUNK * npan;     // K chunks of a block
    if (warp == 0) {
        if (lane == 0) {
            // TMA producer: this CTA's half of A (tile row ti + rank) and of B
            // (tile column tj + rank); rows past the matrix read as zeros
            uint32_t g = 0;
            const uint32_t full0 = cluster_addr(smem_u32(&bars.full[0]), 0);
            for (int t = cid; t < nblocks && !abort_flag; t += ncl) {
                int ti, tj;
                pair_block(t, c0, ti, tj);
                const int ra = (t0 + ti + (int)rank) * PW, rb = (t0 + tj + (int)rank) * PW;
                bool ok = true;
                for (int kc = 0; kc < nchunk; ++kc, ++g) {
                    const int s = g % STAGES;
                    if (!mbar_wait(smem_u32(&bars.empty[s]), ((g / STAGES) & 1) ^ 1, &abort_flag, wlim)) {
                        ok = false;
                        break;
                    }
                    const uint32_t st = sbase + s * STAGE_BYTES;
                    const uint32_t fb = full0 + s * sizeof(uint64_t);
                    const CUtensorMap* mh = kc < NCHUNK ? &map_hi : &map_hi2;
                    const CUtensorMap* ml = kc < NCHUNK ? &map_lo : &map_lo2;
                    const int x = (kc % NCHUNK) * KCP;
                    if (leader) mbar_expect_tx(smem_u32(&bars.full[s]), 2 * STAGE_BYTES);
                    tma_load_2d_pair(st, mh, x, ra, fb);
                    tma_load_2d_pair(st + BOX_BYTES, ml, x, ra, fb);
                    tma_load_2d_pair(st + 2 * BOX_BYTES, mh, x, rb, fb);
                    tma_load_2d_pair(st + 3 * BOX_BYTES, ml, x, rb, fb);
                }
                if (!ok) {
                    stop_pair();
                    break;
                }
            }
            asm volatile("griddepcontrol.launch_dependents;");
            if (abort_flag && leader) {
                // the loads still in flight (the last fill of each stage, both
                // CTAs' bytes) land before the pair exits
                volatile int never = 0;
                for (uint32_t j = g > (uint32_t)STAGES ? g - STAGES : 0; j < g; ++j)
                    mbar_wait(smem_u32(&bars.full[j % STAGES]), (j / STAGES) & 1, &never);
            }
        }
    } else if (warp == 1) {
        if (lane == 0 && leader) {
            // the pair's MMA issuer
            const uint32_t idesc = idesc_f16_256x256();
            uint32_t g = 0, tl = 0;
            for (int t = cid; t < nblocks && !abort_flag; t += ncl, ++tl) {
                const uint32_t b = tl & 1;
                if (!mbar_wait(smem_u32(&bars.accempty[b]), ((tl >> 1) & 1) ^ 1, &abort_flag, wlim)) {
                    stop_pair();
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc = tmem + b * 256;
                bool ok = true;
                for (int kc = 0; kc < nchunk; ++kc, ++g) {
                    const int s = g % STAGES;
                    if (!mbar_wait(smem_u32(&bars.full[s]), (g / STAGES) & 1, &abort_flag, wlim)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t ah = sbase + s * STAGE_BYTES, al = ah + BOX_BYTES;
                    const uint32_t bh = ah + 2 * BOX_BYTES, bl = ah + 3 * BOX_BYTES;
#pragma unroll
                    for (int ks = 0; ks < KSTEPS; ++ks) {
                        const uint32_t off = ks * 32;   // 16 FP16 of K
                        umma_f16_pair(acc, umma_desc_sw128(ah + off), umma_desc_sw128(bh + off), idesc,
                                      (kc | ks) ? 1u : 0u);
                        umma_f16_pair(acc, umma_desc_sw128(ah + off), umma_desc_sw128(bl + off), idesc, 1u);
                        umma_f16_pair(acc, umma_desc_sw128(al + off), umma_desc_sw128(bh + off), idesc, 1u);
                    }
                    umma_commit_pair(smem_u32(&bars.empty[s]));
                }
                if (!ok) {
                    stop_pair();
                    break;
                }
                umma_commit_pair(smem_u32(&bars.accfull[b]));
            }
            if (abort_flag) {
                volatile int never = 0;
                asm volatile(
                    "{\n\t.reg .b16 m;\n\tmov.b16 m, 1;\n\t"
                    "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], "
                    "m;\n\t}" ::"r"(smem_u32(&bars.drain))
                    : "memory");
                mbar_wait(smem_u32(&bars.drain), 0, &never);
            }
        }
    } else {
        // epilogue warps 2..5: this CTA's 128 rows (tile row ti + rank) of
        // the block, its two 128-column tiles in turn; tiles above the
        // diagonal or past the matrix are read from tensor memory (so that
        // the buffer's release is counted alike) but not written
        const int quarter = warp & 3;
        const int rl = 32 * quarter + lane;
        const float is2 = pscale[1];   // 1 / scale^2: the panels' FP16 scaling undone, exactly
        const uint32_t accempty0 = cluster_addr(smem_u32(&bars.accempty[0]), 0);
        uint32_t tl = 0;
        for (int t = cid; t < nblocks; t += ncl, ++tl) {
            int ti, tj;
            pair_block(t, c0, ti, tj);
            ti += (int)rank;
            const uint32_t b = tl & 1;
            if (epi_any(!mbar_wait(smem_u32(&bars.accfull[b]), (tl >> 1) & 1, &abort_flag, wlim))) {
                if (tid == 64) stop_pair();
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
            for (int h = 0; h < 2; ++h) {
                const int tjh = tj + h;
                const bool live = ti < cols && tjh <= ti;
                const bool diag = ti == tjh;
                const int ra = (t0 + ti) * PW, rb = (t0 + tjh) * PW;
#pragma unroll 1
                for (int cc = 0; cc < PW / 32; ++cc) {
                    uint32_t v[32];
                    const uint32_t taddr =
                        tmem + b * 256 + h * 128 + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(32 * cc);
                    asm volatile(
                        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                        "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
                        "%30, %31}, [%32];"
                        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                          "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]),
                          "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                          "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                        : "r"(taddr));
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    if (h == 1 && cc == PW / 32 - 1) {
                        // the buffer is free once both CTAs have read it all
                        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                        __syncwarp();
                        if (lane == 0)
                            asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(
                                             accempty0 + b * (uint32_t)sizeof(uint64_t))
                                         : "memory");
                    }
                    if (!live) continue;
                    if (tid == 64) bulk_wait_read_ring();
                    epi_sync();
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const int c = 32 * cc + 4 * j;
                        float4 d;
                        d.x = (!diag || c <= rl) ? -is2 * __uint_as_float(v[4 * j]) : -0.0f;
                        d.y = (!diag || c + 1 <= rl) ? -is2 * __uint_as_float(v[4 * j + 1]) : -0.0f;
                        d.z = (!diag || c + 2 <= rl) ? -is2 * __uint_as_float(v[4 * j + 2]) : -0.0f;
                        d.w = (!diag || c + 3 <= rl) ? -is2 * __uint_as_float(v[4 * j + 3]) : -0.0f;
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
        }
        if (tid == 64) bulk_wait0();
    }
    if (abort_flag && tid == 0) atomicOr(status, ST_TIMEOUT);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    // neither CTA frees its tensor memory or exits while the other may still
    // signal its barriers or (the leader's MMAs) write its tensor memory
    cluster_sync_all();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
    }
}

// ------------------------------------------------- FP64 trailing update
//
// The plain FP64 path's C -= L_i L_j^T on the FP64 tensor instruction
// (mma.sync m8n8k4 f64; tcgen05 has no FP64 kind): a persistent CTA of 8
// warps per 128x128 tile, warp w owning rows 32 (w mod 4).. and columns
// 64 (w / 4).. as 32 accumulator tiles in registers, initialised from C and
// stored back (lower triangle only on diagonal tiles, whose upper triangle
// holds D). The panel rows of tiles i and j stream through shared memory in
// chunks of 32 columns (cp.async, two stages). The panel solve stores the
// FP64 panel with each group of 8 columns permuted (column c at 2 (c mod 4)
// + (c / 4 mod 2)), so a lane's operands of k-steps kk and kk + 4 are
// adjacent: one 16-byte shared load feeds two k-steps. Rows padded to 40
// doubles (an 8-row quarter-warp's 16-byte loads then hit distinct banks).
// Per chunk a warp issues 256 DMMAs from 48 fragment loads; every
// accumulator takes its k-steps in order, as with natural column order.
static constexpr int S64_THREADS = 256;
static constexpr int S64_KC = 32;                        // panel columns per staged chunk
static constexpr int S64_LD = 40;                        // padded row stride of a staged chunk (doubles)
static constexpr int S64_CHUNK = PW * S64_LD;            // doubles of one operand chunk
static constexpr int S64_SMEM = 2 * 2 * S64_CHUNK * 8;   // two stages of A and B chunks: 160 KB

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// columns [k0, k0 + 32) of the panel rows of tiles ra (A) and rb (B), as
// stored (fragment order): 2 x 2048 16-byte pieces, 8 + 8 per thread
__device__ __forceinline__ void s64_stage(double* As, double* Bs, const double* __restrict__ Lp, int ra, int rb,
                                          int k0, int tid)
{
    constexpr int PIECES = S64_KC / 2;   // 16-byte pieces per row
#pragma unroll
    for (int q = tid; q < PW * PIECES; q += S64_THREADS) {
        const int r = q / PIECES, c = (q % PIECES) * 2;
        cp_async16(smem_u32(As + r * S64_LD + c), Lp + (size_t)(ra + r) * PW + k0 + c);
        cp_async16(smem_u32(Bs + r * S64_LD + c), Lp + (size_t)(rb + r) * PW + k0 + c);
    }
}

__global__ void __launch_bounds__(S64_THREADS, 1) k_syrk64(double* __restrict__ M, int npad,
                                                         const double* __restrict__ Lp, int t0, int ntiles, int mode,
                                                         unsigned* __restrict__ status)
{
    extern __shared__ __align__(16) double sm64[];
    {
        uint32_t dyn;
        asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
        if (blockDim.x != S64_THREADS || dyn < (uint32_t)S64_SMEM) {
            if (threadIdx.x == 0) atomicOr(status, ST_LAUNCH);
            return;
        }
    }
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int fr = lane >> 2, fq = lane & 3;
    const int wr = warp & 3, wc = warp >> 2;
    // a programmatic dependent of the previous kernel on the stream: nothing
    // it produces is read before this. Dependents launch at once after the
    // chain's and the side stream's updates (modes 1, 4), after a bulk
    // update only when each CTA starts its last tile (a bulk dependent
    // launched early would hold free SMs in its wait)
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (mode == 1 || mode == 4) asm volatile("griddepcontrol.launch_dependents;");
    constexpr int NCH = PW / S64_KC;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        if (t + (int)gridDim.x >= ntiles) asm volatile("griddepcontrol.launch_dependents;");
        int ti, tj;
        tile_of_mode(t, mode, ti, tj);
        const int ra = (t0 + ti) * PW, rb = (t0 + tj) * PW;
        const bool diag = ti == tj;
        s64_stage(sm64, sm64 + S64_CHUNK, Lp, ra, rb, 0, tid);
        cp_async_commit();
        double acc[4][8][2];
#pragma unroll
        for (int rt = 0; rt < 4; ++rt)
#pragma unroll
            for (int ct = 0; ct < 8; ++ct) {
                const size_t row = (size_t)ra + 32 * wr + 8 * rt + fr;
                const double2 v = *reinterpret_cast<const double2*>(M + row * npad + rb + 64 * wc + 8 * ct + 2 * fq);
                acc[rt][ct][0] = v.x;
                acc[rt][ct][1] = v.y;
            }
#pragma unroll 1
        for (int kc = 0; kc < NCH; ++kc) {
            const double* As = sm64 + (kc & 1) * 2 * S64_CHUNK;
            const double* Bs = As + S64_CHUNK;
            if (kc + 1 < NCH) {
                double* nA = sm64 + ((kc + 1) & 1) * 2 * S64_CHUNK;
                s64_stage(nA, nA + S64_CHUNK, Lp, ra, rb, (kc + 1) * S64_KC, tid);
                cp_async_commit();
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
#pragma unroll
            for (int kk = 0; kk < S64_KC; kk += 8) {
                // k-steps kk (.x) and kk + 4 (.y) of this lane's fragments
                double2 a[4], b[8];
#pragma unroll
                for (int rt = 0; rt < 4; ++rt) {
                    const double2 v =
                        *reinterpret_cast<const double2*>(As + (32 * wr + 8 * rt + fr) * S64_LD + kk + 2 * fq);
                    a[rt] = make_double2(-v.x, -v.y);
                }
#pragma unroll
                for (int ct = 0; ct < 8; ++ct)
                    b[ct] = *reinterpret_cast<const double2*>(Bs + (64 * wc + 8 * ct + fr) * S64_LD + kk + 2 * fq);
#pragma unroll
                for (int rt = 0; rt < 4; ++rt)
#pragma unroll
                    for (int ct = 0; ct < 8; ++ct) dmma884(acc[rt][ct][0], acc[rt][ct][1], a[rt].x, b[ct].x);
#pragma unroll
                for (int rt = 0; rt < 4; ++rt)
#pragma unroll
                    for (int ct = 0; ct < 8; ++ct) dmma884(acc[rt][ct][0], acc[rt][ct][1], a[rt].y, b[ct].y);
            }
            __syncthreads();   // this stage is read; it may be staged again
        }
#pragma unroll
        for (int rt = 0; rt < 4; ++rt)
#pragma unroll
            for (int ct = 0; ct < 8; ++ct) {
                const int r = 32 * wr + 8 * rt + fr, c = 64 * wc + 8 * ct + 2 * fq;
                double* dst = M + ((size_t)ra + r) * npad + rb + c;
                if (!diag) {
                    *reinterpret_cast<double2*>(dst) = make_double2(acc[rt][ct][0], acc[rt][ct][1]);
                } else {
                    if (c <= r) dst[0] = acc[rt][ct][0];
                    if (c + 1 <= r) dst[1] = acc[rt][ct][1];
                }
            }
    }
}

// ---------------------------------------------------------------- host side

// row-major FP32 [rows][cols] buffer, boxes of 128 rows x 32 columns
// (f16: an FP16 panel buffer [rows][128], boxes of 128 rows x 64 columns;
// otherwise FP32, boxes of 128 rows x 32 columns; 128 bytes a box row)
static int make_panel_map(void* buf, int rows, CUtensorMap* map, int cols = PW, bool f16 = false)
{
    auto enc = get_encode();
    if (!enc) return fail(BDB_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    if (reinterpret_cast<uintptr_t>(buf) % 16) return fail(BDB_ERR_ARG, "panel buffer not 16-byte aligned");
    const size_t es = f16 ? 2 : 4;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)cols * es};
    cuuint32_t box[2] = {(cuuint32_t)(f16 ? KCP : KC), PW};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, f16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, buf, dims,
                     strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(BDB_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    return BDB_OK;
}

// scratch layout in panel64: four panel buffer sets (hi, lo: FP32
// [npad][128] each; on the FP64 path one FP64 [npad][128] panel in their
// room), then four FP64 128x128 hand-offs of L_PP / W_kk; panel P uses set
// P mod 4, so a panel's updates may still read its set (and the previous
// panel's) while the next two panels are solved
static constexpr int PANEL_SETS = 4;

static void panel_ptrs(bdb_system* s, int set, float** hi, float** lo, double** lkk)
{
    const size_t pan = (size_t)s->npad * PW;
    float* base = reinterpret_cast<float*>(s->panel64.p);
    *hi = base + (size_t)set * 2 * pan;
    *lo = *hi + pan;
    *lkk = reinterpret_cast<double*>(base + (size_t)PANEL_SETS * 2 * pan) + (size_t)set * PANEL_FAC;
}

static int tc_setup(bdb_system* s)
{
    if (s->tc_map_ok) return BDB_OK;
    const size_t pan = (size_t)s->npad * PW;
    // floats of the panel sets are counted as half a double each
    if (s->panel64.alloc((size_t)PANEL_SETS * pan + (size_t)PANEL_SETS * PANEL_FAC + 64)) return BDB_ERR_NOMEM;
    BDB_CUDA(dzero(s, s->panel64.p, s->panel64.n * sizeof(double)));
    static_assert(sizeof(CUtensorMap) * (2 * PANEL_SETS + 1) <= sizeof(bdb_system::tc_map), "tensor-map storage");
    CUtensorMap* maps = reinterpret_cast<CUtensorMap*>(s->tc_map);   // hi0, lo0, ..., hi3, lo3, M
    for (int set = 0; set < PANEL_SETS; ++set) {
        float *hi, *lo;
        double* lkk;
        panel_ptrs(s, set, &hi, &lo, &lkk);
        int rc = make_panel_map(hi, s->npad, &maps[2 * set], PW, true);
        if (rc) return rc;
        rc = make_panel_map(lo, s->npad, &maps[2 * set + 1], PW, true);
        if (rc) return rc;
    }
    int rc = make_panel_map(s->M32.p, s->npad, &maps[2 * PANEL_SETS], s->npad);
    if (rc) return rc;
    BDB_CUDA(cudaFuncSetAttribute(k_syrk_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, SYRK_SMEM));
    BDB_CUDA(cudaFuncSetAttribute(k_syrk_tc2, cudaFuncAttributeMaxDynamicSharedMemorySize, SYRK_SMEM));
    if (s->pscale.alloc(2)) return BDB_ERR_NOMEM;
    BDB_CUDA(cudaFuncSetAttribute(k_potrf128<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, POTRF_SMEM));
    BDB_CUDA(cudaFuncSetAttribute(k_trsm128<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, TRSM_SMEM));
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
    return cudaLaunchKernelEx(&cfg, k_syrk_tc, hi, lo, c, t0, ntiles, mode, s->status.p, (uint32_t)s->wait_limit,
                              (const float*)s->pscale.p);
}

// k_syrk_tc2 on `clusters` CTA pairs over block columns c0 .. cols-1 of
// the trailing matrix at block t0 with the updates of npan panels (the
// first in hi / lo, the second in hi2 / lo2), behind the previous kernel on
// the stream like launch_syrk
static cudaError_t launch_syrk_pair(bdb_system* s, int clusters, cudaStream_t st, const CUtensorMap& hi,
                                    const CUtensorMap& lo, const CUtensorMap& hi2, const CUtensorMap& lo2,
                                    const CUtensorMap& c, int t0, int c0, int cols, int npan)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * clusters);
    cfg.blockDim = dim3(192);
    cfg.dynamicSmemBytes = SYRK_SMEM;
    cfg.stream = st;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    at[1].id = cudaLaunchAttributeClusterDimension;
    at[1].val.clusterDim.x = 2;
    at[1].val.clusterDim.y = 1;
    at[1].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 2;
    return cudaLaunchKernelEx(&cfg, k_syrk_tc2, hi, lo, hi2, lo2, c, t0, c0, cols, npan, s->status.p,
                              (uint32_t)s->wait_limit, (const float*)s->pscale.p);
}

// k_potrf128 the same way, behind the update of its block column
template <typename T>
static cudaError_t launch_potrf(bdb_system* s, cudaStream_t st, T* M, int P, double* lkk)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(1);
    cfg.blockDim = dim3(POTRF_THREADS);
    cfg.dynamicSmemBytes = POTRF_SMEM;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_potrf128<T>, M, s->npad, P, lkk, s->status.p, (uint32_t)s->wait_limit);
}

// block row P+1 of panel P's solve (k_trsm128, units 0..15 on 4 CTAs) as a
// programmatic dependent of the diagonal block's factorisation, so that its
// launch overlaps that kernel's tail
template <typename T>
static cudaError_t launch_trsm_top(bdb_system* s, cudaStream_t st, T* M, int P, int units, const double* lkk,
                                   float* hi, float* lo, const float* pscale)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(units / 4);
    cfg.blockDim = dim3(TRSM_THREADS);
    cfg.dynamicSmemBytes = TRSM_SMEM;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_trsm128<T>, M, s->npad, P, 0, units, lkk, hi, lo, s->status.p, pscale);
}

// The factorisation schedule, on three streams. Panel P's trailing update
// is split four ways: the diagonal tile of block column P+1 (A0), the rest
// of that column (A1), block column P+2 (B) and block columns P+3 on (C);
// its panel solve two ways: block row P+1 (top) and the rows below (rest).
//   chain stream: top(P) -> A0(P) -> diagonal block P+1 -> top(P+1) -> ...
//   side stream:  rest(P) -> A1(P) -> rest(P+1) -> ...
//   bulk stream:  B(P) -> C(P) -> B(P+1) -> C(P+1) -> ...
// So the diagonal block P+1 waits only for one panel-solve block row and
// one tile update, while the rest of panel P's solve and of its column
// update run beside it; the bulk updates of panel P run beside the next two
// steps of the chain. Hand-offs:
//   rest(P) after the diagonal block P; top(P) after A1(P-1) and B(P-1)
//   (both update block column P or P+1 before panel P's updates do);
//   A1(P) after top(P) (its B operand rows) and B(P-1); B(P) once the whole
//   panel is solved.
// The mixed path (T = float) pairs the panels for C: an even panel P
// updates block column P+3 alone, and the odd panel P+1 applies both
// panels' updates to block columns P+4 on in one K = 256 pass on CTA pairs,
// which halves the reads and writes of C, the bulk's largest cost. Every tile
// receives the same updates in the same order whatever the GPU split (the
// same bits for every chain_sms). Four panel-buffer sets let C(P) read
// panels P-1 and P while panels P+1 and P+2 are solved. The persistent bulk
// updates leave s->chain_sms SMs to the chain and side kernels (tuned).
template <typename T, typename Update>
static int factor_schedule(bdb_system* s, T* M, Update update)
{
    const int nt = s->npad / PW;
    cudaStream_t st = s->stream, st2 = s->stream2, st3 = s->stream3;
    cudaEvent_t ev_potrf = s->la_ev[0], ev_top = s->la_ev[1], ev_rest = s->la_ev[2], ev_side = s->la_ev[3],
                ev_b = s->la_ev[4], ev_end = s->la_ev[5];
    const int chain = std::min(std::max(s->chain_sms, 1), s->sm_count - 1);
    const int bulk_sms = std::max(1, s->sm_count - chain);
    const int per_cta = TRSM_THREADS / 32, units_top = PW / 8;
    // the side kernels take the chain's SMs but five (the diagonal block,
    // the four CTAs of the top panel solve); the panel solve two CTAs per SM
    // (its registers and shared memory allow it), for more warps on the FP64
    // pipes
    const int side = std::max(1, chain - 5);
    constexpr bool kPairs = sizeof(T) == 4;   // two panels per pass over C (mixed path)
    const float* pscale = sizeof(T) == 4 ? s->pscale.p : nullptr;   // FP16 panel scale (mixed path)
    float *hi, *lo;
    double* lkk;
    panel_ptrs(s, 0, &hi, &lo, &lkk);
    phase_mark_on(s, P_POTRF, st);
    BDB_CUDA(launch_potrf(s, st, M, 0, lkk));
    phase_mark_on(s, P_POTRF, st);
    s->launches += 1;
    BDB_CUDA(cudaEventRecord(ev_potrf, st));
    BDB_CUDA(cudaStreamWaitEvent(st2, ev_potrf, 0));   // the bulk stream starts after what came before
    for (int P = 0; P + 1 < nt; ++P) {
        const int set = P % PANEL_SETS;
        panel_ptrs(s, set, &hi, &lo, &lkk);
        const int rem = nt - P - 1;   // trailing block columns
        const int units_rest = (rem - 1) * PW / 8;
        // side: the panel solve below block row P+1
        BDB_CUDA(cudaStreamWaitEvent(st3, ev_potrf, 0));
        if (units_rest > 0) {
            k_trsm128<T><<<std::min(2 * side, (units_rest + per_cta - 1) / per_cta), TRSM_THREADS, TRSM_SMEM, st3>>>(
                M, s->npad, P, units_top, units_rest, lkk, hi, lo, s->status.p, pscale);
            BDB_CUDA(cudaGetLastError());
            s->launches += 1;
        }
        BDB_CUDA(cudaEventRecord(ev_rest, st3));
        // chain: block row P+1 of the panel solve
        if (P > 0) {
            BDB_CUDA(cudaStreamWaitEvent(st, ev_side, 0));   // A1(P-1)
            BDB_CUDA(cudaStreamWaitEvent(st, ev_b, 0));      // B(P-1)
        }
        phase_mark_on(s, P_TRSM, st);
        // block row P+1: its 16 units on 4 CTAs, so that each unit's warp
        // has an SM sub-partition (and its FP64 pipe) to itself
        BDB_CUDA(launch_trsm_top(s, st, M, P, units_top, lkk, hi, lo, pscale));
        phase_mark_on(s, P_TRSM, st);
        BDB_CUDA(cudaEventRecord(ev_top, st));
        // side: block column P+1 below its diagonal tile
        BDB_CUDA(cudaStreamWaitEvent(st3, ev_top, 0));
        if (P > 0) BDB_CUDA(cudaStreamWaitEvent(st3, ev_b, 0));   // B(P-1)
        if (rem > 1) {
            BDB_CUDA(update(st3, std::min(rem - 1, side), set, -1, P + 1, rem - 1, 4));
            s->launches += 1;
        }
        BDB_CUDA(cudaEventRecord(ev_side, st3));
        // bulk: block column P+2, then the rest
        BDB_CUDA(cudaStreamWaitEvent(st2, ev_top, 0));
        BDB_CUDA(cudaStreamWaitEvent(st2, ev_rest, 0));
        phase_mark_on(s, P_SYRK_REST, st2);
        if (rem >= 2) {
            BDB_CUDA(update(st2, std::min(bulk_sms, rem - 1), set, -1, P + 1, rem - 1, 2));
            s->launches += 1;
        }
        BDB_CUDA(cudaEventRecord(ev_b, st2));
        if (rem >= 3) {
            if (kPairs && P % 2 == 0) {
                // block column P+3 alone; the columns beyond take this
                // panel's update together with panel P+1's
                BDB_CUDA(update(st2, std::min(bulk_sms, rem - 2), set, -1, P + 1, rem - 2, 5));
            } else {
                // block columns P+3 on: panel P, and on the mixed path panel
                // P-1 (deferred there) in the same pass
                const int ntc = (rem - 2) * (rem - 1) / 2;
                const int set_prev = kPairs ? (P - 1) % PANEL_SETS : -1;
                BDB_CUDA(update(st2, std::min(bulk_sms, ntc), set, set_prev, P + 1, ntc, 3));
            }
            s->launches += 1;
        }
        phase_mark_on(s, P_SYRK_REST, st2);
        // chain: the diagonal tile of block column P+1, then its factorisation
        phase_mark_on(s, P_SYRK_COL, st);
        BDB_CUDA(update(st, 1, set, -1, P + 1, 1, 1));
        phase_mark_on(s, P_SYRK_COL, st);
        double* lkk1;
        float *hi1, *lo1;
        panel_ptrs(s, (P + 1) % PANEL_SETS, &hi1, &lo1, &lkk1);
        phase_mark_on(s, P_POTRF, st);
        BDB_CUDA(launch_potrf(s, st, M, P + 1, lkk1));
        phase_mark_on(s, P_POTRF, st);
        BDB_CUDA(cudaEventRecord(ev_potrf, st));
        s->launches += 3;
    }
    // join the side and bulk streams
    BDB_CUDA(cudaEventRecord(ev_side, st3));
    BDB_CUDA(cudaStreamWaitEvent(st, ev_side, 0));
    BDB_CUDA(cudaEventRecord(ev_end, st2));
    BDB_CUDA(cudaStreamWaitEvent(st, ev_end, 0));
    BDB_CUDA(cudaGetLastError());
    return BDB_OK;
}

// The FP16 panel scale of a factorisation, from D's diagonal (dD): 2^e with
// the largest sqrt(D_ii) -- a bound of every |L_ij| -- just below 2^14;
// pscale[0] = 2^e, pscale[1] = 2^-2e. One CTA.
__global__ void k_panel_scale(const double* __restrict__ dD, int n3, float* __restrict__ pscale)
{
    __shared__ double red[32];
    double m = 0.0;
    for (int i = threadIdx.x; i < n3; i += blockDim.x) m = fmax(m, dD[i]);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
        int e = 0, sh = 0;
        if (m > 0.0 && isfinite(m)) {
            frexp(sqrt(m), &e);   // sqrt(m) < 2^e
            sh = 14 - e;
        }
        sh = max(-60, min(60, sh));
        pscale[0] = ldexpf(1.0f, sh);
        pscale[1] = ldexpf(1.0f, -2 * sh);
    }
}

int factor_mixed_tc(bdb_system* s)
{
    int rc = tc_setup(s);
    if (rc) return rc;
    k_panel_scale<<<1, 1024, 0, s->stream>>>(s->dD.p, s->n3, s->pscale.p);
    BDB_CUDA(cudaGetLastError());
    s->launches += 1;
    const CUtensorMap* maps = reinterpret_cast<const CUtensorMap*>(s->tc_map);
    const int nt = s->npad / PW;
    return factor_schedule(s, s->M32.p, [&](cudaStream_t stream, int grid, int set, int set_prev, int t0, int ntiles,
                                            int mode) {
        if (mode == 3) {
            // block columns 2.. of the trailing matrix: 256-wide blocks on
            // CTA pairs, with the previous panel's update too if it is given
            const int cols = nt - t0, nb = (cols - 1) / 2;
            const int clusters = std::max(1, std::min(grid / 2, nb * (nb + 1) / 2));
            const int first = set_prev >= 0 ? set_prev : set;
            return launch_syrk_pair(s, clusters, stream, maps[2 * first], maps[2 * first + 1], maps[2 * set],
                                    maps[2 * set + 1], maps[2 * PANEL_SETS], t0, 2, cols, set_prev >= 0 ? 2 : 1);
        }
        return launch_syrk(s, grid, stream, maps[2 * set], maps[2 * set + 1], maps[2 * PANEL_SETS], t0, ntiles, mode);
    });
}

// ------------------------------------------------------ FP64 factorisation

static int tc64_setup(bdb_system* s)
{
    if (s->tc64_ok) return BDB_OK;
    const size_t pan = (size_t)s->npad * PW;
    // one FP64 panel buffer per set (the room of a mixed-path hi/lo pair)
    if (s->panel64.alloc((size_t)PANEL_SETS * pan + (size_t)PANEL_SETS * PANEL_FAC + 64)) return BDB_ERR_NOMEM;
    BDB_CUDA(dzero(s, s->panel64.p, s->panel64.n * sizeof(double)));
    BDB_CUDA(cudaFuncSetAttribute(k_potrf128<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, POTRF_SMEM));
    BDB_CUDA(cudaFuncSetAttribute(k_trsm128<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, TRSM_SMEM));
    BDB_CUDA(cudaFuncSetAttribute(k_syrk64, cudaFuncAttributeMaxDynamicSharedMemorySize, S64_SMEM));
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    s->sm_count = sms;
    s->tc64_ok = true;
    return BDB_OK;
}

static cudaError_t launch_syrk64(bdb_system* s, int grid, cudaStream_t st, const double* Lp, int t0, int ntiles,
                                 int mode)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(S64_THREADS);
    cfg.dynamicSmemBytes = S64_SMEM;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_syrk64, s->M64.p, s->npad, Lp, t0, ntiles, mode, s->status.p);
}

// The plain FP64 path: the same schedule with FP64 panels and FP64 DMMA
// trailing updates
int factor_fp64_tc(bdb_system* s)
{
    int rc = tc64_setup(s);
    if (rc) return rc;
    return factor_schedule(s, s->M64.p, [&](cudaStream_t stream, int grid, int set, int, int t0, int ntiles,
                                            int mode) {
        float *hi, *lo;
        double* lkk;
        panel_ptrs(s, set, &hi, &lo, &lkk);
        return launch_syrk64(s, grid, stream, reinterpret_cast<const double*>(hi), t0, ntiles, mode);
    });
}

}  // namespace bdb
