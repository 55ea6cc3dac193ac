// Mixed-precision blocked Cholesky for sm_100a: FP64 panels, 3xTF32
// trailing updates on the 5th-generation tensor cores (tcgen05).
//
// M is FP32 (lower triangle: the factor, upper: D, never written here).
// Super-panel P covers columns p0 = 128P .. p0+127:
//   k_potrf128  one CTA factors the 128x128 diagonal block in FP64 (blocked
//               by 16 columns: one warp factors each 16x16 pivot block with
//               shuffles, then all threads solve and update the rest of the
//               block in shared memory); L_PP goes to M (FP32) and, in FP64
//               and transposed, to a 128x128 scratch block for the panel solve;
//   k_trsm128   one warp per row below the block solves x L_PP^T = a in FP64
//               (lane l owns columns 4l..4l+3); writes the row to M and its
//               TF32 split L = L_hi + L_lo (L_hi: low 13 mantissa bits
//               cleared, exactly TF32; L_lo = L - L_hi) to two panel buffers;
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
//             lanes 32(w%4)..), C -= acc in global memory (lower triangle
//             only on diagonal tiles), then hand the accumulator back.
// The epilogue of tile t overlaps the MMAs of tile t+1 and the loads of the
// tiles after it. Every mbarrier wait is bounded; a time-out sets
// ST_TIMEOUT and a shared abort flag that stops all roles, and the CTA frees
// its tensor memory before returning.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>

#include "bdb_common.cuh"

namespace bdb {

static constexpr int PW = 128;                    // super-panel width = tile size
static constexpr int KC = 32;                     // K columns per TMA box (128 B of FP32)
static constexpr int NCHUNK = PW / KC;            // 4
static constexpr int STAGES = 2;
static constexpr int BOX_BYTES = PW * KC * 4;     // 16 KB
static constexpr int STAGE_BYTES = 4 * BOX_BYTES; // A_hi, A_lo, B_hi, B_lo
static constexpr int C_BYTES = PW * PW * 4;       // one C tile, 4 boxes of 128 rows x 32 columns
static constexpr int SYRK_SMEM = STAGES * STAGE_BYTES + C_BYTES + 1024;
static constexpr uint32_t WAIT_LIMIT = 1u << 22;
static constexpr int LDS = PW + 1;                // padded FP64 row in shared memory

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// bounded wait for the phase of the given parity; false on time-out or abort
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort)
{
    for (uint32_t it = 0; it < WAIT_LIMIT; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 1023) == 1023 && *abort) return false;
    }
    *abort = 1;
    return false;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, uint32_t src, int x, int y)
{
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y), "r"(src)
                 : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }

__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// barrier 1 among the 128 epilogue threads only
__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

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

__device__ __forceinline__ float tf32_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }

// ------------------------------------------------------------ FP64 panel

__global__ void __launch_bounds__(256) k_potrf128(float* __restrict__ M, int npad, int P, double* __restrict__ Lkk,
                                                  unsigned* __restrict__ status)
{
    extern __shared__ double S[];   // [PW][LDS]
    __shared__ double dinv16[16];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const size_t base = (size_t)P * PW;
    for (int idx = tid; idx < PW * PW; idx += blockDim.x) {
        const int r = idx / PW, c = idx % PW;
        S[r * LDS + c] = c <= r ? (double)M[(base + r) * npad + base + c] : 0.0;
    }
    __syncthreads();
    bool bad = false;
    for (int c0 = 0; c0 < PW; c0 += 16) {
        // 1. 16x16 pivot block by warp 0 (lane & 15 = row)
        if (warp == 0) {
            const int lr = lane & 15;
            const int r = c0 + lr;
            double a[16];
#pragma unroll
            for (int c = 0; c < 16; ++c) a[c] = S[r * LDS + c0 + c];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const double piv = __shfl_sync(0xffffffffu, a[j], j);
                if (!(piv > 0.0)) bad = true;
                const double inv = rsqrt(piv), d = piv * inv;
                const double lj = lr == j ? d : (lr > j ? a[j] * inv : a[j]);
                a[j] = lj;
#pragma unroll
                for (int c = j + 1; c < 16; ++c) {
                    const double lcj = __shfl_sync(0xffffffffu, lj, c);
                    if (lr >= c) a[c] -= lj * lcj;
                }
            }
            if (lane < 16) {
#pragma unroll
                for (int c = 0; c < 16; ++c)
                    if (c <= lr) S[r * LDS + c0 + c] = a[c];
            }
        }
        if (tid < 16) dinv16[tid] = 1.0 / S[(c0 + tid) * LDS + c0 + tid];
        __syncthreads();
        // 2. rows below inside the block: x L16^T = a
        const int nrow = PW - c0 - 16;
        if (tid < nrow) {
            const int r = c0 + 16 + tid;
            double x[16];
#pragma unroll
            for (int c = 0; c < 16; ++c) x[c] = S[r * LDS + c0 + c];
#pragma unroll
            for (int m = 0; m < 16; ++m) {
                x[m] *= dinv16[m];
#pragma unroll
                for (int c = m + 1; c < 16; ++c) x[c] -= S[(c0 + c) * LDS + c0 + m] * x[m];
            }
#pragma unroll
            for (int c = 0; c < 16; ++c) S[r * LDS + c0 + c] = x[c];
        }
        __syncthreads();
        // 3. trailing update of the block, 4x4 register tiles (lower triangle)
        const int nb4 = nrow / 4;
        const int cnt = nb4 * (nb4 + 1) / 2;
        for (int e = tid; e < cnt; e += blockDim.x) {
            int br, bc;
            tri_index(e, br, bc);
            const int r0 = c0 + 16 + 4 * br, k0 = c0 + 16 + 4 * bc;
            double acc[4][4] = {};
#pragma unroll 4
            for (int m = 0; m < 16; ++m) {
                double a[4], b[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    a[q] = S[(r0 + q) * LDS + c0 + m];
                    b[q] = S[(k0 + q) * LDS + c0 + m];
                }
#pragma unroll
                for (int q = 0; q < 4; ++q)
#pragma unroll
                    for (int p = 0; p < 4; ++p) acc[q][p] += a[q] * b[p];
            }
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int p = 0; p < 4; ++p)
                    if (k0 + p <= r0 + q) S[(r0 + q) * LDS + k0 + p] -= acc[q][p];
        }
        __syncthreads();
    }
    if (bad) atomicOr(status, ST_NOT_SPD);
    // L_PP to M (FP32, lower) and, transposed, to the FP64 scratch block:
    // LkkT[m][c] = L[c][m], the layout the panel solve reads
    for (int idx = tid; idx < PW * PW; idx += blockDim.x) {
        const int r = idx / PW, c = idx % PW;
        if (c <= r) M[(base + r) * npad + base + c] = (float)S[r * LDS + c];
        const int m = idx / PW, cc = idx % PW;
        Lkk[idx] = cc >= m ? S[cc * LDS + m] : 0.0;
    }
}

// rows below block P: x L_PP^T = a; each warp solves R = 4 rows at once so
// every row of L_PP read from shared memory serves four rows; writes M and
// the split panel
static constexpr int TRSM_R = 4;

__global__ void __launch_bounds__(512) k_trsm128(float* __restrict__ M, int npad, int P, const double* __restrict__ Lkk,
                                                 float* __restrict__ Lhi, float* __restrict__ Llo)
{
    extern __shared__ double Lt[];   // Lt[m][c] = L[c][m], [PW][PW]
    __shared__ double dinv[PW];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int idx = tid; idx < PW * PW / 2; idx += blockDim.x)
        reinterpret_cast<double2*>(Lt)[idx] = reinterpret_cast<const double2*>(Lkk)[idx];   // already transposed
    if (tid < PW) dinv[tid] = 1.0 / Lkk[tid * PW + tid];
    __syncthreads();
    const size_t base = (size_t)P * PW;
    const int nw = blockDim.x >> 5;
    const size_t first = base + PW;
    for (size_t row0 = first + ((size_t)blockIdx.x * nw + warp) * TRSM_R; row0 < (size_t)npad;
         row0 += (size_t)gridDim.x * nw * TRSM_R) {
        double x[TRSM_R][4];
#pragma unroll
        for (int q = 0; q < TRSM_R; ++q) {
            const size_t row = row0 + q;
            float4 a4 = make_float4(0.f, 0.f, 0.f, 0.f);
            if (row < (size_t)npad) a4 = reinterpret_cast<const float4*>(M + row * npad + base)[lane];
            x[q][0] = a4.x;
            x[q][1] = a4.y;
            x[q][2] = a4.z;
            x[q][3] = a4.w;
        }
#pragma unroll 1
        for (int mb = 0; mb < PW / 4; ++mb) {
#pragma unroll
            for (int qq = 0; qq < 4; ++qq) {
                const int m = 4 * mb + qq;
                const double dm = dinv[m];
                const double2 l01 = *reinterpret_cast<const double2*>(&Lt[m * PW + 4 * lane]);
                const double2 l23 = *reinterpret_cast<const double2*>(&Lt[m * PW + 4 * lane + 2]);
#pragma unroll
                for (int q = 0; q < TRSM_R; ++q) {
                    if (lane == mb) x[q][qq] *= dm;
                    const double xm = __shfl_sync(0xffffffffu, x[q][qq], mb);
                    if (lane > mb) {
                        x[q][0] -= l01.x * xm;
                        x[q][1] -= l01.y * xm;
                        x[q][2] -= l23.x * xm;
                        x[q][3] -= l23.y * xm;
                    } else if (lane == mb) {
                        if (qq < 1) x[q][1] -= l01.y * xm;
                        if (qq < 2) x[q][2] -= l23.x * xm;
                        if (qq < 3) x[q][3] -= l23.y * xm;
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < TRSM_R; ++q) {
            const size_t row = row0 + q;
            if (row >= (size_t)npad) break;
            float4 o, h, l;
            o.x = (float)x[q][0];
            o.y = (float)x[q][1];
            o.z = (float)x[q][2];
            o.w = (float)x[q][3];
            h.x = tf32_hi(o.x);
            h.y = tf32_hi(o.y);
            h.z = tf32_hi(o.z);
            h.w = tf32_hi(o.w);
            l.x = o.x - h.x;
            l.y = o.y - h.y;
            l.z = o.z - h.z;
            l.w = o.w - h.w;
            reinterpret_cast<float4*>(M + row * npad + base)[lane] = o;
            reinterpret_cast<float4*>(Lhi + row * PW)[lane] = h;
            reinterpret_cast<float4*>(Llo + row * PW)[lane] = l;
        }
    }
}

// ------------------------------------------------------- tensor-core update

struct SyrkBars {
    uint64_t full[STAGES], empty[STAGES], accfull[2], accempty[2], cfull, cempty;
};

// C tile of the output in shared memory: box cc (columns 32cc..32cc+31) holds
// 128 rows of 128 bytes with the 128-byte swizzle (16-byte chunk j of row r
// at position j ^ (r mod 8)), as TMA loads and stores it.
__device__ __forceinline__ float4* c_chunk(unsigned char* cbuf, int cc, int r, int j)
{
    return reinterpret_cast<float4*>(cbuf + cc * BOX_BYTES + r * 128 + ((j ^ (r & 7)) << 4));
}

__global__ void __launch_bounds__(192, 1)
k_syrk_tc(const __grid_constant__ CUtensorMap map_hi, const __grid_constant__ CUtensorMap map_lo,
          const __grid_constant__ CUtensorMap map_c, int t0, int ntiles, unsigned* __restrict__ status)
{
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
        mbar_init(smem_u32(&bars.cfull), 1);
        mbar_init(smem_u32(&bars.cempty), 1);
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

    if (warp == 0) {
        if (lane == 0) {
            // TMA producer of the four K chunks of A/B (hi and lo) per tile
            uint32_t g = 0;
            for (int t = blockIdx.x; t < ntiles && !abort_flag; t += gridDim.x) {
                int ti, tj;
                tri_index(t, ti, tj);
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
        } else if (lane == 1) {
            // TMA producer of the C tile, once the previous one is stored
            uint32_t tl = 0;
            for (int t = blockIdx.x; t < ntiles && !abort_flag; t += gridDim.x, ++tl) {
                int ti, tj;
                tri_index(t, ti, tj);
                const int ra = (t0 + ti) * PW, rb = (t0 + tj) * PW;
                if (!mbar_wait(smem_u32(&bars.cempty), (tl & 1) ^ 1, &abort_flag)) break;
                const uint32_t cb = smem_u32(&bars.cfull);
                mbar_expect_tx(cb, C_BYTES);
                for (int cc = 0; cc < PW / KC; ++cc) tma_load_2d(cbase + cc * BOX_BYTES, &map_c, rb + cc * KC, ra, cb);
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
        // epilogue warps 2..5: TMEM lane quarter = warp % 4
        const int quarter = warp & 3;
        const int rl = 32 * quarter + lane;   // row inside the tile
        uint32_t tl = 0;
        for (int t = blockIdx.x; t < ntiles && !abort_flag; t += gridDim.x, ++tl) {
            int ti, tj;
            tri_index(t, ti, tj);
            const uint32_t b = tl & 1;
            if (!mbar_wait(smem_u32(&bars.accfull[b]), (tl >> 1) & 1, &abort_flag)) break;
            if (!mbar_wait(smem_u32(&bars.cfull), tl & 1, &abort_flag)) break;
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
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    float4* p = c_chunk(cbuf, cc, rl, j);
                    float4 c4 = *p;
                    const int c = 32 * cc + 4 * j;   // column inside the tile
                    const bool diag = ti == tj;
                    if (!diag || c <= rl) c4.x -= __uint_as_float(v[4 * j]);
                    if (!diag || c + 1 <= rl) c4.y -= __uint_as_float(v[4 * j + 1]);
                    if (!diag || c + 2 <= rl) c4.z -= __uint_as_float(v[4 * j + 2]);
                    if (!diag || c + 3 <= rl) c4.w -= __uint_as_float(v[4 * j + 3]);
                    *p = c4;
                }
            }
            // the accumulator is free once all its columns are read
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&bars.accempty[b]));
            // write the tile back with TMA once every epilogue thread is done
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            epi_sync();
            if (tid == 64) {
                const int ra = (t0 + ti) * PW, rb = (t0 + tj) * PW;
                for (int cc = 0; cc < PW / KC; ++cc) tma_store_2d(&map_c, cbase + cc * BOX_BYTES, rb + cc * KC, ra);
                bulk_commit();
                bulk_wait_read0();
                mbar_arrive(smem_u32(&bars.cempty));
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

static PFN_cuTensorMapEncodeTiled_v12000 get_encode()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

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

static int tc_setup(bdb_system* s)
{
    if (s->tc_map_ok) return BDB_OK;
    const size_t pan = (size_t)s->npad * PW;
    if (s->panel64.alloc(pan + PW * PW + 64)) return BDB_ERR_NOMEM;   // hi + lo (FP32 each) + L_PP (FP64)
    float* hi = reinterpret_cast<float*>(s->panel64.p);
    float* lo = hi + pan;
    BDB_CUDA(cudaMemset(s->panel64.p, 0, s->panel64.n * sizeof(double)));
    CUtensorMap* maps = reinterpret_cast<CUtensorMap*>(s->tc_map);
    int rc = make_panel_map(hi, s->npad, &maps[0]);
    if (rc) return rc;
    rc = make_panel_map(lo, s->npad, &maps[1]);
    if (rc) return rc;
    rc = make_panel_map(s->M32.p, s->npad, &maps[2], s->npad);
    if (rc) return rc;
    BDB_CUDA(cudaFuncSetAttribute(k_syrk_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, SYRK_SMEM));
    BDB_CUDA(cudaFuncSetAttribute(k_potrf128, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(PW * LDS * sizeof(double))));
    BDB_CUDA(cudaFuncSetAttribute(k_trsm128, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(PW * PW * sizeof(double))));
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    s->sm_count = sms;
    s->tc_map_ok = true;
    return BDB_OK;
}

int factor_mixed_tc(bdb_system* s)
{
    int rc = tc_setup(s);
    if (rc) return rc;
    const CUtensorMap* maps = reinterpret_cast<const CUtensorMap*>(s->tc_map);
    const size_t pan = (size_t)s->npad * PW;
    float* hi = reinterpret_cast<float*>(s->panel64.p);
    float* lo = hi + pan;
    double* Lkk = reinterpret_cast<double*>(lo + pan);
    const int nt = s->npad / PW;
    for (int P = 0; P < nt; ++P) {
        k_potrf128<<<1, 256, PW * LDS * sizeof(double), s->stream>>>(s->M32.p, s->npad, P, Lkk, s->status.p);
        s->launches += 1;
        const int rows_below = s->npad - (P + 1) * PW;
        if (rows_below <= 0) break;
        const int warps = 16;
        const int blocks = std::min(s->sm_count, (rows_below + warps * TRSM_R - 1) / (warps * TRSM_R));
        k_trsm128<<<blocks, 32 * warps, PW * PW * sizeof(double), s->stream>>>(s->M32.p, s->npad, P, Lkk, hi, lo);
        const int rem = nt - P - 1;
        const int tiles = rem * (rem + 1) / 2;
        const int grid = std::min(s->sm_count, tiles);
        k_syrk_tc<<<grid, 192, SYRK_SMEM, s->stream>>>(maps[0], maps[1], maps[2], P + 1, tiles, s->status.p);
        s->launches += 2;
    }
    BDB_CUDA(cudaGetLastError());
    return BDB_OK;
}

}  // namespace bdb
