// Blocked right-looking Cholesky of the stored diffusion tensor, in place
// in the lower triangle of M (the upper triangle keeps D and is never
// written). This is the device counterpart of my_dpotrf (myblas.c:45-92),
// which the reference calls on the whole 3N x 3N D every step
// (diff_rand.c:64-85). For panel k of NB columns:
//   k_potrf: the NB x NB diagonal block, one thread per row, in FP64;
//   k_trsm:  the panel below, L_ik = A_ik L_kk^-T, one thread per row,
//            forward substitution in FP64 against L_kk in shared memory;
//   k_syrk:  the trailing update A_ij -= L_ik L_jk^T (i >= j > k), 64x64
//            output tiles, 4x4 register blocks per thread.
// T = double is the plain FP64 path; T = float stores FP32 and keeps the
// diagonal blocks and substitutions in FP64 (the SIMT fallback of the
// mixed path; the tcgen05 kernel in chol_tc.cu replaces its k_syrk).
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdlib>

#include "bdb_common.cuh"

namespace bdb {

static constexpr int NB = 64;

template <typename T>
__global__ void __launch_bounds__(NB) k_potrf(T* __restrict__ M, int npad, int k, unsigned* __restrict__ status)
{
    __shared__ double col[NB];
    __shared__ double piv_inv;
    const int r = threadIdx.x;
    const size_t base = (size_t)k * NB;
    double a[NB];
#pragma unroll
    for (int c = 0; c < NB; ++c) a[c] = c <= r ? (double)M[(base + r) * npad + base + c] : 0.0;
    bool bad = false;
#pragma unroll
    for (int j = 0; j < NB; ++j) {
        if (r == j) {
            double d = a[j];
            if (!(d > 0.0)) bad = true;
            d = sqrt(d);
            a[j] = d;
            piv_inv = 1.0 / d;
            col[j] = d;
        }
        __syncthreads();
        if (r > j) {
            a[j] *= piv_inv;
            col[r] = a[j];
        }
        __syncthreads();
        if (r > j) {
#pragma unroll
            for (int c = j + 1; c < NB; ++c)
                if (c <= r) a[c] -= a[j] * col[c];
        }
        __syncthreads();
    }
    if (bad) atomicOr(status, ST_NOT_SPD);
#pragma unroll
    for (int c = 0; c < NB; ++c)
        if (c <= r) M[(base + r) * npad + base + c] = (T)a[c];
}

// rows of the panel below block k: x L_kk^T = a  (x, a row vectors)
template <typename T>
__global__ void __launch_bounds__(128) k_trsm(T* __restrict__ M, int npad, int k)
{
    __shared__ double L[NB][NB + 1];
    __shared__ double dinv[NB];
    const size_t base = (size_t)k * NB;
    for (int idx = threadIdx.x; idx < NB * NB; idx += blockDim.x) {
        const int r = idx / NB, c = idx % NB;
        L[r][c] = c <= r ? (double)M[(base + r) * npad + base + c] : 0.0;
    }
    __syncthreads();
    if (threadIdx.x < NB) dinv[threadIdx.x] = 1.0 / L[threadIdx.x][threadIdx.x];
    __syncthreads();
    const size_t row = base + NB + (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= (size_t)npad) return;
    T* rp = M + row * npad + base;
    double a[NB];
#pragma unroll
    for (int c = 0; c < NB; ++c) a[c] = (double)rp[c];
#pragma unroll
    for (int m = 0; m < NB; ++m) {
        a[m] *= dinv[m];
#pragma unroll
        for (int c = m + 1; c < NB; ++c) a[c] -= L[c][m] * a[m];
    }
#pragma unroll
    for (int c = 0; c < NB; ++c) rp[c] = (T)a[c];
}

// trailing update of the lower triangle: tile (bi, bj), bi >= bj > k
// (only_next: column block k+1 alone, the in-panel update of a 128-wide
// super-panel)
template <typename T>
__global__ void __launch_bounds__(256) k_syrk(T* __restrict__ M, int npad, int k, int only_next)
{
    const int nb_rem = npad / NB - k - 1;
    const int bi = k + 1 + blockIdx.y, bj = k + 1 + blockIdx.x;
    if (blockIdx.x > blockIdx.y || blockIdx.y >= nb_rem) return;
    if (only_next && blockIdx.x != 0) return;
    constexpr int KC = 32;           // panel columns staged per pass
    __shared__ T As[KC][NB + 1];     // As[m][row]
    __shared__ T Bs[KC][NB + 1];
    const size_t pc = (size_t)k * NB;
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    T acc[4][4];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int p = 0; p < 4; ++p) acc[q][p] = 0;
    for (int m0 = 0; m0 < NB; m0 += KC) {
        __syncthreads();
        for (int idx = tid; idx < NB * KC; idx += 256) {
            const int r = idx / KC, m = idx % KC;
            As[m][r] = M[((size_t)bi * NB + r) * npad + pc + m0 + m];
            Bs[m][r] = M[((size_t)bj * NB + r) * npad + pc + m0 + m];
        }
        __syncthreads();
#pragma unroll 8
        for (int m = 0; m < KC; ++m) {
            T a[4], b[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                a[q] = As[m][ty + 16 * q];
                b[q] = Bs[m][tx + 16 * q];
            }
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int p = 0; p < 4; ++p) acc[q][p] += a[q] * b[p];
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int r = ty + 16 * q;
        T* crow = M + ((size_t)bi * NB + r) * npad + (size_t)bj * NB;
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const int c = tx + 16 * p;
            if (bi != bj || c <= r) crow[c] -= acc[q][p];
        }
    }
}

int factor_mixed_tc(bdb_system* s);   // chol_tc.cu
int factor_fp64_tc(bdb_system* s);    // chol_tc.cu

int factor_run(bdb_system* s)
{
    // BDB_NO_TC (diagnostics): the SIMT kernels below instead of the
    // tensor-core factorisations of chol_tc.cu
    const bool no_tc = getenv("BDB_NO_TC") != nullptr;
    if (!no_tc && s->npad % 128 == 0)
        return s->p.precision == BDB_PREC_MIXED ? factor_mixed_tc(s) : factor_fp64_tc(s);
    const int nb = s->npad / NB;
    for (int k = 0; k < nb; ++k) {
        const int rows_below = s->npad - (k + 1) * NB;
        if (s->p.precision == BDB_PREC_FP64) {
            k_potrf<double><<<1, NB, 0, s->stream>>>(s->M64.p, s->npad, k, s->status.p);
            if (rows_below > 0) {
                k_trsm<double><<<(rows_below + 127) / 128, 128, 0, s->stream>>>(s->M64.p, s->npad, k);
                dim3 g(nb - k - 1, nb - k - 1);
                k_syrk<double><<<g, 256, 0, s->stream>>>(s->M64.p, s->npad, k, 0);
            }
        } else {
            k_potrf<float><<<1, NB, 0, s->stream>>>(s->M32.p, s->npad, k, s->status.p);
            if (rows_below > 0) {
                k_trsm<float><<<(rows_below + 127) / 128, 128, 0, s->stream>>>(s->M32.p, s->npad, k);
                dim3 g(nb - k - 1, nb - k - 1);
                k_syrk<float><<<g, 256, 0, s->stream>>>(s->M32.p, s->npad, k, 0);
            }
        }
    }
    s->launches += 3 * nb - 2;
    BDB_CUDA(cudaGetLastError());
    return BDB_OK;
}

// ||L L^T - D||_F / ||D||_F in FP64 over 64x64 tiles (bi >= bj) of the
// lower triangle: L from the lower triangle of M, D from its upper triangle
// (mirrored) and dD on the diagonal.
template <typename T>
__global__ void __launch_bounds__(256) k_llt_err(const T* __restrict__ M, const double* __restrict__ dD, int n3,
                                                 int npad, double* __restrict__ acc)
{
    const int bi = blockIdx.y, bj = blockIdx.x;
    if (bj > bi) return;
    constexpr int KC = 32;
    __shared__ double As[KC][NB + 1];
    __shared__ double Bs[KC][NB + 1];
    __shared__ double red[2][8];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    double s[4][4];
    for (int q = 0; q < 4; ++q)
        for (int p = 0; p < 4; ++p) s[q][p] = 0;
    const int mend = (bj + 1) * NB;   // L[c][m] = 0 beyond the column block's diagonal
    for (int m0 = 0; m0 < mend; m0 += KC) {
        __syncthreads();
        for (int idx = tid; idx < NB * KC; idx += 256) {
            const int r = idx / KC, m = idx % KC;
            const int gr = bi * NB + r, gc = bj * NB + r, gm = m0 + m;
            As[m][r] = (gm <= gr && gr < n3) ? (double)M[(size_t)gr * npad + gm] : 0.0;
            Bs[m][r] = (gm <= gc && gc < n3) ? (double)M[(size_t)gc * npad + gm] : 0.0;
        }
        __syncthreads();
        for (int m = 0; m < KC; ++m)
            for (int q = 0; q < 4; ++q)
                for (int p = 0; p < 4; ++p) s[q][p] += As[m][ty + 16 * q] * Bs[m][tx + 16 * p];
    }
    double num = 0, den = 0;
    for (int q = 0; q < 4; ++q)
        for (int p = 0; p < 4; ++p) {
            const int r = bi * NB + ty + 16 * q, c = bj * NB + tx + 16 * p;
            if (r >= n3 || c >= n3 || c > r) continue;
            const double d = r == c ? dD[r] : (double)M[(size_t)c * npad + r];
            const double w = r == c ? 1.0 : 2.0;
            num += w * (s[q][p] - d) * (s[q][p] - d);
            den += w * d * d;
        }
    for (int o = 16; o > 0; o >>= 1) {
        num += __shfl_xor_sync(0xffffffffu, num, o);
        den += __shfl_xor_sync(0xffffffffu, den, o);
    }
    if ((tid & 31) == 0) {
        red[0][tid >> 5] = num;
        red[1][tid >> 5] = den;
    }
    __syncthreads();
    if (tid == 0) {
        double a = 0, b = 0;
        for (int w = 0; w < 8; ++w) {
            a += red[0][w];
            b += red[1][w];
        }
        atomicAdd(&acc[0], a);
        atomicAdd(&acc[1], b);
    }
}

int factor_error(bdb_system* s, double* rel)
{
    double* acc = s->scal.p + 40;
    BDB_CUDA(cudaMemsetAsync(acc, 0, 2 * sizeof(double), s->stream));
    const int nb = (s->n3 + NB - 1) / NB;
    dim3 grid(nb, nb);
    if (s->p.precision == BDB_PREC_FP64)
        k_llt_err<double><<<grid, 256, 0, s->stream>>>(s->M64.p, s->dD.p, s->n3, s->npad, acc);
    else
        k_llt_err<float><<<grid, 256, 0, s->stream>>>(s->M32.p, s->dD.p, s->n3, s->npad, acc);
    BDB_CUDA(cudaGetLastError());
    double h[2];
    BDB_CUDA(cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
    BDB_CUDA(cudaStreamSynchronize(s->stream));
    *rel = sqrt(h[0] / h[1]);
    return BDB_OK;
}

}  // namespace bdb
