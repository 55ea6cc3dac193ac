// Diffusion tensor on the device.
//
// 1. k_build: the stored 3N x 3N tensor of compute_D (diff_tensor.c:472-544)
//    for the Cholesky path. One CTA per 32x32-bead tile (I >= J) evaluates
//    the 1024 RPY tiles into shared memory and writes the 96x96 block twice
//    with coalesced rows: as rows of block (I, J) below the diagonal and,
//    transposed through shared memory, as rows of block (J, I) above it.
//    The factorisation later overwrites the lower triangle with L; the upper
//    triangle keeps D (the reference keeps Ds and S separately,
//    diff_rand.c:76-82). The diagonal of D goes to dD.
// 2. k_tea: matrix-free D.F (compute_Rf_geyer_in_fly, diff_equation.c:55-117)
//    and the Geyer-Winter sums C_i, Feff_i, eps (compute_r DIFF_GEYER,
//    diff_rand.c:86-196) in one pass over tile pairs (I >= J): every bead
//    pair is evaluated once, staged in shared memory, and summed by rows
//    (into bead i) and by columns (into bead j). Per (tile, bead) partials
//    go to a scratch buffer that k_tea_finish reduces in a fixed order, so
//    the result does not depend on scheduling.
// 3. k_eps_beta + k_tea_finish: eps -> beta (diff_rand.c:197-217), the TEA
//    displacement (:219-228) and the position update with the periodic wrap
//    (compute_hydro_ermak, diff_equation.c:254-264), fused.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "bdb_common.cuh"
#include "rpy_tile.cuh"

namespace bdb {

static constexpr int TB = 32;   // beads per tile

struct TensorArgs {
    int n, npad;
    double preDii, preDij;
    int ewald;
    EwaldConst ec;
};

// Lattice tables of the Ewald sums (see EwaldConst), built once per system
// in the order diff_tensor_calc_ewald_beenakker walks the sphere |m|^2 <= R^2
// (diff_tensor.c:319-326); the k-only factors of the reciprocal term are
// evaluated as the device evaluates them per pair.
static EwaldConst system_ewald(const bdb_system* s)
{
    if (s->p.ewald_method == BDB_EWALD_SMITH)
        return make_ewald_smith(s->p.box[0], s->inv_L[0], s->p.ewald_real,
                                s->p.ewald_alpha > 0 ? s->p.ewald_alpha : BDB_SQRTPI);
    return make_ewald(s->p.box[0], s->inv_L[0], s->p.ewald_real);
}

static int ewald_tables(bdb_system* s)
{
    if (!s->p.ewald || s->ewald_tab.p) return BDB_OK;
    const EwaldConst ec = system_ewald(s);
    // Smith's k-only factors (diff_tensor.c:206-239 with init_tensor's
    // M_PI_ALPHA_SQ = -pi_f^2/alpha^2, pi_f^2 formed in float)
    volatile float pif = BDB_M_PIF;
    volatile float npif2 = -pif * pif;
    volatile float four_pif = 4 * pif;
    const double m_pi_alpha_sq = ec.smith ? (double)npif2 / ec.s_alpha2 : 0.0;
    const double preO = 0.75 * ec.inv_L;
    const double qL3 = ec.inv_L * ec.inv_L * ec.inv_L;
    std::vector<double> rk, img;
    const int R = ec.R;
    for (int h = -R; h <= R; ++h) {
        const int nf = (int)std::sqrt((double)(ec.rr_sq - h * h));
        for (int f = -nf; f <= nf; ++f) {
            const int ng = (int)std::sqrt((double)(ec.rr_sq - h * h - f * f));
            for (int g = -ng; g <= ng; ++g) {
                img.insert(img.end(), {ec.L * h, ec.L * f, ec.L * g, 0.0});
                const bool half = h > 0 || (h == 0 && (f > 0 || (f == 0 && g > 0)));
                if (!half) continue;
                const double k_sq = (double)(h * h + f * f + g * g);
                const double kn = std::sqrt(k_sq), ik = 1 / kn;
                const double e[3] = {h * ik, f * ik, g * ik};
                if (ec.smith) {
                    // Op: A (I + (m k^2 - 1) e e^T), Qp: C e e^T, both times cos;
                    // k and -k together: 2x
                    const double ex = std::exp(m_pi_alpha_sq * k_sq);
                    const double A = 2 * ex / ((double)pif * k_sq);
                    const double C = (double)four_pif * ex;
                    rk.insert(rk.end(), {(double)h, (double)f, (double)g, 2 * preO * A,
                                         2 * preO * A * (-1 + m_pi_alpha_sq * k_sq), 2 * 0.5 * qL3 * C,
                                         e[0] * e[0], e[1] * e[1], e[2] * e[2], e[0] * e[1], e[0] * e[2], e[1] * e[2]});
                    continue;
                }
                const double k2 = k_sq * ec.four_pif2;
                double P = 1 + (ec.inv_alpha2 * k2 / 4) * (1 + ec.inv_alpha2 * k2 / 2);
                P *= ec.six_pif * std::exp(-ec.inv_alpha2 * k2 / 4) / k2;
                rk.insert(rk.end(), {(double)h, (double)f, (double)g, P, k2 / 3 * P, 2 * (1 - e[0] * e[0]),
                                     2 * (1 - e[1] * e[1]), 2 * (1 - e[2] * e[2]), -2 * e[0] * e[1], -2 * e[0] * e[2],
                                     -2 * e[1] * e[2], 0.0});
            }
        }
    }
    s->ewald_nk = (int)(rk.size() / 12);
    s->ewald_nimg = (int)(img.size() / 4);
    if (s->ewald_tab.alloc(rk.size() + img.size())) return BDB_ERR_NOMEM;
    if (!rk.empty())
        BDB_CUDA(h2d(s, s->ewald_tab.p, rk.data(), sizeof(double) * rk.size()));
    BDB_CUDA(h2d(s, s->ewald_tab.p + rk.size(), img.data(), sizeof(double) * img.size()));
    return BDB_OK;
}

static TensorArgs targs(const bdb_system* s)
{
    TensorArgs a;
    a.n = s->n;
    a.npad = s->npad;
    a.preDii = s->preDii;
    a.preDij = s->preDij;
    a.ewald = s->p.ewald;
    a.ec = system_ewald(s);
    if (s->p.ewald) {
        a.ec.rk = s->ewald_tab.p;
        a.ec.nk = s->ewald_nk;
        a.ec.img = reinterpret_cast<const double4*>(s->ewald_tab.p + 12 * (size_t)s->ewald_nk);
        a.ec.nimg = s->ewald_nimg;
        const double rc = 2.5 * s->p.box[0];   // erfc(2.5 sqrt(pi)) ~ 3e-10
        a.ec.rcut_sq = (float)(rc * rc);
    }
    return a;
}

template <typename T, bool kEwald>
__device__ __forceinline__ void tile_of_k(const TensorArgs& A, const double4* pos, int i, int j, T* t)
{
    const double4 pi = pos[i], pj = pos[j];
    if constexpr (kEwald) {
        double d[6];
        if (A.ec.smith)
            rpy_smith_tab<sizeof(T) == 4>(pi, pj, i == j, A.preDii, A.preDij, A.ec, d);
        else
            rpy_ewald_tab<sizeof(T) == 4>(pi, pj, i == j, A.preDii, A.preDij, A.ec, d);
        for (int k = 0; k < 6; ++k) t[k] = (T)d[k];
    } else if (i == j) {
        const T d = (T)(A.preDii / pi.w);
        t[0] = t[1] = t[2] = d;
        t[3] = t[4] = t[5] = 0;
    } else if (i > j) {
        rpy_free<T>(pi, pj, (T)A.preDii, (T)A.preDij, t);
    } else {
        rpy_free<T>(pj, pi, (T)A.preDii, (T)A.preDij, t);
    }
}

template <typename T>
__device__ __forceinline__ void tile_of(const TensorArgs& A, const double4* pos, int i, int j, T* t)
{
    if (A.ewald)
        tile_of_k<T, true>(A, pos, i, j, t);
    else
        tile_of_k<T, false>(A, pos, i, j, t);
}

// One CTA per pair of 32-bead blocks (I >= J): the 96x96 tile of D in
// shared memory, then stored straight and (off the diagonal) transposed,
// both triangles, one warp per matrix row so that every store of a warp is
// one contiguous run of the row. The free-space variant (kEwald false)
// carries none of the Ewald code, so it keeps few registers and several
// CTAs per SM.
template <typename T, bool kEwald>
__global__ void __launch_bounds__(256) k_build(TensorArgs A, const double4* __restrict__ pos, T* __restrict__ M,
                                               double* __restrict__ dD)
{
    extern __shared__ __align__(16) unsigned char build_smem[];
    T(*tile)[3 * TB + 1] = reinterpret_cast<T(*)[3 * TB + 1]>(build_smem);
    const int I = blockIdx.y, J = blockIdx.x;
    if (J > I) return;
    const int tid = threadIdx.x;
    const int n3 = 3 * A.n;
    for (int p = tid; p < TB * TB; p += blockDim.x) {
        const int li = p / TB, lj = p % TB;
        const int i = I * TB + li, j = J * TB + lj;
        T t[6] = {0, 0, 0, 0, 0, 0};
        if (i < A.n && j < A.n) tile_of_k<T, kEwald>(A, pos, i, j, t);
        const int r = 3 * li, c = 3 * lj;
        tile[r][c] = t[0];
        tile[r + 1][c + 1] = t[1];
        tile[r + 2][c + 2] = t[2];
        tile[r][c + 1] = tile[r + 1][c] = t[3];
        tile[r][c + 2] = tile[r + 2][c] = t[4];
        tile[r + 1][c + 2] = tile[r + 2][c + 1] = t[5];
    }
    __syncthreads();
    const int r0 = 3 * TB * I, c0 = 3 * TB * J;
    const int warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
    const int rows = min(3 * TB, n3 - r0), cols = min(3 * TB, n3 - c0);
    for (int r = warp; r < rows; r += nw) {
        T* dst = M + (size_t)(r0 + r) * A.npad + c0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int c = lane + 32 * k;
            if (c < cols) dst[c] = tile[r][c];
        }
    }
    if (I != J) {
        for (int c = warp; c < cols; c += nw) {
            T* dst = M + (size_t)(c0 + c) * A.npad + r0;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int r = lane + 32 * k;
                if (r < rows) dst[r] = tile[r][c];
            }
        }
    } else {
        for (int r = tid; r < 3 * TB; r += blockDim.x)
            if (r0 + r < n3) dD[r0 + r] = (double)tile[r][r];
    }
}

template <typename T>
static size_t build_smem_bytes()
{
    return sizeof(T) * 3 * TB * (3 * TB + 1);
}


static int tensor_attrs();

int tensor_build(bdb_system* s)
{
    int rc = tensor_attrs();
    if (rc) return rc;
    if (int rc_e = ewald_tables(s)) return rc_e;
    const TensorArgs A = targs(s);
    const int nt = (s->n + TB - 1) / TB;
    dim3 grid(nt, nt);
    if (s->p.precision == BDB_PREC_FP64) {
        if (A.ewald)
            k_build<double, true><<<grid, 256, build_smem_bytes<double>(), s->stream>>>(A, s->pos.p, s->M64.p, s->dD.p);
        else
            k_build<double, false><<<grid, 256, build_smem_bytes<double>(), s->stream>>>(A, s->pos.p, s->M64.p,
                                                                                        s->dD.p);
    } else {
        if (A.ewald)
            k_build<float, true><<<grid, 256, build_smem_bytes<float>(), s->stream>>>(A, s->pos.p, s->M32.p, s->dD.p);
        else
            k_build<float, false><<<grid, 256, build_smem_bytes<float>(), s->stream>>>(A, s->pos.p, s->M32.p, s->dD.p);
    }
    s->launches += 1;
    BDB_CUDA(cudaGetLastError());
    return BDB_OK;
}

__global__ void k_one_tile(TensorArgs A, const double4* pos, int i, int j, double* out)
{
    double t[6];
    tile_of<double>(A, pos, i, j, t);
    out[0] = t[0];
    out[4] = t[1];
    out[8] = t[2];
    out[1] = out[3] = t[3];
    out[2] = out[6] = t[4];
    out[5] = out[7] = t[5];
}

int tensor_tile_host(bdb_system* s, int i, int j, double* tD)
{
    if (int rc_e = ewald_tables(s)) return rc_e;
    const TensorArgs A = targs(s);
    double* d = s->work.p;
    k_one_tile<<<1, 1, 0, s->stream>>>(A, s->pos.p, i, j, d);
    BDB_CUDA(cudaGetLastError());
    BDB_CUDA(cudaMemcpyAsync(tD, d, 9 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    BDB_CUDA(cudaStreamSynchronize(s->stream));
    return BDB_OK;
}

// ------------------------------------------------------------------ TEA

// part layout: record (9 doubles: Rf[3], C[3], Feff[3]) for (tile_other T,
// bead b) of segment g at index  g.part_begin + T * g.count + (b - g.begin).
struct TeaSeg {
    int begin, count, ntile, part_begin;
};

// One job = the tile pair (I, J) of a segment (TT x TT beads). Warp w holds
// rows li of the pair (32 / TT rows at a time, one lane per column lj); each
// lane evaluates its tile D_ij in registers and uses it twice: in the row
// sums of bead i (a shuffle tree over the row's lanes) and in the column
// sums of bead j (accumulated by the lane over the rows it visits, then the
// warps' partials added in warp order through shared memory). The tiles never
// go through shared memory. Within a job the sums run in T (FP32 on the mixed
// path); the records they produce and every sum across jobs are FP64. The
// free-space variant (kEwald false) carries none of the lattice-sum code.
// The grid is persistent, as many CTAs as the SMs hold: each CTA takes the
// next job of the whole batch (every replica's tile pairs in one list) from
// a counter until none is left -- fetching its next job while it works on
// the current one -- so replicas of uneven size share the GPU in one launch
// and a CTA that drew short jobs draws more. A job writes only its own
// records, so which CTA runs it does not change a bit.
template <typename T, int TT, bool kEwald>
__global__ void __launch_bounds__(256)
k_tea(TensorArgs A, const TileJob* __restrict__ jobs, int n_jobs, int* __restrict__ next,
      const TeaSeg* __restrict__ segs, const double4* __restrict__ pos, const double* __restrict__ F,
      const double* __restrict__ X, double* __restrict__ part, double* __restrict__ eps_part, int want_rs)
{
    constexpr int NW = 8;              // warps
    constexpr int RPW = 32 / TT;       // rows a warp holds at once
    constexpr int RSTEP = NW * RPW;    // rows of one pass of the block
    static_assert(TT == 16 || TT == 32, "tile edge");
    __shared__ T sF[2][TT][3], sX[2][TT][3], sInv[2][TT];
    __shared__ T sCol[NW][TT][9];      // the warps' column partials
    __shared__ T sRowDiag[TT][9];      // diagonal job: row sums, added to the column records
    __shared__ double sEps[NW];
    __shared__ int sJob[2];
    if (threadIdx.x == 0) sJob[0] = atomicAdd(next, 1);
    __syncthreads();
    int slot = 0;
    for (int job = sJob[0]; job < n_jobs; job = sJob[slot]) {
    // the next job, read after this one's last barrier
    if (threadIdx.x == 0) sJob[slot ^ 1] = atomicAdd(next, 1);
    const TileJob jb = jobs[job];
    const TeaSeg g = segs[jb.seg];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int bi0 = g.begin + jb.I * TT, bj0 = g.begin + jb.J * TT;
    const int ni = min(TT, g.count - jb.I * TT), nj = min(TT, g.count - jb.J * TT);
    const bool diag = jb.I == jb.J;
    if (tid < TT) {
        for (int side = 0; side < 2; ++side) {
            const int b = (side ? bj0 : bi0) + tid;
            const bool ok = tid < (side ? nj : ni);
            for (int k = 0; k < 3; ++k) {
                sF[side][tid][k] = ok ? (T)F[3 * b + k] : (T)0;
                sX[side][tid][k] = ok && want_rs ? (T)X[3 * b + k] : (T)0;
            }
            sInv[side][tid] = ok ? (T)(pos[b].w / A.preDii) : (T)0;   // 1/diag_D (diff_decl.c:94-99)
        }
    }
    __syncthreads();
    const int lj = lane % TT, sub = lane / TT;
    const T* fc = sF[1][lj];
    const T* xc = sX[1][lj];
    const T invc = sInv[1][lj];
    T col[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    T eps = 0;
#pragma unroll 1
    for (int r0 = 0; r0 < TT; r0 += RSTEP) {
        const int li = r0 + warp * RPW + sub;
        T t[6] = {0, 0, 0, 0, 0, 0};
        if (li < ni && lj < nj && (!diag || lj < li)) tile_of_k<T, kEwald>(A, pos, bi0 + li, bj0 + lj, t);
        const T xx = t[0], yy = t[1], zz = t[2], xy = t[3], xz = t[4], yz = t[5];
        // bead li: products with bead lj's F, X and 1/D_jj
        T row[9];
        row[0] = xx * fc[0] + xy * fc[1] + xz * fc[2];
        row[1] = xy * fc[0] + yy * fc[1] + yz * fc[2];
        row[2] = xz * fc[0] + yz * fc[1] + zz * fc[2];
        row[3] = (xx * xx + xy * xy + xz * xz) * invc;
        row[4] = (xy * xy + yy * yy + yz * yz) * invc;
        row[5] = (xz * xz + yz * yz + zz * zz) * invc;
        row[6] = xx * xc[0] + xy * xc[1] + xz * xc[2];
        row[7] = xy * xc[0] + yy * xc[1] + yz * xc[2];
        row[8] = xz * xc[0] + yz * xc[1] + zz * xc[2];
        eps += xx + yy + zz + 2 * (xy + xz + yz);
        // bead lj: products with bead li's
        const T* fr = sF[0][li];
        const T* xr = sX[0][li];
        const T invr = sInv[0][li];
        col[0] += xx * fr[0] + xy * fr[1] + xz * fr[2];
        col[1] += xy * fr[0] + yy * fr[1] + yz * fr[2];
        col[2] += xz * fr[0] + yz * fr[1] + zz * fr[2];
        col[3] += (xx * xx + xy * xy + xz * xz) * invr;
        col[4] += (xy * xy + yy * yy + yz * yz) * invr;
        col[5] += (xz * xz + yz * yz + zz * zz) * invr;
        col[6] += xx * xr[0] + xy * xr[1] + xz * xr[2];
        col[7] += xy * xr[0] + yy * xr[1] + yz * xr[2];
        col[8] += xz * xr[0] + yz * xr[1] + zz * xr[2];
#pragma unroll
        for (int o = 1; o < TT; o <<= 1)
#pragma unroll
            for (int k = 0; k < 9; ++k) row[k] += __shfl_xor_sync(0xffffffffu, row[k], o);
        if (lj == 0 && li < ni) {
            if (diag) {
                for (int k = 0; k < 9; ++k) sRowDiag[li][k] = row[k];
            } else {
                // record (T = J, bead in I)
                double* dst = part + 9 * ((size_t)g.part_begin + (size_t)jb.J * g.count + jb.I * TT + li);
                for (int k = 0; k < 9; ++k) dst[k] = (double)row[k];
            }
        }
    }
    if constexpr (RPW == 2) {
#pragma unroll
        for (int k = 0; k < 9; ++k) col[k] += __shfl_xor_sync(0xffffffffu, col[k], 16);
    }
    if (sub == 0)
        for (int k = 0; k < 9; ++k) sCol[warp][lj][k] = col[k];
    {
        double e = (double)eps;
        for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
        if (lane == 0) sEps[warp] = e;
    }
    __syncthreads();
    if (tid == 0) {
        double e = 0;
        for (int w = 0; w < NW; ++w) e += sEps[w];
        eps_part[job] = e;
    }
    // column records (T = I, bead in J), the warps' partials in order; on a
    // diagonal job the row sums of the same bead join them
    for (int q = tid; q < TT * 9; q += blockDim.x) {
        const int c = q / 9, k = q % 9;
        if (c < nj) {
            T a = 0;
            for (int w = 0; w < NW; ++w) a += sCol[w][c][k];
            double v = (double)a;
            if (diag) v += (double)sRowDiag[c][k];
            part[9 * ((size_t)g.part_begin + (size_t)jb.I * g.count + jb.J * TT + c) + k] = v;
        }
    }
    __syncthreads();   // the job's shared arrays are read; the next job may write them
    slot ^= 1;
    }
}

// eps -> beta per segment (diff_rand.c:197-217); scal[4g+0] = eps, [4g+1] = beta
__global__ void k_eps_beta(const TeaSeg* __restrict__ segs, const int* __restrict__ job_begin,
                           const double* __restrict__ eps_part, double* __restrict__ scal, unsigned* status)
{
    __shared__ double sh[256];
    const TeaSeg g = segs[blockIdx.x];
    const int b = job_begin[blockIdx.x], e = job_begin[blockIdx.x + 1];
    double a = 0;
    for (int k = b + threadIdx.x; k < e; k += blockDim.x) a += eps_part[k];
    sh[threadIdx.x] = a;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const int n3 = 3 * g.count;
        double eps = sh[0];
        eps /= n3;
        eps /= (n3 - 1);
        eps *= 2;
        if (eps > 1.0) eps = 1.0;
        const double aa = (3 * g.count - 1) * eps * eps - (3 * g.count - 2) * eps;
        double beta;
        if (fabs(aa) < (double)0.0000001f) beta = 0.5;
        else beta = (1 - sqrt(1 - aa)) / aa;
        scal[4 * blockIdx.x] = eps;
        scal[4 * blockIdx.x + 1] = beta;
    }
}

__global__ void k_tea_finish(TensorArgs A, int n, const TeaSeg* __restrict__ segs, const int* __restrict__ bead_seg,
                             const double* __restrict__ part, const double* __restrict__ scal,
                             const double4* __restrict__ pos_in, const double* __restrict__ F,
                             const double* __restrict__ X, double pre_f, int want_rs, int hydro,
                             double* __restrict__ Rf, double* __restrict__ Rs)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int gi = bead_seg[i];
    const TeaSeg g = segs[gi];
    const int local = i - g.begin;
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (hydro) {
        for (int T = 0; T < g.ntile; ++T) {
            const double* src = part + 9 * ((size_t)g.part_begin + (size_t)T * g.count + local);
            for (int k = 0; k < 9; ++k) acc[k] += src[k];
        }
    }
    // self tile: D.F uses only its diagonal (diff_equation.c:96-102)
    double self[6];
    tile_of<double>(A, pos_in, i, i, self);
    const double d = A.preDii / pos_in[i].w;   // diag_D (diff_decl.c:94-99)
    const double inv_d = 1 / d;
    for (int k = 0; k < 3; ++k) {
        double rf = hydro ? acc[k] + F[3 * i + k] * self[k] : d * F[3 * i + k];
        Rf[3 * i + k] = hydro ? rf * pre_f : pre_f * d * F[3 * i + k];
    }
    if (want_rs && !hydro) {
        // DIFF_NONE (diff_rand.c:55-63): X already carries sqrt(2 dt D_ii)
        for (int k = 0; k < 3; ++k) Rs[3 * i + k] = X[3 * i + k];
    } else if (want_rs) {
        const double beta = scal[4 * gi + 1];
        for (int k = 0; k < 3; ++k) {
            double c = acc[3 + k] * (beta * beta * inv_d);
            c = 1 / (1 + c);
            c = sqrt(c);
            Rs[3 * i + k] = c * (beta * acc[6 + k] + d * X[3 * i + k]);
        }
    }
}

int tea_setup(bdb_system* s);

template <int TT>
static void tea_launch(bdb_system* s, const TensorArgs& A, const TeaSeg* tsegs, bool want_rs)
{
    // persistent grid: the SMs' capacity for this variant, at most one CTA per job
    auto go = [&](auto kern) {
        int occ = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 256, 0);
        const int grid = std::max(1, std::min(s->n_jobs, std::max(1, occ) * s->sm_count));
        cudaMemsetAsync(s->tea_next.p, 0, sizeof(int), s->stream);
        kern<<<grid, 256, 0, s->stream>>>(A, s->jobs.p, s->n_jobs, s->tea_next.p, tsegs, s->pos.p, s->F.p, s->X.p,
                                          s->part.p, s->eps_part.p, want_rs);
    };
    if (s->p.precision == BDB_PREC_FP64) {
        if (A.ewald) go(k_tea<double, TT, true>);
        else go(k_tea<double, TT, false>);
    } else {
        if (A.ewald) go(k_tea<float, TT, true>);
        else go(k_tea<float, TT, false>);
    }
}

static void tea_dispatch(bdb_system* s, const TensorArgs& A, const TeaSeg* tsegs, bool want_rs)
{
    if (s->tea_tile == 16) tea_launch<16>(s, A, tsegs, want_rs);
    else tea_launch<32>(s, A, tsegs, want_rs);
}

// Autotuning of the TEA tile (16 or 32 beads): each candidate's work list
// is built and its pair kernel timed twice on the system's stream; the
// faster one is kept. Runs at the first TEA call of a system with
// autotuning on (which comes before any graph capture).
static int tea_tune(bdb_system* s, bool want_rs)
{
    const int cands[2] = {16, 32};
    float best_ms = 1e30f;
    int best = s->tea_tile;
    cudaEvent_t e0, e1;
    BDB_CUDA(cudaEventCreate(&e0));
    BDB_CUDA(cudaEventCreate(&e1));
    for (int c : cands) {
        s->tea_tile = c;
        int rc = tea_setup(s);
        if (rc) return rc;
        if (int rc_e = ewald_tables(s)) return rc_e;
        const TensorArgs A = targs(s);
        const TeaSeg* tsegs = reinterpret_cast<const TeaSeg*>(s->tea_meta.p);
        tea_dispatch(s, A, tsegs, want_rs);   // warm-up
        BDB_CUDA(cudaEventRecord(e0, s->stream));
        tea_dispatch(s, A, tsegs, want_rs);
        tea_dispatch(s, A, tsegs, want_rs);
        BDB_CUDA(cudaEventRecord(e1, s->stream));
        BDB_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        BDB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        s->launches += 3;
        if (ms < best_ms) {
            best_ms = ms;
            best = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    s->tea_tile = best;
    s->tea_tuned = true;
    return tea_setup(s);
}

int tea_run(bdb_system* s, bool want_rs)
{
    int rc0 = tensor_attrs();
    if (rc0) return rc0;
    if (s->autotune && !s->tea_tuned && s->p.hydro && s->n_jobs >= 0) {
        int rc = tea_tune(s, want_rs);
        if (rc) return rc;
    } else if (!s->tea_meta.p) {
        int rc = tea_setup(s);
        if (rc) return rc;
    }
    if (int rc_e = ewald_tables(s)) return rc_e;
    const TensorArgs A = targs(s);
    TeaSeg* tsegs = reinterpret_cast<TeaSeg*>(s->tea_meta.p);
    if (s->p.hydro && s->n_jobs) {
        tea_dispatch(s, A, tsegs, want_rs);
        BDB_CUDA(cudaGetLastError());
        if (want_rs) {
            const int* job_begin = reinterpret_cast<const int*>(tsegs + s->segs.size());
            k_eps_beta<<<(int)s->segs.size(), 256, 0, s->stream>>>(tsegs, job_begin, s->eps_part.p, s->scal.p + 64,
                                                                   s->status.p);
            BDB_CUDA(cudaGetLastError());
        }
    }
    s->launches += 1 + ((s->p.hydro && s->n_jobs) ? (want_rs ? 2 : 1) : 0);
    const double pre_f = s->p.dt / (BDB_KB * s->p.T);
    k_tea_finish<<<(s->n + 127) / 128, 128, 0, s->stream>>>(A, s->n, tsegs, s->d_bead_seg.p, s->part.p, s->scal.p + 64,
                                                            s->pos.p, s->F.p, s->X.p, pre_f, want_rs,
                                                            s->p.hydro, s->Rf.p, s->Rs.p);
    BDB_CUDA(cudaGetLastError());
    return BDB_OK;
}

// Work list and scratch layout for k_tea: the TeaSeg table followed by the
// per-segment job offsets, in tea_meta.
int tea_setup(bdb_system* s)
{
    std::vector<TileJob> jobs;
    std::vector<TeaSeg> ts;
    std::vector<int> job_begin;
    size_t part_records = 0;
    for (size_t g = 0; g < s->segs.size(); ++g) {
        const Segment& sg = s->segs[g];
        TeaSeg t;
        t.begin = sg.begin;
        t.count = sg.count;
        t.ntile = (sg.count + s->tea_tile - 1) / s->tea_tile;
        t.part_begin = (int)part_records;
        part_records += (size_t)t.ntile * sg.count;
        ts.push_back(t);
        job_begin.push_back((int)jobs.size());
        for (int I = 0; I < t.ntile; ++I)
            for (int J = 0; J <= I; ++J) jobs.push_back(TileJob{(int)g, I, J});
    }
    job_begin.push_back((int)jobs.size());
    s->n_jobs = (int)jobs.size();
    if (s->jobs.alloc(std::max<size_t>(1, jobs.size()))) return BDB_ERR_NOMEM;
    if (!s->tea_next.p && s->tea_next.alloc(1)) return BDB_ERR_NOMEM;
    if (s->eps_part.alloc(std::max<size_t>(1, jobs.size()))) return BDB_ERR_NOMEM;
    if (s->part.alloc(std::max<size_t>(9, 9 * part_records))) return BDB_ERR_NOMEM;
    const size_t head = sizeof(TeaSeg) * ts.size() + sizeof(int) * job_begin.size();
    if (s->tea_meta.alloc(head)) return BDB_ERR_NOMEM;
    BDB_CUDA(h2d(s, s->jobs.p, jobs.data(), sizeof(TileJob) * jobs.size()));
    BDB_CUDA(h2d(s, s->tea_meta.p, ts.data(), sizeof(TeaSeg) * ts.size()));
    BDB_CUDA(h2d(s, s->tea_meta.p + sizeof(TeaSeg) * ts.size(), job_begin.data(), sizeof(int) * job_begin.size()));
    return BDB_OK;
}

static int tensor_attrs()
{
    static bool done = false;
    if (done) return BDB_OK;
    BDB_CUDA(cudaFuncSetAttribute(k_build<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)build_smem_bytes<double>()));
    BDB_CUDA(cudaFuncSetAttribute(k_build<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)build_smem_bytes<double>()));
    BDB_CUDA(cudaFuncSetAttribute(k_build<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)build_smem_bytes<float>()));
    BDB_CUDA(cudaFuncSetAttribute(k_build<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)build_smem_bytes<float>()));
    done = true;
    return BDB_OK;
}

}  // namespace bdb
