// Forces: compute_forces (potentials/calc_func.c:106-186) on the device.
//
// * Cell lists: one CTA per segment (an independent system of a batch)
//   computes the bounding box (free space) or the periodic grid, keys every
//   bead by its cell and sorts (cell, bead) pairs in shared memory. A bead
//   then finds each of its 27 neighbour cells by binary search in the sorted
//   keys -- no per-cell arrays, so a sparse free-space chain costs O(N).
//   Cells are the widest cutoff plus a skin, and a segment is re-sorted only
//   after some bead has moved more than skin/2 since the last sort (each bead
//   looks up its current cell, and every partner within the cutoff is still
//   in an adjacent cell of the stored list), so most steps skip the sort.
//   This replaces bucket_space / bucket_list (potentials/bucket.c); the pair
//   set is the reference's: every pair inside the cutoffs of force_single.
// * Non-bonded (force_single, calc_func.c:370-409; LJ_force LJ.c:37-64;
//   electro_force electro.c:36-56): one thread per bead gathers the force
//   on its own bead, so no atomics touch forces and the summation order is
//   fixed. Each pair is evaluated in the reference's orientation (lower
//   index first) with unfused double operations, so distances, cutoff
//   tests and pair counts are bit-identical to the reference's.
// * Bonded (bond.c:43-85, angle.c:38-86, angle_cos.c:36-81, dihe.c:42-144,
//   dihe_angle.c:43-255): one thread per term writes per-member force
//   contributions into slots; one thread per bead sums its slots in a fixed
//   order (CSR gather), which seeds the non-bonded accumulation.
// * Energies: per-term / per-block partials reduced by one CTA in a fixed
//   tree, so repeated runs give identical bits.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "bdb_common.cuh"

namespace bdb {

static constexpr int NB_THREADS = 128;
static constexpr int SORT_MAX = 16384;   // beads per segment sorted in shared memory

struct ForceParams {
    int periodic;
    double box[3], inv_L[3];
    int elec;
    double epsilon_c, kappa_c, gamma_c, cutoff_c;
    double alpha_lj, cutoff_lj;
    double lj6;
    double bond_lj_scale, bond_c_scale;
    int check_overlap;
    int conn_live;
};

static ForceParams make_fp(const bdb_system* s)
{
    ForceParams f;
    f.periodic = s->p.bc == 1;
    for (int k = 0; k < 3; ++k) {
        f.box[k] = s->p.box[k];
        f.inv_L[k] = s->inv_L[k];
    }
    f.elec = s->p.elec;
    f.epsilon_c = s->p.epsilon_c;
    f.kappa_c = s->p.kappa_c;
    f.gamma_c = s->p.gamma_c;
    f.cutoff_c = s->p.cutoff_c;
    f.alpha_lj = s->p.alpha_lj;
    f.cutoff_lj = s->p.cutoff_lj;
    f.lj6 = s->p.lj_6_term;
    f.bond_lj_scale = s->p.bond_lj_scale;
    f.bond_c_scale = s->p.bond_c_scale;
    f.check_overlap = s->p.check_overlap;
    f.conn_live = s->conn_live;
    return f;
}

// ---------------------------------------------------------------- cell list

// cell index along one axis. A periodic grid wraps, so that a coordinate
// outside the box (set by a caller; steps wrap positions) lies in its image's
// cell, which the neighbour search's minimum-image distances expect; a
// free-space grid clamps to its table. The wrap is taken in double, so a
// far-flung or non-finite coordinate cannot overflow the conversion (NaN
// converts to 0).
__device__ __forceinline__ int cell_axis(double x, double o, double w, int n, bool periodic)
{
    double t = floor((x - o) / w);
    if (periodic) t -= n * floor(t / n);
    const int ci = (int)t;
    return ci < 0 ? 0 : (ci >= n ? n - 1 : ci);
}

__global__ void k_cells(const double4* __restrict__ pos, const Segment* __restrict__ segs,
                        double cell, double skin, int periodic, double3 box,
                        unsigned long long* __restrict__ keys_out, int* __restrict__ idx_out,
                        double4* __restrict__ grid, int4* __restrict__ dims, double4* __restrict__ pos_build,
                        int* __restrict__ built, int2* __restrict__ cell_range, const long long* __restrict__ cell_off,
                        int* __restrict__ resort)
{
    extern __shared__ unsigned long long sk[];
    __shared__ double red[6][32];
    __shared__ double g_origin[3];
    __shared__ int g_n[3];
    __shared__ int moved;
    const Segment sg = segs[blockIdx.x];
    const int tid = threadIdx.x, nt = blockDim.x;
    const bool big = sg.count > SORT_MAX;   // sorted by the multi-CTA kernels below
    if (big && tid == 0) resort[blockIdx.x] = 0;
    if (built[blockIdx.x]) {
        // re-sort only when a bead has moved more than skin/2 since the last sort
        if (tid == 0) moved = 0;
        __syncthreads();
        const double lim = 0.25 * skin * skin;
        bool far = false;
        for (int i = tid; i < sg.count; i += nt) {
            const double4 a = pos[sg.begin + i], b = pos_build[sg.begin + i];
            double d[3] = {a.x - b.x, a.y - b.y, a.z - b.z};
            if (periodic) {
                d[0] -= box.x * floor(d[0] / box.x + 0.5);
                d[1] -= box.y * floor(d[1] / box.y + 0.5);
                d[2] -= box.z * floor(d[2] / box.z + 0.5);
            }
            if (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] > lim) far = true;
        }
        if (far) moved = 1;
        __syncthreads();
        if (!moved) return;
    }
    if (!periodic) {
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int i = tid; i < sg.count; i += nt) {
            double4 p = pos[sg.begin + i];
            lo[0] = fmin(lo[0], p.x); lo[1] = fmin(lo[1], p.y); lo[2] = fmin(lo[2], p.z);
            hi[0] = fmax(hi[0], p.x); hi[1] = fmax(hi[1], p.y); hi[2] = fmax(hi[2], p.z);
        }
        for (int k = 0; k < 3; ++k)
            for (int o = 16; o > 0; o >>= 1) {
                lo[k] = fmin(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
                hi[k] = fmax(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
            }
        if ((tid & 31) == 0)
            for (int k = 0; k < 3; ++k) {
                red[k][tid >> 5] = lo[k];
                red[3 + k][tid >> 5] = hi[k];
            }
        __syncthreads();
        if (tid == 0) {
            double L[3], H[3];
            for (int k = 0; k < 3; ++k) {
                L[k] = red[k][0];
                H[k] = red[3 + k][0];
                for (int w = 1; w < nt / 32; ++w) {
                    L[k] = fmin(L[k], red[k][w]);
                    H[k] = fmax(H[k], red[3 + k][w]);
                }
            }
            // grow the cell until the grid fits the segment's cell table. The
            // cell count is formed in double so that a far-flung bead cannot
            // overflow it; a non-finite extent (an infinite coordinate) would
            // never fit, so such a segment takes the brute-force path, where
            // the non-finite distances raise the overlap flag.
            const double cap = (double)cell_off[2 * blockIdx.x + 1];
            bool finite = true;
            for (int k = 0; k < 3; ++k) finite = finite && isfinite(H[k] - L[k]) && H[k] >= L[k];
            double c = cell;
            while (finite) {
                double tot = 1;
                for (int k = 0; k < 3; ++k) tot *= floor((H[k] - L[k]) / c) + 1;
                if (tot <= cap) break;
                c *= 1.25;
            }
            for (int k = 0; k < 3; ++k) {
                g_origin[k] = L[k];
                g_n[k] = finite ? (int)floor((H[k] - L[k]) / c) + 1 : 1;
            }
            grid[blockIdx.x] = make_double4(L[0], L[1], L[2], c);
            dims[blockIdx.x] = make_int4(g_n[0], g_n[1], g_n[2], finite ? 0 : 1);
        }
    } else if (tid == 0) {
        int nn[3];
        double bx[3] = {box.x, box.y, box.z};
        int brute = 0;
        const long long cap = cell_off[2 * blockIdx.x + 1];
        double cw = cell;
        for (;;) {
            long long tot = 1;
            for (int k = 0; k < 3; ++k) tot *= (long long)floor(bx[k] / cw);
            if (tot <= cap) break;
            cw *= 1.25;
        }
        for (int k = 0; k < 3; ++k) {
            nn[k] = (int)floor(bx[k] / cw);
            if (nn[k] < 3) brute = 1;
            g_n[k] = nn[k];
            g_origin[k] = -0.5 * bx[k];
        }
        // the periodic cell widths are box/n >= cutoff; w carries them per axis
        grid[blockIdx.x] = make_double4(bx[0] / nn[0], bx[1] / nn[1], bx[2] / nn[2], -1.0);
        dims[blockIdx.x] = make_int4(nn[0], nn[1], nn[2], brute);
    }
    __syncthreads();
    const double4 gr = grid[blockIdx.x];
    const int4 gd = dims[blockIdx.x];
    if (gd.w) return;
    if (big) {
        // the grid is set; k_big_keys .. k_big_fill sort and tabulate
        if (tid == 0) resort[blockIdx.x] = 1;
        return;
    }
    // keys
    int npow = 1;
    while (npow < sg.count) npow <<= 1;
    for (int i = tid; i < npow; i += nt) {
        unsigned long long key = ~0ull;
        if (i < sg.count) {
            double4 p = pos[sg.begin + i];
            double x[3] = {p.x, p.y, p.z};
            int c[3];
            for (int k = 0; k < 3; ++k)
                c[k] = cell_axis(x[k], g_origin[k], periodic ? (&gr.x)[k] : gr.w, g_n[k], periodic);
            unsigned long long cl = ((unsigned long long)c[2] * g_n[1] + c[1]) * g_n[0] + c[0];
            key = (cl << 24) | (unsigned long long)i;
        }
        sk[i] = key;
    }
    __syncthreads();
    // bitonic sort of npow keys
    for (int k = 2; k <= npow; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < npow; i += nt) {
                int ixj = i ^ j;
                if (ixj > i) {
                    unsigned long long a = sk[i], b = sk[ixj];
                    bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        sk[i] = b;
                        sk[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    // dense cell table: [first, end) of every cell, empty cells {0, 0}
    int2* tab = cell_range + cell_off[2 * blockIdx.x];
    const long long ncell = (long long)g_n[0] * g_n[1] * g_n[2];
    for (long long k = tid; k < ncell; k += nt) tab[k] = make_int2(0, 0);
    __syncthreads();
    for (int i = tid; i < sg.count; i += nt) {
        const unsigned long long key = sk[i] >> 24;
        keys_out[sg.begin + i] = key;
        idx_out[sg.begin + i] = sg.begin + (int)(sk[i] & 0xffffffull);
        pos_build[sg.begin + i] = pos[sg.begin + i];
        if (i == 0 || (sk[i - 1] >> 24) != key) tab[key].x = sg.begin + i;
        if (i == sg.count - 1 || (sk[i + 1] >> 24) != key) tab[key].y = sg.begin + i + 1;
    }
    if (tid == 0) built[blockIdx.x] = 1;
}

__device__ __forceinline__ int lower_bound_key(const unsigned long long* keys, int lo, int hi,
                                               unsigned long long key)
{
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (keys[mid] < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// --------------------------------------- cell list of a large segment
//
// A segment of more than SORT_MAX beads is sorted by several CTAs: the keys
// (cell << 24 | bead, the shared-memory path's keys, all distinct, so every
// correct sort gives the same order and the forces the same bits) are
// bitonic-sorted in chunks of SORT_MAX in shared memory, the chunks merged
// pairwise in global memory (each key's place found by a binary search in
// the other run), and the dense cell table rebuilt from the sorted keys.
// Each kernel does nothing unless k_cells flagged the segment for a re-sort
// (a bead moved more than skin/2, or the first build). npow is the
// segment's bead count rounded up to a power of two (at least SORT_MAX);
// the keys past the segment are ~0.

// cell of a position in the segment's grid, as k_cells computes it
__device__ __forceinline__ unsigned long long cell_of(const double4 p, const double4 gr, const int4 gd, int periodic,
                                                      double3 box)
{
    const double x[3] = {p.x, p.y, p.z};
    const double org[3] = {periodic ? -0.5 * box.x : gr.x, periodic ? -0.5 * box.y : gr.y,
                           periodic ? -0.5 * box.z : gr.z};
    const int n[3] = {gd.x, gd.y, gd.z};
    int c[3];
    for (int k = 0; k < 3; ++k) c[k] = cell_axis(x[k], org[k], periodic ? (&gr.x)[k] : gr.w, n[k], periodic);
    return ((unsigned long long)c[2] * n[1] + c[1]) * n[0] + c[0];
}

__global__ void k_big_keys(int g, const double4* __restrict__ pos, const Segment* __restrict__ segs,
                           const double4* __restrict__ grid, const int4* __restrict__ dims, int periodic, double3 box,
                           const int* __restrict__ resort, unsigned long long* __restrict__ keys, int npow)
{
    if (!resort[g]) return;
    const Segment sg = segs[g];
    const double4 gr = grid[g];
    const int4 gd = dims[g];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npow; i += gridDim.x * blockDim.x)
        keys[i] = i < sg.count ? (cell_of(pos[sg.begin + i], gr, gd, periodic, box) << 24) | (unsigned long long)i
                               : ~0ull;
}

// one chunk of SORT_MAX keys per CTA, ascending
__global__ void __launch_bounds__(1024) k_big_chunks(int g, const int* __restrict__ resort,
                                                     unsigned long long* __restrict__ keys)
{
    if (!resort[g]) return;
    extern __shared__ unsigned long long sk[];
    const int tid = threadIdx.x, nt = blockDim.x;
    unsigned long long* src = keys + (size_t)blockIdx.x * SORT_MAX;
    for (int i = tid; i < SORT_MAX; i += nt) sk[i] = src[i];
    __syncthreads();
    for (int k = 2; k <= SORT_MAX; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < SORT_MAX; i += nt) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const unsigned long long a = sk[i], b = sk[ixj];
                    if ((a > b) == ((i & k) == 0)) {
                        sk[i] = b;
                        sk[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int i = tid; i < SORT_MAX; i += nt) src[i] = sk[i];
}

// sorted runs of w keys -> runs of 2w: a key of the left run lands after the
// keys of the right run that are smaller, a key of the right run after
// those of the left run that are smaller or equal (the pad keys repeat)
__global__ void k_big_merge(int g, const int* __restrict__ resort, const unsigned long long* __restrict__ src,
                            unsigned long long* __restrict__ dst, int npow, int w)
{
    if (!resort[g]) return;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npow; p += gridDim.x * blockDim.x) {
        const unsigned long long key = src[p];
        const int base = (p / (2 * w)) * (2 * w);
        const bool left = p - base < w;
        const unsigned long long* other = src + (left ? base + w : base);
        int lo = 0, hi = w;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (left ? other[mid] < key : other[mid] <= key) lo = mid + 1; else hi = mid;
        }
        dst[base + (p - base - (left ? 0 : w)) + lo] = key;
    }
}

__global__ void k_big_clear(int g, const int* __restrict__ resort, const int4* __restrict__ dims,
                            int2* __restrict__ cell_range, const long long* __restrict__ cell_off)
{
    if (!resort[g]) return;
    const int4 gd = dims[g];
    const long long ncell = (long long)gd.x * gd.y * gd.z;
    int2* tab = cell_range + cell_off[2 * g];
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < ncell; k += (long long)gridDim.x * blockDim.x)
        tab[k] = make_int2(0, 0);
}

// the sorted keys -> the segment's sorted bead order, its cell table and
// the positions the next skin test compares against
__global__ void k_big_fill(int g, const int* __restrict__ resort, const Segment* __restrict__ segs,
                           const unsigned long long* __restrict__ sorted, const double4* __restrict__ pos,
                           unsigned long long* __restrict__ keys_out, int* __restrict__ idx_out,
                           double4* __restrict__ pos_build, int2* __restrict__ cell_range,
                           const long long* __restrict__ cell_off, int* __restrict__ built)
{
    if (!resort[g]) return;
    const Segment sg = segs[g];
    int2* tab = cell_range + cell_off[2 * g];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < sg.count; i += gridDim.x * blockDim.x) {
        const unsigned long long key = sorted[i] >> 24;
        keys_out[sg.begin + i] = key;
        idx_out[sg.begin + i] = sg.begin + (int)(sorted[i] & 0xffffffull);
        pos_build[sg.begin + i] = pos[sg.begin + i];
        if (i == 0 || (sorted[i - 1] >> 24) != key) tab[key].x = sg.begin + i;
        if (i == sg.count - 1 || (sorted[i + 1] >> 24) != key) tab[key].y = sg.begin + i + 1;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) built[g] = 1;
}

// ------------------------------------------------------------- non-bonded

__device__ __forceinline__ bool is_conn(const int* conn_ptr, const int* conn_list, int i, int j)
{
    for (int k = conn_ptr[i]; k < conn_ptr[i + 1]; ++k)
        if (conn_list[k] == j) return true;
    return false;
}

// force_single for the pair (a, b), a < b, accumulating the force on `self`
// (a or b). Energies and pair counts are credited only when self == a.
__device__ __forceinline__ void pair_term(const ForceParams& fp, const double4* pos, const double* Q,
                                          const double2* LJ, const int* conn_ptr, const int* conn_list,
                                          int a, int b, int self, double* f, double& e_lj, double& e_c,
                                          unsigned& cnt_c, unsigned& cnt_lj, unsigned& rep)
{
    double v[3];
    dist_vec(pos[a], pos[b], fp.periodic, fp.box, fp.inv_L, v);
    const double r_sq = sq3(v);
    const double2 la = LJ[a], lb = LJ[b];
    const double sig = la.x + lb.x;
    const double lj_lim = fp.cutoff_lj > 0.0 ? fp.cutoff_lj : (double)1.122462f * sig;
    const double r_norm = __dsqrt_rn(r_sq);
    const bool elec_in = fp.elec && r_norm <= fp.cutoff_c;
    const bool lj_in = fp.alpha_lj != 0.0 && r_norm <= lj_lim;
    if (!elec_in && !lj_in) {
        // LJ_force_check (LJ.c:95-99)
        if (fp.check_overlap && sig * sig > r_sq) rep = 1;
        return;
    }
    const double inv = 1.0 / r_norm;
    const double e[3] = {v[0] * inv, v[1] * inv, v[2] * inv};
    const double sgn = self == a ? -1.0 : 1.0;   // F1 -= e F on a, F2 += e F on b
    const bool conn = fp.conn_live && is_conn(conn_ptr, conn_list, a, b);
    int r = 0;
    if (elec_in) {
        if (self == a) cnt_c++;
        double scale = 1.0;
        bool on = true;
        if (conn) {
            if (fp.bond_c_scale != 0.0) scale = fp.bond_c_scale; else on = false;
        }
        if (on) {
            const double g = fp.gamma_c / fp.epsilon_c;
            double Fm = g * Q[a] * Q[b] * (1 + fp.kappa_c * r_norm);
            const double ex = exp(-fp.kappa_c * r_norm);
            Fm *= ex / r_sq;
            if (scale != 1.0) Fm *= scale;
            if (self == a) {
                double en = g * Q[a] * Q[b] * ex / r_norm;
                if (scale != 1.0) en = scale * g * Q[a] * Q[b] * ex / r_norm;
                e_c += en;
            }
            f[0] += sgn * e[0] * Fm;
            f[1] += sgn * e[1] * Fm;
            f[2] += sgn * e[2] * Fm;
            if (isnan(Fm) || isinf(Fm)) r = 1;
        }
    }
    if (lj_in) {
        if (self == a) cnt_lj++;
        if (!conn || fp.bond_lj_scale != 0.0) {
            const double scale = conn ? fp.bond_lj_scale : 1.0;
            const double eps_ij = sqrt(la.y * lb.y);
            double s6 = sig / r_norm;
            s6 *= s6;
            s6 *= s6 * s6;
            double Fm = fp.alpha_lj * eps_ij * 6 * (s6 * (2 * s6 - fp.lj6)) / r_norm;
            if (scale != 1.0) Fm *= scale;
            if (self == a) e_lj += scale * (fp.alpha_lj * eps_ij * (s6 * (s6 - fp.lj6)));
            f[0] += sgn * e[0] * Fm;
            f[1] += sgn * e[1] * Fm;
            f[2] += sgn * e[2] * Fm;
            if (sig > r_norm || isnan(Fm) || isinf(Fm)) r = 1;
        } else if (sig * sig > r_sq) {
            r = 1;
        }
    } else if (sig * sig > r_sq) {
        r = 1;
    }
    if (isnan(e[0]) || isnan(e[1]) || isnan(e[2]) || isinf(e[0]) || isinf(e[1]) || isinf(e[2])) r = 1;
    if (fp.check_overlap && r) rep = 1;
}

// One warp per bead i: the lanes split the candidate beads of the 27
// neighbour cells (or of the whole segment for brute-force segments); each
// lane accumulates in a fixed order and the warp combines the lanes with a
// fixed xor tree, so the result is deterministic.
__global__ void __launch_bounds__(NB_THREADS)
k_nonbonded(ForceParams fp, int n, const double4* __restrict__ pos, const double* __restrict__ Q,
            const double2* __restrict__ LJ, const int* __restrict__ bead_seg,
            const Segment* __restrict__ segs, const int2* __restrict__ cell_range,
            const long long* __restrict__ cell_off, const int* __restrict__ sidx,
            const double4* __restrict__ grid, const int4* __restrict__ dims, const int* __restrict__ conn_ptr,
            const int* __restrict__ conn_list, const double* __restrict__ F_bonded,
            double* __restrict__ F, double* __restrict__ e_part,
            unsigned long long* __restrict__ counts, unsigned* __restrict__ status)
{
    const int lane = threadIdx.x & 31;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= n) return;
    double f[3] = {0, 0, 0};
    double e_lj = 0, e_c = 0;
    unsigned cnt_c = 0, cnt_lj = 0, rep = 0;
    const int sgi = bead_seg[i];
    const Segment sg = segs[sgi];
    const int4 gd = dims[sgi];
    if (fp.elec || fp.alpha_lj != 0.0) {
        if (gd.w) {
            for (int j = sg.begin + lane; j < sg.begin + sg.count; j += 32) {
                if (j == i) continue;
                const int a = i < j ? i : j, b = i < j ? j : i;
                pair_term(fp, pos, Q, LJ, conn_ptr, conn_list, a, b, i, f, e_lj, e_c, cnt_c, cnt_lj, rep);
            }
        } else {
            const double4 gr = grid[sgi];
            const double4 p = pos[i];
            const double x[3] = {p.x, p.y, p.z};
            int c[3];
            const int nn[3] = {gd.x, gd.y, gd.z};
            for (int k = 0; k < 3; ++k)
                c[k] = cell_axis(x[k], fp.periodic ? -0.5 * fp.box[k] : (&gr.x)[k], fp.periodic ? (&gr.x)[k] : gr.w,
                                 nn[k], fp.periodic);
            const int2* tab = cell_range + cell_off[2 * sgi];
            // lanes 0..26 fetch the [first, end) range of one neighbour cell each
            int2 rg = make_int2(0, 0);
            if (lane < 27) {
                int cc[3] = {c[0] + lane % 3 - 1, c[1] + (lane / 3) % 3 - 1, c[2] + lane / 9 - 1};
                bool skip = false;
                for (int k = 0; k < 3; ++k) {
                    if (cc[k] < 0 || cc[k] >= nn[k]) {
                        if (!fp.periodic) skip = true;
                        else cc[k] = (cc[k] + nn[k]) % nn[k];
                    }
                }
                if (!skip) rg = tab[((long long)cc[2] * nn[1] + cc[1]) * nn[0] + cc[0]];
            }
            // the 27 cells' beads as one list: lane k's candidates are
            // entries k, k + 32, ... of it (a scan of the cell counts and a
            // search over it), so a warp does a few full rounds instead of
            // one sparse round per cell; the rounds are warp-uniform
            const int cnt = rg.y - rg.x;
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            for (int base = 0; base < total; base += 32) {
                const int q = base + lane;
                // the cell holding entry q: the first lane whose inclusive
                // count exceeds q (cells 27..31 add nothing)
                int c = 0;
#pragma unroll
                for (int step = 16; step > 0; step >>= 1) {
                    const int probe = __shfl_sync(0xffffffffu, incl, c + step - 1);
                    if (probe <= q) c += step;
                }
                const int first = __shfl_sync(0xffffffffu, rg.x, c);
                const int excl = __shfl_sync(0xffffffffu, incl, c) - __shfl_sync(0xffffffffu, cnt, c);
                if (q < total) {
                    const int j = sidx[first + (q - excl)];
                    if (j != i) {
                        const int a = i < j ? i : j, b = i < j ? j : i;
                        pair_term(fp, pos, Q, LJ, conn_ptr, conn_list, a, b, i, f, e_lj, e_c, cnt_c, cnt_lj, rep);
                    }
                }
            }
        }
    } else if (fp.check_overlap) {
        for (int j = sg.begin + lane; j < sg.begin + sg.count; j += 32) {
            if (j == i) continue;
            const int a = i < j ? i : j, b = i < j ? j : i;
            double v[3];
            dist_vec(pos[a], pos[b], fp.periodic, fp.box, fp.inv_L, v);
            const double sig = LJ[a].x + LJ[b].x;
            if (sig * sig > sq3(v)) rep = 1;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        f[0] += __shfl_xor_sync(0xffffffffu, f[0], o);
        f[1] += __shfl_xor_sync(0xffffffffu, f[1], o);
        f[2] += __shfl_xor_sync(0xffffffffu, f[2], o);
        e_lj += __shfl_xor_sync(0xffffffffu, e_lj, o);
        e_c += __shfl_xor_sync(0xffffffffu, e_c, o);
        cnt_c += __shfl_xor_sync(0xffffffffu, cnt_c, o);
        cnt_lj += __shfl_xor_sync(0xffffffffu, cnt_lj, o);
        rep |= __shfl_xor_sync(0xffffffffu, rep, o);
    }
    if (lane == 0) {
        F[3 * i] = F_bonded[3 * i] + f[0];
        F[3 * i + 1] = F_bonded[3 * i + 1] + f[1];
        F[3 * i + 2] = F_bonded[3 * i + 2] + f[2];
        e_part[2 * i] = e_lj;
        e_part[2 * i + 1] = e_c;
        if (cnt_c) atomicAdd(&counts[0], (unsigned long long)cnt_c);
        if (cnt_lj) atomicAdd(&counts[1], (unsigned long long)cnt_lj);
        if (rep) atomicOr(status, ST_OVERLAP);
    }
}

// ---------------------------------------------------------------- bonded

struct BondedArgs {
    int periodic;
    double box[3], inv_L[3];
    int n_bond, n_angle, n_angle_cos, n_dihe, n_dihe_angle;
    const int *bond_pairs, *angle_pairs, *angle_cos_pairs, *dihe_pairs, *dihe_angle_pairs;
    const double *bond_parms, *angle_parms, *angle_cos_parms, *dihe_parms, *dihe_angle_parms;
};

__device__ __forceinline__ bool bad(double v) { return isnan(v) || isinf(v); }

// ---- vector algebra of the bonded terms ----------------------------------
struct V3 {
    double x, y, z;
};
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ bool bad(V3 v) { return bad(v.x) || bad(v.y) || bad(v.z); }
// clamp into [-1, 1] by comparisons, so that a NaN stays NaN and reaches the
// overlap flag (fmin/fmax would drop it)
__device__ __forceinline__ double clamp_unit(double c) { return c <= -1.0 ? -1.0 : (c >= 1.0 ? 1.0 : c); }

// r_to - r_from, with the minimum image when periodic (trans_dist_vec,
// trans.c:111-121, evaluated exactly)
__device__ __forceinline__ V3 separation(const BondedArgs& A, const double4* pos, int from, int to)
{
    double v[3];
    dist_vec(pos[from], pos[to], A.periodic, A.box, A.inv_L, v);
    return {v[0], v[1], v[2]};
}

// The two unit bond vectors of a bond angle at its apex j: u along r_i - r_j
// and w along r_k - r_j, and cos(theta) = u.w clamped to [-1, 1].
struct AngleFrame {
    V3 u, w;
    double c;
};
__device__ __forceinline__ AngleFrame angle_frame(const BondedArgs& A, const double4* pos, int i, int j, int k)
{
    AngleFrame f;
    const V3 a = separation(A, pos, j, i), b = separation(A, pos, j, k);
    f.u = (1.0 / sqrt(dot(a, a))) * a;
    f.w = (1.0 / sqrt(dot(b, b))) * b;
    f.c = clamp_unit(dot(f.u, f.w));
    return f;
}

// Dihedral geometry of the bond vectors b1 = r_j - r_i, b2 = r_k - r_j,
// b3 = r_l - r_k with the IUPAC sign: n1 = b1 x b2, n2 = b2 x b3,
// cos phi = n1.n2 / |n1||n2|, sin phi = |b2| b1.n2 / |n1||n2|, and the
// gradient of phi with respect to the four positions in the form of
// Blondel and Karplus (J. Comput. Chem. 17, 1132 (1996)):
//   d phi/d r_i = -|b2| n1 / |n1|^2,   d phi/d r_l = |b2| n2 / |n2|^2,
//   d phi/d r_j = (b3.b2/|b2|^2) d phi/d r_l - (1 + b1.b2/|b2|^2) d phi/d r_i,
//   d phi/d r_k = -(the other three),
// which has no 1/sin phi or 1/cos phi branch. h1, h2: the distances of r_i
// and r_l from the axis through r_j and r_k (|n1|/|b2|, |n2|/|b2|).
struct DiheFrame {
    double c, s, h1, h2;
    V3 g[4];
};
__device__ __forceinline__ DiheFrame dihedral_frame(V3 b1, V3 b2, V3 b3)
{
    DiheFrame f;
    const V3 n1 = cross(b1, b2), n2 = cross(b2, b3);
    const double q1 = dot(n1, n1), q2 = dot(n2, n2), bb = dot(b2, b2);
    const double lb = sqrt(bb), inv_n = 1.0 / sqrt(q1 * q2);
    f.c = dot(n1, n2) * inv_n;
    f.s = lb * dot(b1, n2) * inv_n;
    f.h1 = sqrt(q1) / lb;
    f.h2 = sqrt(q2) / lb;
    f.g[0] = (-lb / q1) * n1;
    f.g[3] = (lb / q2) * n2;
    f.g[1] = (dot(b3, b2) / bb) * f.g[3] - (1.0 + dot(b1, b2) / bb) * f.g[0];
    f.g[2] = -(f.g[0] + f.g[1] + f.g[3]);
    return f;
}

// Chebyshev polynomial T_m(c) = cos(m theta) for c = cos(theta) and its
// derivative T_m'(c) = m U_{m-1}(c), by the three-term recurrences. BD_BOX
// tabulates m = 1..6 and takes T = 1, T' = 0 for any other m
// (get_m_cos / get_delta_cos, dihe.c:146-184).
__device__ __forceinline__ void chebyshev(int m, double c, double& T, double& dT)
{
    if (m < 1 || m > 6) {
        T = 1.0;
        dT = 0.0;
        return;
    }
    double t_prev = 1.0, t = c, u_prev = 0.0, u = 1.0;   // T_0, T_1; U_-1, U_0
    for (int k = 1; k < m; ++k) {
        const double tn = 2.0 * c * t - t_prev, un = 2.0 * c * u - u_prev;
        t_prev = t;
        t = tn;
        u_prev = u;
        u = un;
    }
    T = t;
    dT = m * u;
}

// Term t writes its members' forces into contrib[slot0 + 3*member ...]; slot
// layout: bonds 2 slots, angles 3, cosine angles 3, dihedrals 4, harmonic
// dihedrals 4, in that order of term types.
__global__ void k_bonded(BondedArgs A, const double4* __restrict__ pos, double* __restrict__ contrib,
                         double* __restrict__ energy, unsigned* __restrict__ status)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int slot = 0;
    unsigned st = 0;
    if (t < A.n_bond) {
        // FENE-type bond (bond.c:43-85): force H (r0 - r) / (1 - r^2/rmax^2)
        // along the bond, pushing the beads apart when positive; energy
        // -H/2 [rmax^2 ln((rmax^2 - r^2)/(rmax^2 - r0^2))
        //       + r0 rmax ln((rmax + r)(rmax - r0) / ((rmax - r)(rmax + r0)))].
        // r >= rmax is BD_BOX's fatal over-stretch: flagged, no force.
        const int a = A.bond_pairs[2 * t], b = A.bond_pairs[2 * t + 1];
        const double r0 = A.bond_parms[3 * t], rmax = A.bond_parms[3 * t + 1], H = A.bond_parms[3 * t + 2];
        const V3 d = separation(A, pos, a, b);
        const double r2 = dot(d, d), r = sqrt(r2);
        const V3 e = (1 / r) * d;                 // unit vector from a to b
        double push = 0, en = 0;
        if (r < rmax) {
            const double m2 = rmax * rmax;
            en = -0.5 * H * (m2 * log((m2 - r2) / (m2 - r0 * r0)) +
                             r0 * rmax * log((rmax + r) * (rmax - r0) / ((rmax - r) * (rmax + r0))));
            push = H * (r0 - r) / (1 - r2 / m2);
        } else {
            st |= ST_BOND;
        }
        slot = 2 * t;
        double* c = contrib + 3 * slot;
        const V3 fb = push * e;
        c[0] = -fb.x;
        c[1] = -fb.y;
        c[2] = -fb.z;
        c[3] = fb.x;
        c[4] = fb.y;
        c[5] = fb.z;
        energy[t] = en;
        if (bad(push) || bad(e) || bad(en)) st |= ST_OVERLAP;
    } else if (t - A.n_bond < A.n_angle + A.n_angle_cos) {
        // Bond angles at apex j: harmonic in theta (angle.c:38-86) or in
        // cos theta (angle_cos.c:36-81). BD_BOX's force on an end bead is
        // the derivative of the energy with respect to its UNIT bond vector:
        // g times the component of the other bond's unit vector normal to
        // its own (|w - c u| = sin theta); the 1/|bond| of d theta/d r is
        // absent in BD_BOX and is left out here too. The apex takes minus
        // the sum. A harmonic angle within 1e-6 of 0 or pi in cos theta
        // contributes nothing, energy included.
        const int ta = t - A.n_bond;
        const bool harm = ta < A.n_angle;
        const int tt = harm ? ta : ta - A.n_angle;
        const int* q = (harm ? A.angle_pairs : A.angle_cos_pairs) + 3 * tt;
        const double2 prm = reinterpret_cast<const double2*>(harm ? A.angle_parms : A.angle_cos_parms)[tt];
        const AngleFrame fr = angle_frame(A, pos, q[0], q[1], q[2]);
        double g = 0.0, en = 0.0;
        if (harm) {
            if (!(fr.c >= 1.0 - 0.000001 || fr.c <= -1.0 + 0.000001)) {   // NaN passes on
                const double d = acos(fr.c) - prm.x;            // theta - theta0
                en = 0.5 * prm.y * d * d;
                g = prm.y * d / sqrt(1.0 - fr.c * fr.c);
            }
        } else {
            const double d = fr.c - prm.x;                      // cos theta - cos theta0
            en = 0.5 * prm.y * d * d;
            g = -prm.y * d;
        }
        const V3 fi = g * (fr.w - fr.c * fr.u), fk = g * (fr.u - fr.c * fr.w);
        slot = 2 * A.n_bond + 3 * ta;
        double* c = contrib + 3 * slot;
        const V3 f3[3] = {fi, -(fi + fk), fk};
        for (int m = 0; m < 3; ++m) {
            c[3 * m] = f3[m].x;
            c[3 * m + 1] = f3[m].y;
            c[3 * m + 2] = f3[m].z;
        }
        energy[t] = en;
        if (bad(fi) || bad(fk) || bad(en)) st |= ST_OVERLAP;
    } else if ((t -= A.n_bond + A.n_angle + A.n_angle_cos) < A.n_dihe) {
        // Cosine dihedral E = |p| (1 + |p| cos(m phi)), p = -k delta
        // (dihe.c:42-144, parameters as add_dihe stores them, dihe.c:186-203),
        // bond vectors with the minimum image. Its force is
        // p T_m'(cos phi) grad(cos phi) = -p sin(phi) T_m'(cos phi) grad(phi).
        // Nothing (energy included) when r_i or r_l lies within 1e-6 of the
        // j-k axis.
        const int* q = A.dihe_pairs + 4 * t;
        const double2 prm = reinterpret_cast<const double2*>(A.dihe_parms)[t];
        const DiheFrame fr = dihedral_frame(separation(A, pos, q[0], q[1]), separation(A, pos, q[1], q[2]),
                                            separation(A, pos, q[2], q[3]));
        double en = 0.0, g = 0.0;
        const bool live = !(fr.h1 < 0.000001) && !(fr.h2 < 0.000001);   // NaN passes on
        if (live) {
            double T, dT;
            chebyshev((int)prm.y, clamp_unit(fr.c), T, dT);
            en = fabs(prm.x) * (1.0 + fabs(prm.x) * T);
            g = -prm.x * fr.s * dT;
        }
        slot = 2 * A.n_bond + 3 * A.n_angle + 3 * A.n_angle_cos + 4 * t;
        double* c = contrib + 3 * slot;
        for (int m = 0; m < 4; ++m) {
            const V3 f = live ? g * fr.g[m] : V3{0.0, 0.0, 0.0};
            c[3 * m] = f.x;
            c[3 * m + 1] = f.y;
            c[3 * m + 2] = f.z;
            if (bad(f)) st |= ST_OVERLAP;
        }
        energy[A.n_bond + A.n_angle + A.n_angle_cos + t] = en;
        if (bad(en)) st |= ST_OVERLAP;
    } else if ((t -= A.n_dihe) < A.n_dihe_angle) {
        // Harmonic dihedral E = k/2 (phi - phi0)^2 (dihe_angle.c:43-99),
        // phi with BD_BOX's sign (minus the IUPAC angle) and the difference
        // wrapped into [-pi, pi] with the float pi; bond vectors WITHOUT the
        // periodic image, as BD_BOX takes raw differences here. Force
        // -k (phi - phi0) grad(phi_BD_BOX) = k (phi - phi0) grad(phi_IUPAC);
        // a collinear triple makes the gradient non-finite, which flags a
        // retry.
        const int* q = A.dihe_angle_pairs + 4 * t;
        const double2 prm = reinterpret_cast<const double2*>(A.dihe_angle_parms)[t];
        const double4 P0 = pos[q[0]], P1 = pos[q[1]], P2 = pos[q[2]], P3 = pos[q[3]];
        const DiheFrame fr = dihedral_frame({P1.x - P0.x, P1.y - P0.y, P1.z - P0.z},
                                            {P2.x - P1.x, P2.y - P1.y, P2.z - P1.z},
                                            {P3.x - P2.x, P3.y - P2.y, P3.z - P2.z});
        const double pif = (double)BDB_M_PIF;
        double d = -atan2(fr.s, fr.c) - prm.y;
        if (d < -pif) d += 2 * pif;
        if (d > pif) d -= 2 * pif;
        const double g = prm.x * d;
        const double en = 0.5 * g * d;
        slot = 2 * A.n_bond + 3 * A.n_angle + 3 * A.n_angle_cos + 4 * A.n_dihe + 4 * t;
        double* c = contrib + 3 * slot;
        for (int m = 0; m < 4; ++m) {
            const V3 f = g * fr.g[m];
            c[3 * m] = f.x;
            c[3 * m + 1] = f.y;
            c[3 * m + 2] = f.z;
            if (bad(fr.g[m])) st |= ST_OVERLAP;
        }
        energy[A.n_bond + A.n_angle + A.n_angle_cos + A.n_dihe + t] = en;
        if (bad(g) || bad(en)) st |= ST_OVERLAP;
    }
    if (st) atomicOr(status, st);
}

__global__ void k_bonded_gather(int n, const int* __restrict__ slot_ptr, const int* __restrict__ slot_list,
                                const double* __restrict__ contrib, double* __restrict__ F)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double f[3] = {0, 0, 0};
    for (int k = slot_ptr[i]; k < slot_ptr[i + 1]; ++k) {
        const double* c = contrib + 3 * slot_list[k];
        f[0] += c[0];
        f[1] += c[1];
        f[2] += c[2];
    }
    F[3 * i] = f[0];
    F[3 * i + 1] = f[1];
    F[3 * i + 2] = f[2];
}

// External forces per bead, after the bonded terms (bonded_inter,
// pre_func.c:135-158): the electric field on charged beads
// (electro_ext_force, electro_ext.c:38-51; DC, AC = cos(w t) on dir1, RF =
// cos on dir1 and sin on dir2, at the force time t) and the bounding-sphere
// force (sboundary_ext, sboundary.c:36-73: -A x / (r R^n) beyond the cutoff
// radius, R = sphere_radius - r; a bead within 1e-6 of the wall flags a
// retry). No energy term, as in BD_BOX. The force time is a device scalar
// so that replayed graphs see the current step's time.
struct ExtArgs {
    int e_ext, e_type, dir1, dir2;
    double e_factor, e_magn, e_freq;
    int sbound, sb_n;
    double sb_A, sb_cut, sphere_R;
};

__global__ void k_external(int n, ExtArgs a, const double4* __restrict__ pos, const double* __restrict__ Q,
                           const double* __restrict__ t_force, double* __restrict__ F, unsigned* __restrict__ status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double f[3] = {F[3 * i], F[3 * i + 1], F[3 * i + 2]};
    bool bad = false;
    const double q = Q[i];
    if (a.e_ext && q != 0.0) {
        const double base = q * a.e_factor * a.e_magn;
        if (a.e_type == 0) {
            f[a.dir1] += base;
        } else {
            const double wt = a.e_freq * *t_force;
            f[a.dir1] += base * cos(wt);
            if (a.e_type == 2) f[a.dir2] += base * sin(wt);
        }
        bad = isnan(f[a.dir1]) || isinf(f[a.dir1]) || (a.e_type == 2 && (isnan(f[a.dir2]) || isinf(f[a.dir2])));
    }
    if (a.sbound) {
        const double4 p = pos[i];
        const double r = sqrt(p.x * p.x + p.y * p.y + p.z * p.z);
        if (r >= a.sb_cut) {
            const double R = a.sphere_R - r;
            if (R >= 0.000001) {
                // 1 / (r R^n) by binary powers of 1/R, as sboundary_ext forms it
                double inr = 1.0 / r, inR = 1.0 / R;
                for (int b = 1; b <= a.sb_n; b *= 2) {
                    if (a.sb_n & b) inr *= inR;
                    inR *= inR;
                }
                f[0] -= a.sb_A * p.x * inr;
                f[1] -= a.sb_A * p.y * inr;
                f[2] -= a.sb_A * p.z * inr;
            } else {
                bad = true;
            }
        }
    }
    F[3 * i] = f[0];
    F[3 * i + 1] = f[1];
    F[3 * i + 2] = f[2];
    if (bad) atomicOr(status, ST_OVERLAP);
}

__global__ void k_set_time(double* t_force, double t) { *t_force = t; }

static bool has_external(const bdb_system* s) { return s->p.e_ext || (s->p.sboundary && s->p.bc == 2); }

int set_force_time(bdb_system* s, double t)
{
    if (!(s->p.e_ext && s->p.e_type != 0)) return BDB_OK;   // only AC and RF depend on time
    k_set_time<<<1, 1, 0, s->stream>>>(s->scal.p + 8, t);
    BDB_CUDA(cudaGetLastError());
    s->launches += 1;
    return BDB_OK;
}

// Energies: E[1..5] from the bonded terms (sums per type), E[6], E[7] from
// the non-bonded block partials. One CTA, fixed order.
struct TermRanges {
    int lim[6];   // [lim[t], lim[t+1]) are the terms of type t
};

__global__ void k_energy_reduce(int nb_blocks, const double* __restrict__ e_part,
                                const double* __restrict__ term_energy, TermRanges tr, double* __restrict__ E)
{
    __shared__ double sh[256];
    const int tid = threadIdx.x;
    for (int type = 0; type < 7; ++type) {
        double a = 0;
        if (type < 5) {
            for (int k = tr.lim[type] + tid; k < tr.lim[type + 1]; k += blockDim.x) a += term_energy[k];
        } else {
            for (int k = tid; k < nb_blocks; k += blockDim.x) a += e_part[2 * k + (type - 5)];
        }
        sh[tid] = a;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if (tid < o) sh[tid] += sh[tid + o];
            __syncthreads();
        }
        if (tid == 0) E[1 + type] = sh[0];
        __syncthreads();
    }
    if (tid == 0) {
        E[0] = 0;
        E[8] = 0;
    }
}

// ---------------------------------------------------------------- host side

int bonded_setup(bdb_system* s)
{
    // slots in term order (bond 2, angle 3, angle_cos 3, dihe 4, dihe_angle 4)
    std::vector<std::vector<int>> per_bead(s->n);
    int slot = 0;
    auto add_terms = [&](int count, int members, const std::vector<int>& idx) {
        for (int t = 0; t < count; ++t)
            for (int m = 0; m < members; ++m) per_bead[idx[t * members + m]].push_back(slot++);
    };
    auto fetch = [&](DevBuf<int>& b, int count) {
        std::vector<int> v(count);
        if (count) d2h(s, v.data(), b.p, sizeof(int) * count);
        return v;
    };
    add_terms(s->n_bond, 2, fetch(s->bond_pairs, 2 * s->n_bond));
    add_terms(s->n_angle, 3, fetch(s->angle_pairs, 3 * s->n_angle));
    add_terms(s->n_angle_cos, 3, fetch(s->angle_cos_pairs, 3 * s->n_angle_cos));
    add_terms(s->n_dihe, 4, fetch(s->dihe_pairs, 4 * s->n_dihe));
    add_terms(s->n_dihe_angle, 4, fetch(s->dihe_angle_pairs, 4 * s->n_dihe_angle));
    s->n_slots = slot;
    s->n_terms = s->n_bond + s->n_angle + s->n_angle_cos + s->n_dihe + s->n_dihe_angle;
    std::vector<int> ptr(s->n + 1, 0), list;
    for (int i = 0; i < s->n; ++i) {
        ptr[i + 1] = ptr[i] + (int)per_bead[i].size();
        list.insert(list.end(), per_bead[i].begin(), per_bead[i].end());
    }
    if (s->slot_ptr.alloc(s->n + 1)) return BDB_ERR_NOMEM;
    if (s->slot_list.alloc(std::max<size_t>(1, list.size()))) return BDB_ERR_NOMEM;
    if (s->contrib.alloc(3 * std::max(1, s->n_slots))) return BDB_ERR_NOMEM;
    if (s->term_energy.alloc(std::max(1, s->n_terms))) return BDB_ERR_NOMEM;
    BDB_CUDA(h2d(s, s->slot_ptr.p, ptr.data(), sizeof(int) * (s->n + 1)));
    if (!list.empty())
        BDB_CUDA(h2d(s, s->slot_list.p, list.data(), sizeof(int) * list.size()));

    // are_conn (bond.c:87-92, alloc_connections :113-130): live only when a
    // 1-2 scale factor differs from 1
    const bdb_params& p = s->p;
    s->conn_live = s->n_bond && ((p.elec && p.bond_c_scale != 1) || (p.alpha_lj != 0.0 && p.bond_lj_scale != 1));
    std::vector<std::vector<int>> nb(s->n);
    std::vector<int> bp = fetch(s->bond_pairs, 2 * s->n_bond);
    for (int t = 0; t < s->n_bond; ++t) {
        nb[bp[2 * t]].push_back(bp[2 * t + 1]);
        nb[bp[2 * t + 1]].push_back(bp[2 * t]);
    }
    std::vector<int> cptr(s->n + 1, 0), clist;
    for (int i = 0; i < s->n; ++i) {
        std::sort(nb[i].begin(), nb[i].end());
        cptr[i + 1] = cptr[i] + (int)nb[i].size();
        clist.insert(clist.end(), nb[i].begin(), nb[i].end());
    }
    if (s->conn_ptr.alloc(s->n + 1)) return BDB_ERR_NOMEM;
    if (s->conn_list.alloc(std::max<size_t>(1, clist.size()))) return BDB_ERR_NOMEM;
    BDB_CUDA(h2d(s, s->conn_ptr.p, cptr.data(), sizeof(int) * (s->n + 1)));
    if (!clist.empty())
        BDB_CUDA(h2d(s, s->conn_list.p, clist.data(), sizeof(int) * clist.size()));
    return BDB_OK;
}

}  // namespace bdb

extern "C" int bdb_cell_grid(bdb_system* s, int segment, int* dims)
{
    using namespace bdb;
    if (!s || !dims) return fail(BDB_ERR_ARG, "null argument");
    if (segment < 0 || segment >= (int)s->segs.size()) return fail(BDB_ERR_ARG, "segment out of range");
    if (!s->grid_dims.p) return fail(BDB_ERR_ARG, "no force evaluation yet");
    int4 d;
    BDB_CUDA(d2h(s, &d, s->grid_dims.p + segment, sizeof(int4)));
    dims[0] = d.x;
    dims[1] = d.y;
    dims[2] = d.z;
    dims[3] = d.w;
    return BDB_OK;
}

namespace bdb {

int forces_setup(bdb_system* s)
{
    const int nseg = (int)s->segs.size();
    if (s->sorted_keys.alloc(s->n)) return BDB_ERR_NOMEM;
    if (s->sorted_idx.alloc(s->n)) return BDB_ERR_NOMEM;
    if (s->grid.alloc(nseg)) return BDB_ERR_NOMEM;
    if (s->grid_dims.alloc(nseg)) return BDB_ERR_NOMEM;
    if (s->pos_build.alloc(s->n) || s->cells_built.alloc(nseg)) return BDB_ERR_NOMEM;
    BDB_CUDA(dzero(s, s->cells_built.p, sizeof(int) * nseg));
    // dense cell tables: 32 cells per bead (at least 4096) per segment
    std::vector<long long> off(2 * nseg);
    long long tot = 0;
    for (int g = 0; g < nseg; ++g) {
        const long long cap = std::max<long long>(4096, 32ll * s->segs[g].count);
        off[2 * g] = tot;
        off[2 * g + 1] = cap;
        tot += cap;
    }
    if (s->cell_range.alloc(tot) || s->cell_off.alloc(2 * nseg)) return BDB_ERR_NOMEM;
    if (s->cells_resort.alloc(nseg)) return BDB_ERR_NOMEM;
    BDB_CUDA(dzero(s, s->cells_resort.p, sizeof(int) * nseg));
    int big = 0;
    for (auto& g : s->segs) big = std::max(big, g.count > SORT_MAX ? g.count : 0);
    if (big) {
        // bead index in the low 24 bits of a key
        if (big > (1 << 24)) return fail(BDB_ERR_ARG, "segment of more than 2^24 beads");
        size_t np = SORT_MAX;
        while (np < (size_t)big) np <<= 1;
        s->big_npow = np;
        if (s->big_keys.alloc(2 * np)) return BDB_ERR_NOMEM;
        BDB_CUDA(cudaFuncSetAttribute(k_big_chunks, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      SORT_MAX * (int)sizeof(unsigned long long)));
    }
    BDB_CUDA(h2d(s, s->cell_off.p, off.data(), sizeof(long long) * 2 * nseg));
    if (s->e_part.alloc(2 * s->n + 16)) return BDB_ERR_NOMEM;
    if (s->status.alloc(4)) return BDB_ERR_NOMEM;
    if (s->counts.alloc(2)) return BDB_ERR_NOMEM;
    if (s->F.alloc(3 * s->n) || s->F_save.alloc(3 * s->n) || s->work.alloc(3 * s->n + 16)) return BDB_ERR_NOMEM;
    BDB_CUDA(cudaFuncSetAttribute(k_cells, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  SORT_MAX * (int)sizeof(unsigned long long)));
    // cell size: the widest interaction range of force_single plus the
    // LJ_force_check distance (init_cutoff, pre_func.c:197-232)
    std::vector<double2> lj(s->n);
    BDB_CUDA(d2h(s, lj.data(), s->LJ.p, sizeof(double2) * s->n));
    double maxsig = 0;
    for (int i = 0; i < s->n; ++i) maxsig = std::max(maxsig, lj[i].x);
    double c = 2 * maxsig;
    if (s->p.elec) c = std::max(c, s->p.cutoff_c);
    if (s->p.alpha_lj != 0) c = std::max(c, s->p.cutoff_lj > 0 ? s->p.cutoff_lj : (double)1.122462f * 2 * maxsig);
    c = std::max(c, s->p.max_force_cutoff);
    s->skin = std::max(0.5, 0.1 * c);
    s->cell_size = (c + s->skin) * (1 + 1e-12) + 1e-9;
    return BDB_OK;
}

static BondedArgs bonded_args(bdb_system* s)
{
    BondedArgs A;
    A.periodic = s->p.bc == 1;
    for (int k = 0; k < 3; ++k) {
        A.box[k] = s->p.box[k];
        A.inv_L[k] = s->inv_L[k];
    }
    A.n_bond = s->n_bond;
    A.n_angle = s->n_angle;
    A.n_angle_cos = s->n_angle_cos;
    A.n_dihe = s->n_dihe;
    A.n_dihe_angle = s->n_dihe_angle;
    A.bond_pairs = s->bond_pairs.p;
    A.angle_pairs = s->angle_pairs.p;
    A.angle_cos_pairs = s->angle_cos_pairs.p;
    A.dihe_pairs = s->dihe_pairs.p;
    A.dihe_angle_pairs = s->dihe_angle_pairs.p;
    A.bond_parms = s->bond_parms.p;
    A.angle_parms = s->angle_parms.p;
    A.angle_cos_parms = s->angle_cos_parms.p;
    A.dihe_parms = s->dihe_parms.p;
    A.dihe_angle_parms = s->dihe_angle_parms.p;
    return A;
}

// Forces at the current positions into s->F; energies into s->scal[8..16]
// when requested (device), counts and status on the device.
int forces_run(bdb_system* s, bool want_energy, bool want_counts)
{
    cudaStream_t st = s->stream;
    const int nseg = (int)s->segs.size();
    (void)want_counts;
    BDB_CUDA(cudaMemsetAsync(s->counts.p, 0, 2 * sizeof(unsigned long long), st));
    double3 box = make_double3(s->p.box[0], s->p.box[1], s->p.box[2]);
    int smax = 0;
    for (auto& g : s->segs) smax = std::max(smax, g.count);
    int np = 1;
    while (np < smax) np <<= 1;
    size_t shm = sizeof(unsigned long long) * (size_t)std::min(np, SORT_MAX);
    k_cells<<<nseg, 1024, shm, st>>>(s->pos.p, s->d_segs.p, s->cell_size, s->skin, s->p.bc == 1, box,
                                      s->sorted_keys.p, s->sorted_idx.p, s->grid.p, s->grid_dims.p,
                                      s->pos_build.p, s->cells_built.p, s->cell_range.p, s->cell_off.p,
                                      s->cells_resort.p);
    BDB_CUDA(cudaGetLastError());
    for (int g = 0; g < nseg; ++g) {
        const int cnt = s->segs[g].count;
        if (cnt <= SORT_MAX) continue;
        int np = SORT_MAX;
        while (np < cnt) np <<= 1;
        unsigned long long *a = s->big_keys.p, *b = a + s->big_npow;
        const int blocks = std::min(4 * s->sm_count, (np + 255) / 256);
        k_big_keys<<<blocks, 256, 0, st>>>(g, s->pos.p, s->d_segs.p, s->grid.p, s->grid_dims.p, s->p.bc == 1, box,
                                           s->cells_resort.p, a, np);
        k_big_chunks<<<np / SORT_MAX, 1024, SORT_MAX * sizeof(unsigned long long), st>>>(g, s->cells_resort.p, a);
        s->launches += 2;
        for (int w = SORT_MAX; w < np; w <<= 1) {
            k_big_merge<<<blocks, 256, 0, st>>>(g, s->cells_resort.p, a, b, np, w);
            std::swap(a, b);
            s->launches += 1;
        }
        k_big_clear<<<blocks, 256, 0, st>>>(g, s->cells_resort.p, s->grid_dims.p, s->cell_range.p, s->cell_off.p);
        k_big_fill<<<blocks, 256, 0, st>>>(g, s->cells_resort.p, s->d_segs.p, a, s->pos.p, s->sorted_keys.p,
                                           s->sorted_idx.p, s->pos_build.p, s->cell_range.p, s->cell_off.p,
                                           s->cells_built.p);
        s->launches += 2;
        BDB_CUDA(cudaGetLastError());
    }
    double* Fb = s->work.p;
    if (s->n_terms) {
        BondedArgs A = bonded_args(s);
        k_bonded<<<(s->n_terms + 127) / 128, 128, 0, st>>>(A, s->pos.p, s->contrib.p, s->term_energy.p,
                                                           s->status.p);
        BDB_CUDA(cudaGetLastError());
        k_bonded_gather<<<(s->n + 127) / 128, 128, 0, st>>>(s->n, s->slot_ptr.p, s->slot_list.p,
                                                             s->contrib.p, Fb);
    } else {
        BDB_CUDA(cudaMemsetAsync(Fb, 0, sizeof(double) * 3 * s->n, st));
    }
    BDB_CUDA(cudaGetLastError());
    if (has_external(s)) {
        ExtArgs a;
        a.e_ext = s->p.e_ext;
        a.e_type = s->p.e_type;
        a.dir1 = s->p.e_dir1;
        a.dir2 = s->p.e_dir2;
        a.e_factor = s->p.e_factor;
        a.e_magn = s->p.e_magn;
        a.e_freq = s->p.e_freq;
        a.sbound = s->p.sboundary && s->p.bc == 2;
        a.sb_n = s->p.sboundary_n;
        a.sb_A = s->p.sboundary_A;
        a.sb_cut = s->p.sboundary_cutoff;
        a.sphere_R = s->p.sphere_radius;
        k_external<<<(s->n + 127) / 128, 128, 0, st>>>(s->n, a, s->pos.p, s->Q.p, s->scal.p + 8, Fb, s->status.p);
        BDB_CUDA(cudaGetLastError());
        s->launches += 1;
    }
    const int nblk = (s->n * 32 + NB_THREADS - 1) / NB_THREADS;
    k_nonbonded<<<nblk, NB_THREADS, 0, st>>>(make_fp(s), s->n, s->pos.p, s->Q.p, s->LJ.p, s->d_bead_seg.p,
                                             s->d_segs.p, s->cell_range.p, s->cell_off.p, s->sorted_idx.p, s->grid.p,
                                             s->grid_dims.p, s->conn_ptr.p, s->conn_list.p, Fb, s->F.p,
                                             s->e_part.p, s->counts.p, s->status.p);
    BDB_CUDA(cudaGetLastError());
    if (want_energy) {
        TermRanges tr;
        tr.lim[0] = 0;
        tr.lim[1] = s->n_bond;
        tr.lim[2] = tr.lim[1] + s->n_angle;
        tr.lim[3] = tr.lim[2] + s->n_angle_cos;
        tr.lim[4] = tr.lim[3] + s->n_dihe;
        tr.lim[5] = tr.lim[4] + s->n_dihe_angle;
        k_energy_reduce<<<1, 256, 0, st>>>(s->n, s->e_part.p, s->term_energy.p, tr, s->scal.p + 16);
        BDB_CUDA(cudaGetLastError());
    }
    s->launches += 2 + (s->n_terms ? 2 : 0) + (want_energy ? 1 : 0);
    s->have_forces = true;
    return BDB_OK;
}

}  // namespace bdb
