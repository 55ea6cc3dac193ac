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

__global__ void k_cells(const double4* __restrict__ pos, const Segment* __restrict__ segs,
                        double cell, double skin, int periodic, double3 box,
                        unsigned long long* __restrict__ keys_out, int* __restrict__ idx_out,
                        double4* __restrict__ grid, int4* __restrict__ dims, double4* __restrict__ pos_build,
                        int* __restrict__ built, int2* __restrict__ cell_range, const long long* __restrict__ cell_off)
{
    extern __shared__ unsigned long long sk[];
    __shared__ double red[6][32];
    __shared__ double g_origin[3];
    __shared__ int g_n[3];
    __shared__ int moved;
    const Segment sg = segs[blockIdx.x];
    const int tid = threadIdx.x, nt = blockDim.x;
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
    if (sg.count > SORT_MAX) {
        if (tid == 0) dims[blockIdx.x] = make_int4(0, 0, 0, 1);   // brute force
        return;
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
            // grow the cell until the grid fits the segment's cell table
            const long long cap = cell_off[2 * blockIdx.x + 1];
            double c = cell;
            for (;;) {
                long long tot = 1;
                for (int k = 0; k < 3; ++k) tot *= (long long)floor((H[k] - L[k]) / c) + 1;
                if (tot <= cap) break;
                c *= 1.25;
            }
            for (int k = 0; k < 3; ++k) {
                g_origin[k] = L[k];
                g_n[k] = (int)floor((H[k] - L[k]) / c) + 1;
            }
            grid[blockIdx.x] = make_double4(L[0], L[1], L[2], c);
            dims[blockIdx.x] = make_int4(g_n[0], g_n[1], g_n[2], 0);
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
    // keys
    int npow = 1;
    while (npow < sg.count) npow <<= 1;
    for (int i = tid; i < npow; i += nt) {
        unsigned long long key = ~0ull;
        if (i < sg.count) {
            double4 p = pos[sg.begin + i];
            double x[3] = {p.x, p.y, p.z};
            int c[3];
            for (int k = 0; k < 3; ++k) {
                double w = periodic ? (&gr.x)[k] : gr.w;
                int ci = (int)floor((x[k] - g_origin[k]) / w);
                if (periodic) ci = ci < 0 ? 0 : (ci >= g_n[k] ? g_n[k] - 1 : ci);
                c[k] = ci;
            }
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
            for (int k = 0; k < 3; ++k) {
                const double w = fp.periodic ? (&gr.x)[k] : gr.w;
                const double o = fp.periodic ? -0.5 * fp.box[k] : (&gr.x)[k];
                const int ci = (int)floor((x[k] - o) / w);
                c[k] = ci < 0 ? 0 : (ci >= nn[k] ? nn[k] - 1 : ci);
            }
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
            for (int nc = 0; nc < 27; ++nc) {
                const int lo = __shfl_sync(0xffffffffu, rg.x, nc);
                const int hi = __shfl_sync(0xffffffffu, rg.y, nc);
                for (int q = lo + lane; q < hi; q += 32) {
                    const int j = sidx[q];
                    if (j == i) continue;
                    const int a = i < j ? i : j, b = i < j ? j : i;
                    pair_term(fp, pos, Q, LJ, conn_ptr, conn_list, a, b, i, f, e_lj, e_c, cnt_c, cnt_lj, rep);
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

__device__ void v2n(const BondedArgs& A, const double4* pos, int p1, int p2, double* e, double& r, double& r_sq)
{
    dist_vec(pos[p1], pos[p2], A.periodic, A.box, A.inv_L, e);
    r_sq = sq3(e);
    r = sqrt(r_sq);
    double inv = 1 / r;
    e[0] *= inv;
    e[1] *= inv;
    e[2] *= inv;
}

__device__ void v3n(const BondedArgs& A, const double4* pos, int p1, int p2, int p3, double* e1, double* e2)
{
    dist_vec(pos[p1], pos[p2], A.periodic, A.box, A.inv_L, e1);
    dist_vec(pos[p3], pos[p2], A.periodic, A.box, A.inv_L, e2);
    double n1 = 1.0 / sqrt(sq3(e1)), n2 = 1.0 / sqrt(sq3(e2));
    for (int k = 0; k < 3; ++k) {
        e1[k] *= n1;
        e2[k] *= n2;
    }
}

__device__ __forceinline__ double dcos_m(int m, double c)
{
    switch (m) {
    case 1: return 1;
    case 2: return 4 * c;
    case 3: return 12 * c * c - 3;
    case 4: return c * (32 * c * c - 16);
    case 5: return c * c * (80 * c * c - 60) + 5;
    case 6: return c * (192 * c * c * (c * c - 1) + 36);
    default: return 0;
    }
}

__device__ __forceinline__ double cos_m(int m, double c)
{
    switch (m) {
    case 1: return c;
    case 2: return 2 * c * c - 1;
    case 3: return 4 * c * c * c - 3 * c;
    case 4: return 8 * c * c * (c * c - 1) + 1;
    case 5: return c * (c * c * (16 * c * c - 20) + 5);
    case 6: return c * c * (c * c * (32 * c * c - 48) + 18) - 1;
    default: return 1;
    }
}

__device__ __forceinline__ void cross3(const double* a, const double* b, double* o)
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
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
        // bond.c:43-85
        const int a = A.bond_pairs[2 * t], b = A.bond_pairs[2 * t + 1];
        const double r0 = A.bond_parms[3 * t], rmax = A.bond_parms[3 * t + 1], H = A.bond_parms[3 * t + 2];
        double e[3], r, r_sq;
        v2n(A, pos, a, b, e, r, r_sq);
        double Ff = 0, en = 0;
        if (r < rmax) {
            en = -0.5 * H * (rmax * rmax * log((rmax * rmax - r_sq) / (rmax * rmax - r0 * r0)) +
                             r0 * rmax * log((rmax + r) * (rmax - r0) / ((rmax - r) * (rmax + r0))));
            double dist_rmax = 1 - r_sq / (rmax * rmax);
            Ff = H * (r0 - r) / dist_rmax;
        } else {
            st |= ST_BOND;
        }
        slot = 2 * t;
        double* c = contrib + 3 * slot;
        for (int k = 0; k < 3; ++k) {
            c[k] = -Ff * e[k];
            c[3 + k] = Ff * e[k];
        }
        energy[t] = en;
        if (bad(Ff) || bad(e[0]) || bad(e[1]) || bad(e[2]) || bad(en)) st |= ST_OVERLAP;
    } else if ((t -= A.n_bond) < A.n_angle) {
        // angle.c:38-86
        const int* q = A.angle_pairs + 3 * t;
        const double phi0 = A.angle_parms[2 * t];
        double kphi = A.angle_parms[2 * t + 1];
        double e1[3], e2[3], Fi[3] = {0, 0, 0}, Fk[3] = {0, 0, 0}, en = 0;
        v3n(A, pos, q[0], q[1], q[2], e1, e2);
        double cphi = e1[0] * e2[0] + e1[1] * e2[1] + e1[2] * e2[2];
        cphi = cphi <= -1.0 ? -1.0 : (cphi >= 1.0 ? 1.0 : cphi);
        if (!(cphi >= 1 - 0.000001 || cphi <= -1 + 0.000001)) {
            double phi = acos(cphi);
            kphi *= (phi - phi0);
            en = 0.5 * kphi * (phi - phi0);
            kphi /= sqrt(1 - cphi * cphi);
            for (int k = 0; k < 3; ++k) {
                Fi[k] = -kphi * (e2[k] - e1[k] * cphi);
                Fk[k] = -kphi * (e1[k] - e2[k] * cphi);
            }
        }
        slot = 2 * A.n_bond + 3 * t;
        double* c = contrib + 3 * slot;
        for (int k = 0; k < 3; ++k) {
            c[k] = Fi[k];
            c[3 + k] = -Fi[k] - Fk[k];
            c[6 + k] = Fk[k];
        }
        energy[A.n_bond + t] = en;
        for (int k = 0; k < 3; ++k)
            if (bad(Fi[k]) || bad(Fk[k])) st |= ST_OVERLAP;
        if (bad(en)) st |= ST_OVERLAP;
    } else if ((t -= A.n_angle) < A.n_angle_cos) {
        // angle_cos.c:36-81
        const int* q = A.angle_cos_pairs + 3 * t;
        const double phi0 = A.angle_cos_parms[2 * t];
        double kphi = A.angle_cos_parms[2 * t + 1];
        double e1[3], e2[3], Fi[3], Fk[3];
        v3n(A, pos, q[0], q[1], q[2], e1, e2);
        double cphi = e1[0] * e2[0] + e1[1] * e2[1] + e1[2] * e2[2];
        cphi = cphi <= -1.0 ? -1.0 : (cphi >= 1.0 ? 1.0 : cphi);
        kphi *= (cphi - phi0);
        double en = 0.5 * kphi * (cphi - phi0);
        for (int k = 0; k < 3; ++k) {
            Fi[k] = kphi * (e2[k] - e1[k] * cphi);
            Fk[k] = kphi * (e1[k] - e2[k] * cphi);
        }
        slot = 2 * A.n_bond + 3 * A.n_angle + 3 * t;
        double* c = contrib + 3 * slot;
        for (int k = 0; k < 3; ++k) {
            c[k] = Fi[k];
            c[3 + k] = -Fi[k] - Fk[k];
            c[6 + k] = Fk[k];
        }
        energy[A.n_bond + A.n_angle + t] = en;
        for (int k = 0; k < 3; ++k)
            if (bad(Fi[k]) || bad(Fk[k])) st |= ST_OVERLAP;
        if (bad(en)) st |= ST_OVERLAP;
    } else if ((t -= A.n_angle_cos) < A.n_dihe) {
        // dihe.c:42-144
        const int* q = A.dihe_pairs + 4 * t;
        const double mkcd = A.dihe_parms[2 * t];
        const int m = (int)A.dihe_parms[2 * t + 1];
        double rkj[3], rij[3], rkl[3], rim[3], rln[3];
        double Fi[3] = {0, 0, 0}, Fj[3] = {0, 0, 0}, Fk[3] = {0, 0, 0}, Fl[3] = {0, 0, 0}, en = 0;
        dist_vec(pos[q[2]], pos[q[1]], A.periodic, A.box, A.inv_L, rkj);
        const double nkjsq = rkj[0] * rkj[0] + rkj[1] * rkj[1] + rkj[2] * rkj[2];
        dist_vec(pos[q[0]], pos[q[1]], A.periodic, A.box, A.inv_L, rij);
        dist_vec(pos[q[2]], pos[q[3]], A.periodic, A.box, A.inv_L, rkl);
        const double sijkj = (rij[0] * rkj[0] + rij[1] * rkj[1] + rij[2] * rkj[2]) / nkjsq;
        const double sklkj = (rkl[0] * rkj[0] + rkl[1] * rkj[1] + rkl[2] * rkj[2]) / nkjsq;
        for (int k = 0; k < 3; ++k) {
            rim[k] = -rij[k] + sijkj * rkj[k];
            rln[k] = rkl[k] - sklkj * rkj[k];
        }
        const double nim = sqrt(rim[0] * rim[0] + rim[1] * rim[1] + rim[2] * rim[2]);
        const double nln = sqrt(rln[0] * rln[0] + rln[1] * rln[1] + rln[2] * rln[2]);
        if (!(fabs(nim) < 0.000001) && !(fabs(nln) < 0.000001)) {
            const double inv_nrim = 1.0 / nim, inv_nrln = 1.0 / nln;
            double ct = (rim[0] * rln[0] + rim[1] * rln[1] + rim[2] * rln[2]) * inv_nrln * inv_nrim;
            ct = ct < -1 ? -1 : (ct > 1 ? 1 : ct);
            en = fabs(mkcd) * (1 + fabs(mkcd) * cos_m(m, ct));
            const double dc = dcos_m(m, ct);
            double tmp = mkcd * dc * inv_nrim;
            for (int k = 0; k < 3; ++k) Fi[k] = tmp * (rln[k] * inv_nrln - rim[k] * inv_nrim * ct);
            tmp = mkcd * dc * inv_nrln;
            for (int k = 0; k < 3; ++k) Fl[k] = tmp * (rim[k] * inv_nrim - rln[k] * inv_nrln * ct);
            for (int k = 0; k < 3; ++k) Fj[k] = (sijkj - 1) * Fi[k] - sklkj * Fl[k];
            for (int k = 0; k < 3; ++k) Fk[k] = -Fi[k] - Fj[k] - Fl[k];
        }
        slot = 2 * A.n_bond + 3 * A.n_angle + 3 * A.n_angle_cos + 4 * t;
        double* c = contrib + 3 * slot;
        for (int k = 0; k < 3; ++k) {
            c[k] = Fi[k];
            c[3 + k] = Fj[k];
            c[6 + k] = Fk[k];
            c[9 + k] = Fl[k];
        }
        energy[A.n_bond + A.n_angle + A.n_angle_cos + t] = en;
        for (int k = 0; k < 3; ++k)
            if (bad(Fi[k]) || bad(Fj[k]) || bad(Fk[k]) || bad(Fl[k])) st |= ST_OVERLAP;
        if (bad(en)) st |= ST_OVERLAP;
    } else if ((t -= A.n_dihe) < A.n_dihe_angle) {
        // dihe_angle.c:43-255 (no periodic images: measureAndCalcGradDihedral
        // takes raw coordinate differences)
        const int* q = A.dihe_angle_pairs + 4 * t;
        double kt = A.dihe_angle_parms[2 * t];
        const double t0 = A.dihe_angle_parms[2 * t + 1];
        const double4 P1 = pos[q[0]], P2 = pos[q[1]], P3 = pos[q[2]], P4 = pos[q[3]];
        double r12[3] = {P2.x - P1.x, P2.y - P1.y, P2.z - P1.z};
        double r23[3] = {P3.x - P2.x, P3.y - P2.y, P3.z - P2.z};
        double r34[3] = {P4.x - P3.x, P4.y - P3.y, P4.z - P3.z};
        double Av[3], Bv[3], Cv[3], f1[3], f2[3], f3[3];
        cross3(r12, r23, Av);
        cross3(r23, r34, Bv);
        cross3(r23, Av, Cv);
        const double rA = 1.0 / sqrt(Av[0] * Av[0] + Av[1] * Av[1] + Av[2] * Av[2]);
        const double rB = 1.0 / sqrt(Bv[0] * Bv[0] + Bv[1] * Bv[1] + Bv[2] * Bv[2]);
        const double rC = 1.0 / sqrt(Cv[0] * Cv[0] + Cv[1] * Cv[1] + Cv[2] * Cv[2]);
        double cp = (Av[0] * Bv[0] + Av[1] * Bv[1] + Av[2] * Bv[2]) * (rA * rB);
        double sp = (Cv[0] * Bv[0] + Cv[1] * Bv[1] + Cv[2] * Bv[2]) * (rC * rB);
        cp = cp < -1 ? -1 : (cp > 1 ? 1 : cp);
        sp = sp < -1 ? -1 : (sp > 1 ? 1 : sp);
        const double phi = -atan2(sp, cp);
        for (int k = 0; k < 3; ++k) Bv[k] *= rB;
        if (fabs(sp) > 0.1) {
            double dA[3], dB[3];
            for (int k = 0; k < 3; ++k) Av[k] *= rA;
            for (int k = 0; k < 3; ++k) {
                dA[k] = rA * (cp * Av[k] - Bv[k]);
                dB[k] = rB * (cp * Bv[k] - Av[k]);
            }
            const double K1 = 1.0 / sp;
            f1[0] = K1 * (r23[1] * dA[2] - r23[2] * dA[1]);
            f1[1] = K1 * (r23[2] * dA[0] - r23[0] * dA[2]);
            f1[2] = K1 * (r23[0] * dA[1] - r23[1] * dA[0]);
            f3[0] = K1 * (r23[2] * dB[1] - r23[1] * dB[2]);
            f3[1] = K1 * (r23[0] * dB[2] - r23[2] * dB[0]);
            f3[2] = K1 * (r23[1] * dB[0] - r23[0] * dB[1]);
            f2[0] = K1 * (r12[2] * dA[1] - r12[1] * dA[2] + r34[1] * dB[2] - r34[2] * dB[1]);
            f2[1] = K1 * (r12[0] * dA[2] - r12[2] * dA[0] + r34[2] * dB[0] - r34[0] * dB[2]);
            f2[2] = K1 * (r12[1] * dA[0] - r12[0] * dA[1] + r34[0] * dB[1] - r34[1] * dB[0]);
        } else {
            double dC[3], dB[3];
            for (int k = 0; k < 3; ++k) Cv[k] *= rC;
            for (int k = 0; k < 3; ++k) {
                dC[k] = rC * (sp * Cv[k] - Bv[k]);
                dB[k] = rB * (sp * Bv[k] - Cv[k]);
            }
            const double K1 = -1.0 / cp;
            f1[0] = K1 * ((r23[1] * r23[1] + r23[2] * r23[2]) * dC[0] - r23[0] * r23[1] * dC[1] - r23[0] * r23[2] * dC[2]);
            f1[1] = K1 * ((r23[2] * r23[2] + r23[0] * r23[0]) * dC[1] - r23[1] * r23[2] * dC[2] - r23[1] * r23[0] * dC[0]);
            f1[2] = K1 * ((r23[0] * r23[0] + r23[1] * r23[1]) * dC[2] - r23[2] * r23[0] * dC[0] - r23[2] * r23[1] * dC[1]);
            cross3(dB, r23, f3);
            for (int k = 0; k < 3; ++k) f3[k] *= K1;
            f2[0] = K1 * (-(r23[1] * r12[1] + r23[2] * r12[2]) * dC[0] + (2.0 * r23[0] * r12[1] - r12[0] * r23[1]) * dC[1] +
                          (2.0 * r23[0] * r12[2] - r12[0] * r23[2]) * dC[2] + dB[2] * r34[1] - dB[1] * r34[2]);
            f2[1] = K1 * (-(r23[2] * r12[2] + r23[0] * r12[0]) * dC[1] + (2.0 * r23[1] * r12[2] - r12[1] * r23[2]) * dC[2] +
                          (2.0 * r23[1] * r12[0] - r12[1] * r23[0]) * dC[0] + dB[0] * r34[2] - dB[2] * r34[0]);
            f2[2] = K1 * (-(r23[0] * r12[0] + r23[1] * r12[1]) * dC[2] + (2.0 * r23[2] * r12[0] - r12[2] * r23[0]) * dC[0] +
                          (2.0 * r23[2] * r12[1] - r12[2] * r23[1]) * dC[1] + dB[1] * r34[0] - dB[0] * r34[1]);
        }
        double g[12];
        for (int k = 0; k < 3; ++k) {
            g[k] = f1[k];
            g[3 + k] = f2[k] - f1[k];
            g[6 + k] = f3[k] - f2[k];
            g[9 + k] = -f3[k];
        }
        double tmp = phi - t0;
        const double pif = (double)BDB_M_PIF;
        if (tmp < -pif) tmp += 2 * pif;
        if (tmp > pif) tmp -= 2 * pif;
        kt *= -tmp;
        const double en = -(0.5 * kt * tmp);
        slot = 2 * A.n_bond + 3 * A.n_angle + 3 * A.n_angle_cos + 4 * A.n_dihe + 4 * t;
        double* c = contrib + 3 * slot;
        for (int k = 0; k < 12; ++k) {
            c[k] = kt * g[k];
            if (bad(g[k])) st |= ST_OVERLAP;
        }
        energy[A.n_bond + A.n_angle + A.n_angle_cos + A.n_dihe + t] = en;
        if (bad(kt) || bad(en)) st |= ST_OVERLAP;
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
        if (count) cudaMemcpy(v.data(), b.p, sizeof(int) * count, cudaMemcpyDeviceToHost);
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
    BDB_CUDA(cudaMemcpy(s->slot_ptr.p, ptr.data(), sizeof(int) * (s->n + 1), cudaMemcpyHostToDevice));
    if (!list.empty())
        BDB_CUDA(cudaMemcpy(s->slot_list.p, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice));

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
    BDB_CUDA(cudaMemcpy(s->conn_ptr.p, cptr.data(), sizeof(int) * (s->n + 1), cudaMemcpyHostToDevice));
    if (!clist.empty())
        BDB_CUDA(cudaMemcpy(s->conn_list.p, clist.data(), sizeof(int) * clist.size(), cudaMemcpyHostToDevice));
    return BDB_OK;
}

int forces_setup(bdb_system* s)
{
    const int nseg = (int)s->segs.size();
    if (s->sorted_keys.alloc(s->n)) return BDB_ERR_NOMEM;
    if (s->sorted_idx.alloc(s->n)) return BDB_ERR_NOMEM;
    if (s->grid.alloc(nseg)) return BDB_ERR_NOMEM;
    if (s->grid_dims.alloc(nseg)) return BDB_ERR_NOMEM;
    if (s->pos_build.alloc(s->n) || s->cells_built.alloc(nseg)) return BDB_ERR_NOMEM;
    BDB_CUDA(cudaMemset(s->cells_built.p, 0, sizeof(int) * nseg));
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
    BDB_CUDA(cudaMemcpy(s->cell_off.p, off.data(), sizeof(long long) * 2 * nseg, cudaMemcpyHostToDevice));
    if (s->e_part.alloc(2 * s->n + 16)) return BDB_ERR_NOMEM;
    if (s->status.alloc(4)) return BDB_ERR_NOMEM;
    if (s->counts.alloc(2)) return BDB_ERR_NOMEM;
    if (s->F.alloc(3 * s->n) || s->F_save.alloc(3 * s->n) || s->work.alloc(3 * s->n + 16)) return BDB_ERR_NOMEM;
    BDB_CUDA(cudaFuncSetAttribute(k_cells, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  SORT_MAX * (int)sizeof(unsigned long long)));
    // cell size: the widest interaction range of force_single plus the
    // LJ_force_check distance (init_cutoff, pre_func.c:197-232)
    std::vector<double2> lj(s->n);
    BDB_CUDA(cudaMemcpy(lj.data(), s->LJ.p, sizeof(double2) * s->n, cudaMemcpyDeviceToHost));
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
                                      s->pos_build.p, s->cells_built.p, s->cell_range.p, s->cell_off.p);
    BDB_CUDA(cudaGetLastError());
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
