// Elastic-collision overlap removal: the recovery of comp_step_ermak_newton
// (diff_comp.c:181-210) after a move that overlaps. From the step's saved
// start state (bdb_save_state) and the overlapping move:
//   newton_init_vel (newton.c:202-213)  v = (r - r_start) / dt, r = r_start;
//   newton_moves    (newton.c:140-200)  until dt has elapsed: the earliest
//                   contact time of the approaching pairs (comp_time,
//                   newton.c:57-138), a ballistic move to just before it,
//                   and elastic collisions of the pairs that reach it;
// then the forces at the result. The pair scan is an all-pairs kernel with
// a min-reduction of the contact time (a non-negative double compares like
// its bit pattern) and a second pass that collects the pairs at that time;
// the host orders them as BD_BOX's serial loop does (i, then j) and a
// one-thread kernel applies the collisions in that order. All arithmetic
// mirrors BD_BOX's operation order without contraction, so that the
// contact-time comparisons decide the same way.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstring>
#include <vector>

#include "bdb_common.cuh"

namespace bdb {

static constexpr double NW_EPSILON = 0.000001;   // NEWTON_EPSILON (data.h:217)
static constexpr double NW_OFFSET = 0.0001;      // NEWTON_OFFSET (data.h:218)

struct NwGeom {
    int periodic;
    double box[3], inv_L[3];
};

// trans_dist_vec(a, b) (trans.c:111-122): b - a, nearest image in the box
__device__ __forceinline__ void nw_dist(const NwGeom& g, const double* a, const double* b, double* v)
{
    for (int k = 0; k < 3; ++k) {
        v[k] = sub(b[k], a[k]);
        if (g.periodic) v[k] = sub(v[k], mul(g.box[k], floor(add(mul(v[k], g.inv_L[k]), 0.5))));
    }
}

__device__ __forceinline__ void xyz(const double4& p, double* c)
{
    c[0] = p.x;
    c[1] = p.y;
    c[2] = p.z;
}

__global__ void k_nw_init(int n, NwGeom g, double inv_t, double4* __restrict__ pos,
                          const double4* __restrict__ pos_save, double* __restrict__ vel)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double a[3], b[3], v[3];
    xyz(pos_save[i], a);
    xyz(pos[i], b);
    nw_dist(g, a, b, v);
    for (int k = 0; k < 3; ++k) vel[3 * i + k] = mul(v[k], inv_t);
    pos[i] = pos_save[i];
}

// contact time of pair (i, j), i < j, or -1 when it does not approach
__device__ __forceinline__ double nw_t2(const NwGeom& g, const double4* pos, const double* vel, const double2* LJ,
                                        int i, int j)
{
    double ci[3], cj[3], r[3], v[3];
    xyz(pos[i], ci);
    xyz(pos[j], cj);
    nw_dist(g, cj, ci, r);
    const double l = add(add(LJ[j].x, LJ[i].x), NW_OFFSET);   // sigma/2 of both beads
    for (int k = 0; k < 3; ++k) v[k] = sub(vel[3 * i + k], vel[3 * j + k]);
    const double rv = add(add(mul(r[0], v[0]), mul(r[1], v[1])), mul(r[2], v[2]));
    if (!(rv < 0)) return -1.0;
    const double vv = add(add(mul(v[0], v[0]), mul(v[1], v[1])), mul(v[2], v[2]));
    const double rr = add(add(mul(r[0], r[0]), mul(r[1], r[1])), mul(r[2], r[2]));
    double delta = sub(mul(rv, rv), mul(vv, sub(rr, mul(l, l))));
    if (!(delta > 0)) return -1.0;
    const double inv_vv = 1.0 / vv;
    delta = sqrt(delta);
    const double t2 = mul(-add(rv, delta), inv_vv);
    return t2 < 0 ? 0.0 : t2;
}

__global__ void k_nw_time(int n, NwGeom g, const double4* __restrict__ pos, const double* __restrict__ vel,
                          const double2* __restrict__ LJ, unsigned long long* __restrict__ tmin)
{
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || j >= n || j <= i) return;
    const double t2 = nw_t2(g, pos, vel, LJ, i, j);
    if (t2 >= 0) atomicMin(tmin, (unsigned long long)__double_as_longlong(t2));
}

__global__ void k_nw_pairs(int n, NwGeom g, const double4* __restrict__ pos, const double* __restrict__ vel,
                           const double2* __restrict__ LJ, const unsigned long long* __restrict__ tmin,
                           int* __restrict__ npairs, int2* __restrict__ pairs, int cap)
{
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || j >= n || j <= i) return;
    const double t2 = nw_t2(g, pos, vel, LJ, i, j);
    if (t2 >= 0 && (unsigned long long)__double_as_longlong(t2) == *tmin) {
        const int k = atomicAdd(npairs, 1);
        if (k < cap) pairs[k] = make_int2(i, j);
    }
}

// ballistic move; bc sphere: flag a bead outside the sphere (iscorrect)
__global__ void k_nw_move(int n, NwGeom g, double t, int sphere, double sr, double4* __restrict__ pos,
                          const double* __restrict__ vel, int* __restrict__ outside)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 p = pos[i];
    p.x = add(p.x, mul(vel[3 * i], t));
    p.y = add(p.y, mul(vel[3 * i + 1], t));
    p.z = add(p.z, mul(vel[3 * i + 2], t));
    if (g.periodic) {
        p.x = sub(p.x, mul(g.box[0], floor(add(mul(p.x, g.inv_L[0]), 0.5))));
        p.y = sub(p.y, mul(g.box[1], floor(add(mul(p.y, g.inv_L[1]), 0.5))));
        p.z = sub(p.z, mul(g.box[2], floor(add(mul(p.z, g.inv_L[2]), 0.5))));
    }
    pos[i] = p;
    if (sphere && add(add(mul(p.x, p.x), mul(p.y, p.y)), mul(p.z, p.z)) > sr) atomicOr(outside, 1);
}

// the collisions, one after the other in the given order (one thread)
__global__ void k_nw_collide(int np, const int2* __restrict__ pairs, NwGeom g, const double4* __restrict__ pos,
                             const double* __restrict__ mass, double e_collision, double* __restrict__ vel)
{
    if (blockIdx.x || threadIdx.x) return;
    for (int q = 0; q < np; ++q) {
        const int p1 = pairs[q].x, p2 = pairs[q].y;
        double c1[3], c2[3], e[3], v[3];
        xyz(pos[p1], c1);
        xyz(pos[p2], c2);
        // get_v2_norms(p2, p1) (math_help.c:40-55)
        nw_dist(g, c2, c1, e);
        const double rr = sqrt(add(add(mul(e[0], e[0]), mul(e[1], e[1])), mul(e[2], e[2])));
        const double inv = 1.0 / rr;
        for (int k = 0; k < 3; ++k) e[k] = mul(e[k], inv);
        for (int k = 0; k < 3; ++k) v[k] = sub(vel[3 * p1 + k], vel[3 * p2 + k]);
        const double m1 = mass[p1], m2 = mass[p2];
        double ev = add(add(mul(e[0], v[0]), mul(e[1], v[1])), mul(e[2], v[2]));
        ev = mul(ev, (1 + e_collision) / add(m1, m2));
        for (int k = 0; k < 3; ++k) vel[3 * p1 + k] = sub(vel[3 * p1 + k], mul(mul(m2, ev), e[k]));
        for (int k = 0; k < 3; ++k) vel[3 * p2 + k] = add(vel[3 * p2 + k], mul(mul(m1, ev), e[k]));
    }
}

static unsigned long long bits_of(double x)
{
    unsigned long long b;
    std::memcpy(&b, &x, sizeof b);
    return b;
}

static double double_of(unsigned long long b)
{
    double x;
    std::memcpy(&x, &b, sizeof x);
    return x;
}

}  // namespace bdb

using namespace bdb;

extern "C" int bdb_newton_resolve(bdb_system* s, double e_collision, const double* masses, int move_attempts,
                                  int* count)
{
    if (!s || !masses || !count) return fail(BDB_ERR_ARG, "null argument");
    if (s->segs.size() != 1) return fail(BDB_ERR_UNSUPPORTED, "elastic collisions need a single system");
    const int n = s->n;
    cudaStream_t st = s->stream;
    if (s->nw_vel.n < (size_t)3 * n && s->nw_vel.alloc(3 * (size_t)n)) return BDB_ERR_NOMEM;
    if (s->nw_mass.n < (size_t)n && s->nw_mass.alloc(n)) return BDB_ERR_NOMEM;
    if (s->nw_pairs.n < (size_t)2 * n && s->nw_pairs.alloc(2 * (size_t)n)) return BDB_ERR_NOMEM;
    if (s->nw_scal.n < 3 && s->nw_scal.alloc(3)) return BDB_ERR_NOMEM;
    BDB_CUDA(cudaMemcpyAsync(s->nw_mass.p, masses, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    NwGeom g;
    g.periodic = s->p.bc == 1;
    for (int k = 0; k < 3; ++k) {
        g.box[k] = s->p.box[k];
        g.inv_L[k] = s->inv_L[k];
    }
    const double dt = s->p.dt;
    const int threads = 128, blocks = (n + threads - 1) / threads;
    const dim3 pb(16, 16), pg((n + 15) / 16, (n + 15) / 16);
    unsigned long long* tmin = s->nw_scal.p;
    int* npairs = reinterpret_cast<int*>(s->nw_scal.p + 1);
    int* outside = reinterpret_cast<int*>(s->nw_scal.p + 2);
    k_nw_init<<<blocks, threads, 0, st>>>(n, g, 1.0 / dt, s->pos.p, s->pos_save.p, s->nw_vel.p);
    BDB_CUDA(cudaGetLastError());
    s->launches += 1;
    std::vector<int2> hp;
    int& prev_ints = s->nw_prev_ints;   // BD_BOX's global size_pairs: the list check reads the previous scan's
    double elapsed = 0.0;
    int ret = 0;
    while (elapsed < dt - 2 * NW_EPSILON) {
        ret = 0;
        // comp_time
        const unsigned long long none = bits_of(DBL_MAX);
        BDB_CUDA(cudaMemcpyAsync(tmin, &none, sizeof none, cudaMemcpyHostToDevice, st));
        BDB_CUDA(cudaMemsetAsync(s->nw_scal.p + 1, 0, 2 * sizeof(unsigned long long), st));
        k_nw_time<<<pg, pb, 0, st>>>(n, g, s->pos.p, s->nw_vel.p, s->LJ.p, tmin);
        k_nw_pairs<<<pg, pb, 0, st>>>(n, g, s->pos.p, s->nw_vel.p, s->LJ.p, tmin, npairs,
                                      reinterpret_cast<int2*>(s->nw_pairs.p), n);
        BDB_CUDA(cudaGetLastError());
        s->launches += 2;
        unsigned long long tb = 0;
        int np = 0;
        BDB_CUDA(cudaMemcpyAsync(&tb, tmin, sizeof tb, cudaMemcpyDeviceToHost, st));
        BDB_CUDA(cudaMemcpyAsync(&np, npairs, sizeof np, cudaMemcpyDeviceToHost, st));
        BDB_CUDA(cudaStreamSynchronize(st));
        np = std::min(np, n);
        hp.resize(np);
        if (np) {
            BDB_CUDA(d2h(s, hp.data(), s->nw_pairs.p, sizeof(int2) * np));
            std::sort(hp.begin(), hp.end(), [](const int2& a, const int2& b) {
                return a.x != b.x ? a.x < b.x : a.y < b.y;
            });
        }
        if (!(prev_ints + 1 < 2 * n)) hp.clear();
        prev_ints = 2 * (int)hp.size();
        double next = double_of(tb);
        // newton_moves
        if (next < 0 || next > dt - elapsed) next = dt - elapsed;
        next = (next > NW_EPSILON) ? next - NW_EPSILON : 0;
        elapsed += next;
        if (next > 0.0) {
            const int sphere = s->p.bc == 2;
            k_nw_move<<<blocks, threads, 0, st>>>(n, g, next, sphere, s->p.sphere_radius * s->p.sphere_radius,
                                                 s->pos.p, s->nw_vel.p, outside);
            BDB_CUDA(cudaGetLastError());
            s->launches += 1;
            if (sphere) {
                int out = 0;
                BDB_CUDA(cudaMemcpyAsync(&out, outside, sizeof out, cudaMemcpyDeviceToHost, st));
                BDB_CUDA(cudaStreamSynchronize(st));
                ret = out != 0;
            }
        }
        if (ret) break;
        if (!hp.empty()) {
            BDB_CUDA(cudaMemcpyAsync(s->nw_pairs.p, hp.data(), sizeof(int2) * hp.size(), cudaMemcpyHostToDevice, st));
            k_nw_collide<<<1, 1, 0, st>>>((int)hp.size(), reinterpret_cast<int2*>(s->nw_pairs.p), g, s->pos.p,
                                          s->nw_mass.p, e_collision, s->nw_vel.p);
            BDB_CUDA(cudaGetLastError());
            s->launches += 1;
            BDB_CUDA(cudaStreamSynchronize(st));   // hp is reused by the next round
        }
        ++*count;
        if (*count > move_attempts) return fail(BDB_ERR_ARG, "Ermak Newton error");
    }
    // the forces at the result, at the step's end time
    BDB_CUDA(cudaMemsetAsync(s->status.p, 0, sizeof(unsigned), st));
    s->have_forces = false;
    int rc = forces_run(s, false, false);
    if (rc) return rc;
    bool ov = false;
    if ((rc = check_status(s, &ov))) return rc;
    if (ret || ov) return 1;
    // the step's frame, if one was taken of the overlapping move
    if ((rc = frames_redo_current(s))) return rc;
    return 0;
}
