// Gaussian noise and the position update.
//
// rand_move.c:132-168 draws unit Gaussians on the host (Marsaglia polar on
// drand48_r) and the reference GPU build copies them to the device every
// step (diff_alg/cuda/diff_rand.cu:143-180). Here they are either generated
// on the device -- Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) keyed
// by the seed, counter = (step, pair index), two 53-bit uniforms per call
// and the Box-Muller transform -- or copied from a caller array (parity
// runs that replay the reference's exact stream).
//
// The same kernel applies the per-method scaling of compute_r
// (diff_rand.c:47-236): sqrt(2 dt) for Cholesky, sqrt(2 dt / D_ii) for TEA,
// sqrt(2 dt D_ii) for hydro none.
#include <cuda_runtime.h>

#include "bdb_common.cuh"
#include "philox.cuh"

namespace bdb {

// mode: 1 cholesky sqrt(2 dt); 2 TEA sqrt(2 dt / D_ii); 0 none sqrt(D_ii 2 dt)
// The Philox stream index (one per call) lives in device memory, ctr[0],
// so that a step captured once in a CUDA graph draws fresh noise on every
// replay; the last block to finish advances it (ctr[1] counts finished
// blocks). ctr[2] tags noise drawn ahead by the fused Cholesky step
// (matvec.cu): this kernel overwrites X, so it clears the tag.
__global__ void k_noise(int n3, int mode, double dt, double preDii, const double4* __restrict__ pos,
                        const double* __restrict__ host_g, uint64_t seed, unsigned long long* __restrict__ ctr,
                        double* __restrict__ X)
{
    const uint64_t stream = *reinterpret_cast<volatile unsigned long long*>(ctr);
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int i0 = 2 * t;
    if (i0 < n3) {
        double g[2];
        if (host_g) {
            g[0] = host_g[i0];
            g[1] = i0 + 1 < n3 ? host_g[i0 + 1] : 0.0;
        } else {
            gauss2(seed, stream, (uint32_t)t, g[0], g[1]);
        }
        for (int q = 0; q < 2; ++q) {
            const int i = i0 + q;
            if (i >= n3) break;
            const double d = preDii / pos[i / 3].w;   // diag_D (diff_decl.c:94-99)
            double sc;
            if (mode == 1) sc = sqrt(2 * dt);
            else if (mode == 2) sc = sqrt(2 * dt * (1 / d));
            else sc = sqrt(d * 2 * dt);
            X[i] = g[q] * sc;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned done = atomicAdd(reinterpret_cast<unsigned*>(ctr + 1), 1u);
        if (done == gridDim.x - 1) {
            ctr[1] = 0;
            ctr[2] = 0;
            ctr[0] = stream + 1;
            __threadfence();
        }
    }
}

int noise_fill(bdb_system* s, const double* dev_gauss)
{
    const int n3 = s->n3;
    const int threads = (n3 + 1) / 2;
    k_noise<<<(threads + 255) / 256, 256, 0, s->stream>>>(n3, s->p.hydro, s->p.dt, s->preDii, s->pos.p, dev_gauss,
                                                          s->p.seed, s->ctr.p, s->X.p);
    BDB_CUDA(cudaGetLastError());
    s->launches += 1;
    return BDB_OK;
}

// Flowing solvent (vel_grad_tensor, diff_decl.c:72): the displacement
// dt G r of the flow at the step's start, G row-major
struct Flow {
    int on;
    double dt, G[9];
};

// coord_out = Rf + Rs + coord (+ dt G coord in a flow); trans_to_box
// (diff_equation.c:254-283)
__global__ void k_update(int n, int periodic, double3 box, double3 inv_L, Flow fl, const double* __restrict__ Rf,
                         const double* __restrict__ Rs, double4* __restrict__ pos, double* __restrict__ fs)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 p = pos[i];
    const double x = p.x, y = p.y, z = p.z;
    p.x = add(add(Rf[3 * i], Rs[3 * i]), p.x);
    p.y = add(add(Rf[3 * i + 1], Rs[3 * i + 1]), p.y);
    p.z = add(add(Rf[3 * i + 2], Rs[3 * i + 2]), p.z);
    if (fl.on) {
        const double* G = fl.G;
        const double t0 = mul(fl.dt, add(add(mul(G[0], x), mul(G[1], y)), mul(G[2], z)));
        const double t1 = mul(fl.dt, add(add(mul(G[3], x), mul(G[4], y)), mul(G[5], z)));
        const double t2 = mul(fl.dt, add(add(mul(G[6], x), mul(G[7], y)), mul(G[8], z)));
        p.x = add(p.x, t0);
        p.y = add(p.y, t1);
        p.z = add(p.z, t2);
        if (fs) {
            // the flow displacement of an IGT predictor, FS = tmp + dt G r'
            // at the unwrapped predicted position (diff_equation.c:275-277)
            fs[3 * i] = add(t0, mul(fl.dt, add(add(mul(G[0], p.x), mul(G[1], p.y)), mul(G[2], p.z))));
            fs[3 * i + 1] = add(t1, mul(fl.dt, add(add(mul(G[3], p.x), mul(G[4], p.y)), mul(G[5], p.z))));
            fs[3 * i + 2] = add(t2, mul(fl.dt, add(add(mul(G[6], p.x), mul(G[7], p.y)), mul(G[8], p.z))));
        }
    }
    if (periodic) {
        p.x = sub(p.x, mul(box.x, floor(add(mul(p.x, inv_L.x), 0.5))));
        p.y = sub(p.y, mul(box.y, floor(add(mul(p.y, inv_L.y), 0.5))));
        p.z = sub(p.z, mul(box.z, floor(add(mul(p.z, inv_L.z), 0.5))));
    }
    pos[i] = p;
}

int update_positions(bdb_system* s, double* fs)
{
    Flow fl;
    fl.on = s->p.flow && s->p.bc != 2;   // a sphere turns the flow off (input.c:462-468)
    fl.dt = s->p.dt;
    for (int k = 0; k < 9; ++k) fl.G[k] = s->p.vel_grad[k];
    k_update<<<(s->n + 127) / 128, 128, 0, s->stream>>>(
        s->n, s->p.bc == 1, make_double3(s->p.box[0], s->p.box[1], s->p.box[2]),
        make_double3(s->inv_L[0], s->inv_L[1], s->inv_L[2]), fl, s->Rf.p, s->Rs.p, s->pos.p, fl.on ? fs : nullptr);
    s->launches += 1;
    BDB_CUDA(cudaGetLastError());
    return BDB_OK;
}

}  // namespace bdb
