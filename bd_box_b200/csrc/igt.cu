// IGT predictor-corrector step (comp_step_IGT_const, diff_comp.c:76-107;
// compute_hydro_IGT and compute_hydro_IGT_second_phase,
// diff_equation.c:288-374) for hydro none and the stored-tensor (Cholesky)
// path, in either precision.
//
// One step from positions r with forces F = F(r):
//   predictor  D(r) built and factored in the stored matrix M (upper: D,
//              lower: L), Rf = dt/kT D F, Rs = L X1 (X1 scaled Gaussians),
//              r' = r + Rf + Rs (periodic wrap), as compute_hydro_ermak;
//   forces     F' = F(r');
//   tensor     D(r') built into the second matrix M', Rf' = dt/kT D(r') F';
//   average    lower triangle of M = (D(r) + D(r'))/2, D(r) read from the
//              upper triangle of M and diag(D) at r (the diagonal 3x3 blocks
//              do not depend on the positions, so averaging them too leaves
//              them bit for bit);
//   corrector  M factored again, Rs = L X2 with fresh Gaussians,
//              r <- r + ((Rf + Rf')/2 + Rs) (periodic wrap), F = F(r).
// No retries: the overlap flags of both force passes are returned (bit 0
// the forces at r', bit 1 the forces after the step), as bdb_step leaves
// comp_step_ermak's retries to the caller.
#include <algorithm>
#include <utility>

#include "bdb_common.cuh"

namespace bdb {

// lower triangle (and diagonal) of M = (D(r) + D(r'))/2 over the real rows
// and columns (< n3), 32x32 blocks: D(r) from the upper triangle of M (read
// transposed through shared memory) and dD0 on the diagonal, D(r') from M'
template <typename T>
__global__ void k_igt_average(int n3, int npad, T* __restrict__ M, const T* __restrict__ Mp,
                              const double* __restrict__ dD0)
{
    const int bi = blockIdx.y, bj = blockIdx.x;
    if (bj > bi) return;
    __shared__ T up[32][33];
    const int tx = threadIdx.x, ty = threadIdx.y;   // 32 x 8
    // upper block (bj, bi) of M: rows 32 bj.., columns 32 bi..
    for (int r = ty; r < 32; r += 8) {
        const int row = 32 * bj + r, col = 32 * bi + tx;
        up[tx][r] = (row < n3 && col < n3) ? M[(size_t)row * npad + col] : T(0);
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int row = 32 * bi + r, col = 32 * bj + tx;
        if (row >= n3 || col >= n3 || col > row) continue;
        const double a = row == col ? dD0[row] : (double)up[r][tx];
        const double b = (double)Mp[(size_t)row * npad + col];
        M[(size_t)row * npad + col] = (T)((a + b) / 2);
    }
}

// r <- r0 + ((Rf1 + Rf2)/2 + Rs), periodic wrap (diff_equation.c:296-301
// with Rf0 = (Rf + Rs)/2 from :333-336)
__global__ void k_igt_update(int n, int periodic, double3 box, double3 inv_L, const double4* __restrict__ pos0,
                             const double* __restrict__ Rf1, const double* __restrict__ Rf2,
                             const double* __restrict__ Rs, const double* __restrict__ fs, double4* __restrict__ pos)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 p = pos0[i];
    const double d0 = mul(0.5, add(Rf1[3 * i], Rf2[3 * i]));
    const double d1 = mul(0.5, add(Rf1[3 * i + 1], Rf2[3 * i + 1]));
    const double d2 = mul(0.5, add(Rf1[3 * i + 2], Rf2[3 * i + 2]));
    if (fs) {
        // in a flowing solvent, half the predictor's flow displacement too
        // (diff_equation.c:303-311)
        p.x = add(p.x, add(add(d0, Rs[3 * i]), mul(0.5, fs[3 * i])));
        p.y = add(p.y, add(add(d1, Rs[3 * i + 1]), mul(0.5, fs[3 * i + 1])));
        p.z = add(p.z, add(add(d2, Rs[3 * i + 2]), mul(0.5, fs[3 * i + 2])));
    } else {
        p.x = add(p.x, add(d0, Rs[3 * i]));
        p.y = add(p.y, add(d1, Rs[3 * i + 1]));
        p.z = add(p.z, add(d2, Rs[3 * i + 2]));
    }
    if (periodic) {
        p.x = sub(p.x, mul(box.x, floor(add(mul(p.x, inv_L.x), 0.5))));
        p.y = sub(p.y, mul(box.y, floor(add(mul(p.y, inv_L.y), 0.5))));
        p.z = sub(p.z, mul(box.z, floor(add(mul(p.z, inv_L.z), 0.5))));
    }
    pos[i] = p;
}

// the second stored matrix, with the same identity padding as the first
static int ensure_matrix_b(bdb_system* s)
{
    const size_t nn = (size_t)s->npad * s->npad;
    if (s->p.precision == BDB_PREC_FP64) {
        if (s->M64b.p) return BDB_OK;
        if (s->M64b.alloc(nn)) return BDB_ERR_NOMEM;
        BDB_CUDA(dzero(s, s->M64b.p, nn * sizeof(double)));
        const double one = 1.0;
        for (int r = s->n3; r < s->npad; ++r)
            BDB_CUDA(h2d(s, s->M64b.p + (size_t)r * s->npad + r, &one, sizeof(double)));
    } else {
        if (s->M32b.p) return BDB_OK;
        if (s->M32b.alloc(nn)) return BDB_ERR_NOMEM;
        BDB_CUDA(dzero(s, s->M32b.p, nn * sizeof(float)));
        const float one = 1.0f;
        for (int r = s->n3; r < s->npad; ++r)
            BDB_CUDA(h2d(s, s->M32b.p + (size_t)r * s->npad + r, &one, sizeof(float)));
    }
    return BDB_OK;
}

// the build and the stored product write and read M; pointing M at the
// second matrix for them leaves the factorisation (whose tensor maps hold
// the first matrix's address) untouched
static void swap_matrices(bdb_system* s)
{
    std::swap(s->M64.p, s->M64b.p);
    std::swap(s->M64.n, s->M64b.n);
    std::swap(s->M32.p, s->M32b.p);
    std::swap(s->M32.n, s->M32b.n);
}

// D.F and the random displacement of the current positions and noise X
static int displacements(bdb_system* s, bool want_rs)
{
    if (s->p.hydro == BDB_HYDRO_CHOLESKY) {
        phase_mark(s, P_MATVEC);
        int rc = stored_matvec(s, want_rs);
        phase_mark(s, P_MATVEC);
        return rc;
    }
    phase_mark(s, P_TEA);
    int rc = tea_run(s, want_rs);
    phase_mark(s, P_TEA);
    return rc;
}

// predictor, forces at r', D(r') F', and the averaged tensor's factor;
// with stop_on_overlap the rest is skipped when the forces at r' overlap
// (compute_hydro_IGT returns 1 there, diff_equation.c:325-329)
static int igt_predictor(bdb_system* s, const double* g1, bool stop_on_overlap, unsigned* flags)
{
    int rc;
    const bool chol = s->p.hydro == BDB_HYDRO_CHOLESKY;
    const size_t v3 = sizeof(double) * s->n3;
    if (!s->have_forces && ((rc = set_force_time(s, s->sim_time)) || (rc = forces_phase(s)))) return rc;
    // both force passes of the step act at its end time (diff_equation.c:314, 327)
    if ((rc = set_force_time(s, s->sim_time + s->p.dt))) return rc;
    // predictor
    if (chol) {
        if ((rc = ensure_matrix(s)) || (rc = ensure_matrix_b(s))) return rc;
        if ((rc = build_and_factor(s))) return rc;
        s->factor_valid = false;   // the stored matrix holds the corrector's factor after this step
        BDB_CUDA(cudaMemcpyAsync(s->dD_igt.p, s->dD.p, v3, cudaMemcpyDeviceToDevice, s->stream));
    }
    phase_mark(s, P_NOISE);
    if ((rc = noise_fill(s, g1))) return rc;
    phase_mark(s, P_NOISE);
    if ((rc = displacements(s, true))) return rc;
    BDB_CUDA(cudaMemcpyAsync(s->pos_igt.p, s->pos.p, sizeof(double4) * s->n, cudaMemcpyDeviceToDevice, s->stream));
    BDB_CUDA(cudaMemcpyAsync(s->Rf_igt.p, s->Rf.p, v3, cudaMemcpyDeviceToDevice, s->stream));
    phase_mark(s, P_UPDATE);
    if ((rc = update_positions(s, s->fs_igt.p))) return rc;
    phase_mark(s, P_UPDATE);
    // forces and D(r') F' at the predicted positions
    if ((rc = forces_phase(s))) return rc;
    bool ov = false;
    if ((rc = check_status(s, &ov))) return rc;
    if (ov) *flags |= 1;
    BDB_CUDA(cudaMemsetAsync(s->status.p, 0, sizeof(unsigned), s->stream));
    s->igt_ready = false;
    if (ov && stop_on_overlap) return BDB_OK;
    if (chol) {
        swap_matrices(s);
        phase_mark(s, P_BUILD);
        rc = tensor_build(s);
        phase_mark(s, P_BUILD);
        if (!rc) rc = displacements(s, false);
        swap_matrices(s);
        if (rc) return rc;
    } else if ((rc = displacements(s, false))) {
        return rc;
    }
    BDB_CUDA(cudaMemcpyAsync(s->Rf2_igt.p, s->Rf.p, v3, cudaMemcpyDeviceToDevice, s->stream));
    // averaged tensor and its factor
    if (chol) {
        const int nb = (s->n3 + 31) / 32;
        const dim3 grid(nb, nb), block(32, 8);
        if (s->p.precision == BDB_PREC_FP64)
            k_igt_average<double><<<grid, block, 0, s->stream>>>(s->n3, s->npad, s->M64.p, s->M64b.p, s->dD_igt.p);
        else
            k_igt_average<float><<<grid, block, 0, s->stream>>>(s->n3, s->npad, s->M32.p, s->M32b.p, s->dD_igt.p);
        BDB_CUDA(cudaGetLastError());
        BDB_CUDA(cudaMemcpyAsync(s->dD.p, s->dD_igt.p, v3, cudaMemcpyDeviceToDevice, s->stream));
        s->launches += 1;
        phase_mark(s, P_FACTOR);
        if ((rc = factor_run(s))) return rc;
        phase_mark(s, P_FACTOR);
    }
    s->igt_ready = true;
    return BDB_OK;
}

// corrector: fresh Gaussians, r <- r0 + ((Rf + Rf')/2 + L X2), forces
static int igt_corrector(bdb_system* s, const double* g2)
{
    int rc;
    BDB_CUDA(cudaMemcpyAsync(s->pos.p, s->pos_igt.p, sizeof(double4) * s->n, cudaMemcpyDeviceToDevice, s->stream));
    phase_mark(s, P_NOISE);
    if ((rc = noise_fill(s, g2))) return rc;
    phase_mark(s, P_NOISE);
    if ((rc = displacements(s, true))) return rc;
    phase_mark(s, P_UPDATE);
    k_igt_update<<<(s->n + 127) / 128, 128, 0, s->stream>>>(
        s->n, s->p.bc == 1, make_double3(s->p.box[0], s->p.box[1], s->p.box[2]),
        make_double3(s->inv_L[0], s->inv_L[1], s->inv_L[2]), s->pos_igt.p, s->Rf_igt.p, s->Rf2_igt.p, s->Rs.p,
        (s->p.flow && s->p.bc != 2) ? s->fs_igt.p : nullptr, s->pos.p);
    BDB_CUDA(cudaGetLastError());
    s->launches += 1;
    phase_mark(s, P_UPDATE);
    return forces_phase(s);
}

}  // namespace bdb

using namespace bdb;

static int igt_buffers(bdb_system* s)
{
    if (s->pos_igt.n < (size_t)s->n && s->pos_igt.alloc(s->n)) return BDB_ERR_NOMEM;
    for (DevBuf<double>* b : {&s->Rf_igt, &s->Rf2_igt, &s->dD_igt, &s->fs_igt})
        if (b->n < (size_t)s->n3 && b->alloc(s->n3)) return BDB_ERR_NOMEM;
    return BDB_OK;
}

static int igt_checks(bdb_system* s, const double* gauss)
{
    if (!s) return fail(BDB_ERR_ARG, "null system");
    if (s->p.noise == BDB_NOISE_HOST && !gauss) return fail(BDB_ERR_ARG, "host noise mode needs Gaussians");
    if (s->p.hydro == BDB_HYDRO_GEYER)
        return fail(BDB_ERR_UNSUPPORTED, "IGT steps need hydro none or cholesky (the averaged tensor is stored)");
    if (s->segs.size() > 1) return fail(BDB_ERR_UNSUPPORTED, "IGT steps take one system");
    return igt_buffers(s);
}

static int stage_gauss(bdb_system* s, const double* gauss, size_t count)
{
    if (!gauss) return BDB_OK;
    if (s->gbuf.n < count && s->gbuf.alloc(count)) return BDB_ERR_NOMEM;
    BDB_CUDA(cudaMemcpyAsync(s->gbuf.p, gauss, sizeof(double) * count, cudaMemcpyHostToDevice, s->stream));
    return BDB_OK;
}

extern "C" int bdb_step_igt(bdb_system* s, int K, const double* gauss)
{
    if (K < 0) return fail(BDB_ERR_ARG, "bad arguments");
    int rc0 = igt_checks(s, gauss);
    if (rc0) return rc0;
    phase_mark(s, P_STEP);
    if ((rc0 = stage_gauss(s, gauss, (size_t)K * 2 * s->n3))) return rc0;
    unsigned flags = 0;
    for (int k = 0; k < K; ++k) {
        BDB_CUDA(cudaMemsetAsync(s->status.p, 0, sizeof(unsigned), s->stream));
        const double* g1 = gauss ? s->gbuf.p + (size_t)k * 2 * s->n3 : nullptr;
        const double* g2 = gauss ? g1 + s->n3 : nullptr;
        int rc = igt_predictor(s, g1, false, &flags);
        if (!rc) rc = igt_corrector(s, g2);
        if (!rc) rc = after_step(s, s->p.dt);
        if (rc) return rc;
        bool ov = false;
        rc = check_status(s, &ov);
        if (rc) return rc;
        if (ov) flags |= 2;
    }
    phase_mark(s, P_STEP);
    return (int)flags;
}

// compute_hydro_IGT's first part (diff_equation.c:317-368): the predictor
// from the current positions and forces, the forces at r' and, unless they
// overlap, D(r') F' and the averaged factor for bdb_step_igt_corrector
extern "C" int bdb_step_igt_predictor(bdb_system* s, const double* gauss)
{
    int rc = igt_checks(s, gauss);
    if (rc) return rc;
    if ((rc = stage_gauss(s, gauss, s->n3))) return rc;
    BDB_CUDA(cudaMemsetAsync(s->status.p, 0, sizeof(unsigned), s->stream));
    unsigned flags = 0;
    if ((rc = igt_predictor(s, gauss ? s->gbuf.p : nullptr, true, &flags))) return rc;
    return flags ? 1 : 0;
}

// compute_hydro_IGT_second_phase (diff_equation.c:288-315), after
// bdb_step_igt_predictor or again after an overlap (comp_step_IGT_const,
// diff_comp.c:87-96): from the step's start positions, fresh Gaussians with
// the same averaged factor and deterministic displacement, then forces
extern "C" int bdb_step_igt_corrector(bdb_system* s, const double* gauss)
{
    int rc = igt_checks(s, gauss);
    if (rc) return rc;
    if (!s->igt_ready) return fail(BDB_ERR_ARG, "no IGT predictor to finish");
    if ((rc = stage_gauss(s, gauss, s->n3))) return rc;
    BDB_CUDA(cudaMemsetAsync(s->status.p, 0, sizeof(unsigned), s->stream));
    if ((rc = igt_corrector(s, gauss ? s->gbuf.p : nullptr))) return rc;
    bool ov = false;
    if ((rc = check_status(s, &ov))) return rc;
    return ov ? 1 : 0;
}
