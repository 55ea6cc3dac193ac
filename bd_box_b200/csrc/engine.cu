// The bdb_* C ABI (include/bdb200.h): system lifetime, host <-> device
// copies and the step driver that sequences the kernels of one
// Ermak-McCammon step exactly as compute_hydro_ermak (diff_equation.c:
// 216-286) orders the work: D.F from the forces at the start of the step,
// the random displacement, r += Rf + Rs with the periodic wrap, then the
// forces at the new positions (comp_step_ermak, diff_comp.c:152-179).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "bdb_common.cuh"

namespace bdb {

static thread_local std::string g_err;

void set_error(const std::string& msg) { g_err = msg; }

int fail(int code, const std::string& msg)
{
    g_err = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* what)
{
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? BDB_ERR_NOMEM : BDB_ERR_CUDA;
}

template <typename T>
int DevBuf<T>::alloc(size_t count)
{
    release();
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), count * sizeof(T));
    if (e != cudaSuccess) {
        p = nullptr;
        n = 0;
        cuda_fail(e, "cudaMalloc");
        return 1;
    }
    n = count;
    return 0;
}

template <typename T>
void DevBuf<T>::release()
{
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
}

template struct DevBuf<double>;
template struct DevBuf<float>;
template struct DevBuf<int>;
template struct DevBuf<unsigned>;
template struct DevBuf<unsigned long long>;
template struct DevBuf<unsigned char>;
template struct DevBuf<double2>;
template struct DevBuf<double4>;
template struct DevBuf<int4>;
template struct DevBuf<int2>;
template struct DevBuf<long long>;
template struct DevBuf<Segment>;
template struct DevBuf<TileJob>;

static const char* kPhaseNames[P_COUNT] = {"step",   "refresh", "build",    "factor",   "matvec",
                                           "tea",    "forces",  "noise",    "update",   "potrf",
                                           "trsm",   "syrk_col", "syrk_rest"};

void phase_mark_on(bdb_system* s, int ph, cudaStream_t stream)
{
    if (!s->profiling) return;
    auto& r = s->phases[ph];
    if (r.used == r.ev.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return;
        r.ev.push_back(e);
    }
    cudaEventRecord(r.ev[r.used++], stream);
}

void phase_mark(bdb_system* s, int ph) { phase_mark_on(s, ph, s->stream); }

int check_status(bdb_system* s, bool* overlap)
{
    unsigned st = 0;
    BDB_CUDA(cudaMemcpyAsync(&st, s->status.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s->stream));
    BDB_CUDA(cudaStreamSynchronize(s->stream));
    // a factorisation that met a non-positive pivot, gave up waiting or was
    // launched wrongly left no usable factor: the next step rebuilds it
    if (st & (ST_NOT_SPD | ST_TIMEOUT | ST_LAUNCH)) s->factor_valid = false;
    if (st & ST_BOND) return fail(BDB_ERR_BOND, "Overstretched bond (bond.c:73-78)");
    // a kernel that did nothing or gave up leaves the rest of the
    // factorisation working on partial data, whose pivots may then fail:
    // report the cause first
    if (st & ST_LAUNCH) return fail(BDB_ERR_CUDA, "a kernel was launched with the wrong shape");
    if (st & ST_TIMEOUT) return fail(BDB_ERR_TIMEOUT, "device wait timed out");
    if (st & ST_NOT_SPD) return fail(BDB_ERR_NOT_SPD, "Cholesky decomposition error: non-positive pivot");
    if (overlap) *overlap = (st & ST_OVERLAP) != 0;
    return BDB_OK;
}

int ensure_matrix(bdb_system* s)
{
    const size_t nn = (size_t)s->npad * s->npad;
    if (s->p.precision == BDB_PREC_FP64) {
        if (s->M64.p) return BDB_OK;
        if (s->M64.alloc(nn)) return BDB_ERR_NOMEM;
        BDB_CUDA(dzero(s, s->M64.p, nn * sizeof(double)));
        std::vector<double> one(1, 1.0);
        for (int r = s->n3; r < s->npad; ++r)
            BDB_CUDA(h2d(s, s->M64.p + (size_t)r * s->npad + r, one.data(), sizeof(double)));
    } else {
        if (s->M32.p) return BDB_OK;
        if (s->M32.alloc(nn)) return BDB_ERR_NOMEM;
        BDB_CUDA(dzero(s, s->M32.p, nn * sizeof(float)));
        float one = 1.0f;
        for (int r = s->n3; r < s->npad; ++r)
            BDB_CUDA(h2d(s, s->M32.p + (size_t)r * s->npad + r, &one, sizeof(float)));
    }
    return BDB_OK;
}

int build_and_factor(bdb_system* s)
{
    phase_mark(s, P_BUILD);
    int rc = tensor_build(s);
    if (rc) return rc;
    phase_mark(s, P_BUILD);
    phase_mark(s, P_FACTOR);
    rc = factor_run(s);
    if (rc) return rc;
    phase_mark(s, P_FACTOR);
    return BDB_OK;
}

// One refresh (tensor build + factorisation) with the chain reserve c, timed
// the way every refresh after the first runs: captured into a CUDA graph
// (node priorities kept) and replayed, the faster of two replays after a
// warm one. Eagerly, one run, where refreshes run eagerly (refresh graphs
// switched off, or phases being profiled).
static int tune_time(bdb_system* s, int c, cudaEvent_t e0, cudaEvent_t e1, float* ms_out)
{
    s->chain_sms = c;
    *ms_out = 1e30f;
    if (s->profiling || !s->graph_refresh) {
        BDB_CUDA(cudaEventRecord(e0, s->stream));
        const int rc = build_and_factor(s);
        if (rc) return rc;
        BDB_CUDA(cudaEventRecord(e1, s->stream));
        BDB_CUDA(cudaEventSynchronize(e1));
        BDB_CUDA(cudaEventElapsedTime(ms_out, e0, e1));
        return BDB_OK;
    }
    const long long before = s->launches;
    BDB_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    int rc = build_and_factor(s);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    const long long per = s->launches - before;
    s->launches = before;
    if (rc || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return rc ? rc : cuda_fail(e, "cudaStreamEndCapture");
    }
    cudaGraphExec_t x = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&x, g, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) return cuda_fail(ei, "cudaGraphInstantiate");
    cudaError_t err = cudaSuccess;
    for (int r = 0; r < 3 && err == cudaSuccess; ++r) {
        err = cudaEventRecord(e0, s->stream);
        if (err == cudaSuccess) err = cudaGraphLaunch(x, s->stream);
        if (err == cudaSuccess) err = cudaEventRecord(e1, s->stream);
        if (err == cudaSuccess) err = cudaEventSynchronize(e1);
        float ms = 0.0f;
        if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
        if (err == cudaSuccess && r > 0) *ms_out = std::min(*ms_out, ms);
        s->launches += per;
    }
    cudaGraphExecDestroy(x);
    return err == cudaSuccess ? BDB_OK : cuda_fail(err, "factor tuning replay");
}

// Autotuning of the mixed Cholesky's split of the GPU between its panel
// chain and its bulk updates (chol_tc.cu). One eager refresh first (it
// allocates and encodes what the kernels use), then each candidate reserve
// is timed as a replayed refresh graph (tune_time); the last one leaves the
// factor of the current positions in place (every reserve gives the same
// bits).
static int factor_tune(bdb_system* s)
{
    const int cands[7] = {16, 24, 32, 40, 48, 56, 64};
    int rc = build_and_factor(s);
    if (rc) return rc;
    float best_ms = 1e30f;
    int best = s->chain_sms;
    cudaEvent_t e0, e1;
    BDB_CUDA(cudaEventCreate(&e0));
    BDB_CUDA(cudaEventCreate(&e1));
    for (int c : cands) {
        if (c >= s->sm_count) break;
        float ms = 0.0f;
        if ((rc = tune_time(s, c, e0, e1, &ms))) break;
        if (ms < best_ms) {
            best_ms = ms;
            best = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    s->chain_sms = best;
    s->factor_tuned = true;
    return rc;
}

// D (and its factor) at the current positions. After one eager refresh
// (which allocates and encodes everything the kernels use), the mixed path
// replays the ~400 launches of a refresh -- both streams of the look-ahead
// factorisation included -- from a captured CUDA graph.
static int refresh_factor(bdb_system* s)
{
    int rc = ensure_matrix(s);
    if (rc) return rc;
    phase_mark(s, P_REFRESH);
    const bool graph = s->graph_refresh && !s->profiling && s->p.precision == BDB_PREC_MIXED && s->eager_refreshes > 0;
    if (graph) {
        if (!s->refresh_graph) {
            const long long before = s->launches;
            BDB_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
            rc = build_and_factor(s);
            cudaGraph_t g = nullptr;
            const cudaError_t e = cudaStreamEndCapture(s->stream, &g);
            if (rc || e != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                return rc ? rc : cuda_fail(e, "cudaStreamEndCapture");
            }
            // the nodes keep the priorities of the streams they were captured
            // from (chain high, side middle, bulk low); without this flag a
            // replay runs every node at the priority of the launching stream
            const cudaError_t ei =
                cudaGraphInstantiate(&s->refresh_graph, g, cudaGraphInstantiateFlagUseNodePriority);
            cudaGraphDestroy(g);
            if (ei != cudaSuccess) {
                s->refresh_graph = nullptr;
                return cuda_fail(ei, "cudaGraphInstantiate");
            }
            s->refresh_launches = s->launches - before;
            s->launches = before;
        }
        BDB_CUDA(cudaGraphLaunch(s->refresh_graph, s->stream));
        s->launches += s->refresh_launches;
    } else {
        if (s->autotune && !s->factor_tuned && s->p.precision == BDB_PREC_MIXED) {
            rc = factor_tune(s);
        } else {
            rc = build_and_factor(s);
        }
        if (rc) return rc;
        s->eager_refreshes++;
    }
    phase_mark(s, P_REFRESH);
    s->factor_valid = true;
    s->steps_since_refresh = 0;
    return BDB_OK;
}

int forces_phase(bdb_system* s)
{
    phase_mark(s, P_FORCES);
    int rc = forces_run(s, false, false);
    phase_mark(s, P_FORCES);
    return rc;
}

// noise, D.F and the random displacement, the update and the new forces:
// the part of a step that is the same every step while no refresh is due
static int step_body(bdb_system* s, const double* dev_gauss)
{
    int rc;
    // the mixed Cholesky step with device noise and no flow: the product
    // draws the noise and its finisher moves the beads (two launches fewer,
    // no noise vector in HBM; the same bits as the separate kernels)
    if (s->fuse_step && !dev_gauss && s->p.hydro == BDB_HYDRO_CHOLESKY && s->p.precision != BDB_PREC_FP64 &&
        !(s->p.flow && s->p.bc != 2)) {
        phase_mark(s, P_MATVEC);
        if ((rc = stored_matvec_step(s))) return rc;
        phase_mark(s, P_MATVEC);
        return forces_phase(s);
    }
    phase_mark(s, P_NOISE);
    if ((rc = noise_fill(s, dev_gauss))) return rc;
    phase_mark(s, P_NOISE);
    if (s->p.hydro == BDB_HYDRO_CHOLESKY) {
        phase_mark(s, P_MATVEC);
        if ((rc = stored_matvec(s, true))) return rc;
        phase_mark(s, P_MATVEC);
    } else {
        phase_mark(s, P_TEA);
        if ((rc = tea_run(s, true))) return rc;
        phase_mark(s, P_TEA);
    }
    phase_mark(s, P_UPDATE);
    if ((rc = update_positions(s))) return rc;
    phase_mark(s, P_UPDATE);
    return forces_phase(s);
}

void drop_graph(bdb_system* s)
{
    if (s->step_graph) cudaGraphExecDestroy(s->step_graph);
    s->step_graph = nullptr;
    if (s->step_graph_host) cudaGraphExecDestroy(s->step_graph_host);
    s->step_graph_host = nullptr;
    s->step_graph_host_src = nullptr;
    if (s->refresh_graph) cudaGraphExecDestroy(s->refresh_graph);
    s->refresh_graph = nullptr;
}

// step_body captured once as a CUDA graph and replayed (not while
// profiling, whose event records would be frozen into the graph). Device
// noise has one graph; caller Gaussians have another, which holds the device
// address of the Gaussians it was captured with and is captured again when a
// step's Gaussians sit elsewhere (a K-step call walks its staging buffer).
static int step_body_graph(bdb_system* s, const double* dev_gauss)
{
    cudaGraphExec_t* exec = dev_gauss ? &s->step_graph_host : &s->step_graph;
    long long* nl = dev_gauss ? &s->graph_launches_host : &s->graph_launches;
    if (dev_gauss && *exec && s->step_graph_host_src != dev_gauss) {
        cudaGraphExecDestroy(*exec);
        *exec = nullptr;
    }
    if (!*exec) {
        const long long before = s->launches;
        BDB_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = step_body(s, dev_gauss);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(s->stream, &g);
        if (rc || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return rc ? rc : cuda_fail(e, "cudaStreamEndCapture");
        }
        const cudaError_t ei = cudaGraphInstantiate(exec, g, cudaGraphInstantiateFlagUseNodePriority);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            *exec = nullptr;
            return cuda_fail(ei, "cudaGraphInstantiate");
        }
        *nl = s->launches - before;
        s->launches = before;
        if (dev_gauss) s->step_graph_host_src = dev_gauss;
    }
    BDB_CUDA(cudaGraphLaunch(*exec, s->stream));
    s->launches += *nl;
    return BDB_OK;
}

static int one_step(bdb_system* s, const double* dev_gauss)
{
    int rc;
    if (!s->have_forces) {
        if ((rc = set_force_time(s, s->sim_time)) || (rc = forces_phase(s))) return rc;
    }
    if (s->p.hydro == BDB_HYDRO_CHOLESKY) {
        if (!s->factor_valid || s->steps_since_refresh >= std::max(1, s->p.refresh)) {
            rc = refresh_factor(s);
            if (rc) return rc;
        }
        s->steps_since_refresh++;
    }
    // the forces after the step act at the step's end time (diff_comp.c:161)
    if ((rc = set_force_time(s, s->sim_time + s->p.dt))) return rc;
    // the first step runs eagerly, so that buffers allocated on first use
    // exist (at fixed addresses) before a graph captures them
    if (s->graphs && !s->profiling && s->eager_steps > 0) return step_body_graph(s, dev_gauss);
    s->eager_steps++;
    return step_body(s, dev_gauss);
}

int engine_step(bdb_system* s) { return one_step(s, nullptr); }

}  // namespace bdb

using namespace bdb;

extern "C" {

const char* bdb_version(void) { return "bdb200 1.0 (sm_100a)"; }

const char* bdb_last_error(void) { return g_err.c_str(); }

}  // extern "C"

// One system of nseg independent segments (replicas) of counts[g] beads,
// stored back to back; nseg = 1 is a single system.
static int create_system(bdb_system** out, const bdb_params* p, int nseg, const int* counts, const double* coord,
                         const double* Q, const double* LJ)
{
    if (!out || !p || !coord || !Q || !LJ || !counts) return fail(BDB_ERR_ARG, "null argument");
    if (nseg < 1) return fail(BDB_ERR_ARG, "need at least one segment");
    long long total = 0;
    for (int g = 0; g < nseg; ++g) {
        if (counts[g] < 2) return fail(BDB_ERR_ARG, "every segment needs at least two beads");
        total += counts[g];
    }
    if (total != p->n) return fail(BDB_ERR_ARG, "params.n must equal the sum of the segment bead counts");
    if (nseg > 1 && p->hydro == BDB_HYDRO_CHOLESKY)
        return fail(BDB_ERR_UNSUPPORTED, "batched segments need hydro none or geyer (the stored tensor holds one system)");
    if (p->n <= 1) return fail(BDB_ERR_ARG, "need at least two beads");
    if (p->hydro < 0 || p->hydro > 2) return fail(BDB_ERR_ARG, "hydro must be none, cholesky or geyer");
    if (p->bc < 0 || p->bc > 2) return fail(BDB_ERR_ARG, "bc must be none, periodic or sphere");
    if (p->bc == 1 && (p->box[0] <= 0 || p->box[1] <= 0 || p->box[2] <= 0))
        return fail(BDB_ERR_ARG, "Wrong box size");
    if (p->bc == 2) {
        // iscorrect (trans.c:130-145): every bead inside the sphere
        const double sr = p->sphere_radius * p->sphere_radius;
        for (int i = 0; i < p->n; ++i) {
            const double* c = coord + 4 * i;
            if (c[0] * c[0] + c[1] * c[1] + c[2] * c[2] > sr) return fail(BDB_ERR_ARG, "Wrong correction");
        }
    }
    if (p->e_ext && (p->e_type < 0 || p->e_type > 2 || p->e_dir1 < 0 || p->e_dir1 > 2 || p->e_dir2 < 0 || p->e_dir2 > 2))
        return fail(BDB_ERR_ARG, "E_type must be DC, AC or RF and E_dir1/E_dir2 x, y or z");
    if (p->sboundary && p->sboundary_n < 0) return fail(BDB_ERR_ARG, "sboundary_n must be >= 0");
    if (p->ewald && (p->ewald_real < 0 || p->ewald_real > 5)) return fail(BDB_ERR_ARG, "ewald_real wrong value, only 0..5");
    if (p->ewald && p->ewald_method != BDB_EWALD_BEENAKKER && p->ewald_method != BDB_EWALD_SMITH)
        return fail(BDB_ERR_ARG, "ewald_method must be beenakker or smith");
    if (p->ewald && !(p->box[0] == p->box[1] && p->box[1] == p->box[2]))
        return fail(BDB_ERR_ARG, "In Ewald box must be cube");
    if (p->visc == 0.0 || p->vfactor == 0.0) return fail(BDB_ERR_ARG, "Wrong value for visc/vfactor");
    for (int i = 0; i < p->n; ++i)
        if (!(coord[4 * i + 3] > 0.0)) return fail(BDB_ERR_ARG, "Wrong atom radii");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(BDB_ERR_CUDA, "no CUDA device");
    bdb_system* s = new bdb_system();
    cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, dev);
    s->p = *p;
    if (s->p.refresh < 1) s->p.refresh = 1;
    s->n = p->n;
    s->n3 = 3 * p->n;
    s->npad = (s->n3 + 127) / 128 * 128;
    for (int k = 0; k < 3; ++k) s->inv_L[k] = p->bc == 1 ? 1 / p->box[k] : 0.0;
    s->preDii = BDB_KB_1_6PI * p->T / (p->visc * p->vfactor);
    s->preDij = BDB_KB_1_8PI * p->T / (p->visc * p->vfactor);
    // BDB_NO_FUSE (diagnostics): separate noise and update kernels on the
    // Cholesky path, to compare against the fused step
    s->fuse_step = getenv("BDB_NO_FUSE") == nullptr;
    // the Cholesky's chain reserve, measured at 3N = 12288 on B200: the
    // mixed path's bulk update is fast enough to spare 32 SMs; the FP64
    // path's DMMA update is the slower side and keeps all but 16
    s->chain_sms = p->precision == BDB_PREC_FP64 ? 16 : 32;
    int rc = BDB_OK;
#define TRY(x)                       \
    do {                             \
        if ((rc = (x)) != BDB_OK) {  \
            bdb_destroy(s);          \
            return rc;               \
        }                            \
    } while (0)
#define TRYA(b, cnt)                             \
    do {                                         \
        if ((b).alloc(cnt)) {                    \
            bdb_destroy(s);                      \
            return BDB_ERR_NOMEM;                \
        }                                        \
    } while (0)
    // stream priorities: the main stream (which runs the Cholesky's panel
    // chain) first, then the chain's side work, then its bulk updates, so
    // that a chain kernel's CTAs are dispatched ahead of queued bulk CTAs
    int prio_low = 0, prio_high = 0;
    cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
    if (cudaStreamCreateWithPriority(&s->stream, cudaStreamNonBlocking, prio_high) != cudaSuccess ||
        cudaStreamCreateWithPriority(&s->stream2, cudaStreamNonBlocking, prio_low) != cudaSuccess ||
        cudaStreamCreateWithPriority(&s->stream3, cudaStreamNonBlocking, (prio_low + prio_high) / 2) != cudaSuccess) {
        bdb_destroy(s);
        return fail(BDB_ERR_CUDA, "stream creation failed");
    }
    for (auto& e : s->la_ev)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            bdb_destroy(s);
            return fail(BDB_ERR_CUDA, "event creation failed");
        }
    {
        int b = 0;
        for (int g = 0; g < nseg; ++g) {
            s->segs.push_back(Segment{b, counts[g], 0});
            b += counts[g];
        }
    }
    TRYA(s->d_segs, nseg);
    TRYA(s->d_bead_seg, s->n);
    TRYA(s->pos, s->n);
    TRYA(s->pos_save, s->n);
    TRYA(s->Q, s->n);
    TRYA(s->LJ, s->n);
    TRYA(s->Rf, s->n3);
    TRYA(s->Rs, s->n3);
    TRYA(s->X, s->n3);
    TRYA(s->dD, s->npad);
    TRYA(s->scal, 64 + 4 * (size_t)nseg + 64);
    TRYA(s->ctr, 3);
    BDB_CUDA(h2d(s, s->d_segs.p, s->segs.data(), sizeof(Segment) * nseg));
    {
        std::vector<int> bs(s->n);
        for (int g = 0; g < nseg; ++g)
            for (int i = 0; i < counts[g]; ++i) bs[s->segs[g].begin + i] = g;
        BDB_CUDA(h2d(s, s->d_bead_seg.p, bs.data(), sizeof(int) * s->n));
    }
    BDB_CUDA(h2d(s, s->pos.p, coord, sizeof(double) * 4 * s->n));
    BDB_CUDA(h2d(s, s->Q.p, Q, sizeof(double) * s->n));
    BDB_CUDA(h2d(s, s->LJ.p, LJ, sizeof(double) * 2 * s->n));
    BDB_CUDA(dzero(s, s->scal.p, sizeof(double) * s->scal.n));
    BDB_CUDA(dzero(s, s->ctr.p, sizeof(unsigned long long) * 3));
    BDB_CUDA(dzero(s, s->Rf.p, sizeof(double) * s->n3));
    BDB_CUDA(dzero(s, s->Rs.p, sizeof(double) * s->n3));
    BDB_CUDA(dzero(s, s->X.p, sizeof(double) * s->n3));
    {
        std::vector<double> dd(s->npad, 1.0);
        BDB_CUDA(h2d(s, s->dD.p, dd.data(), sizeof(double) * s->npad));
    }
    TRY(forces_setup(s));
    TRY(bonded_setup(s));
    BDB_CUDA(dzero(s, s->status.p, sizeof(unsigned) * 4));
#undef TRY
#undef TRYA
    *out = s;
    return BDB_OK;
}

extern "C" {

int bdb_create(bdb_system** out, const bdb_params* p, const double* coord, const double* Q, const double* LJ)
{
    if (!p) return fail(BDB_ERR_ARG, "null argument");
    return create_system(out, p, 1, &p->n, coord, Q, LJ);
}

int bdb_create_batch(bdb_system** out, const bdb_params* p, int nseg, const int* counts, const double* coord,
                     const double* Q, const double* LJ)
{
    return create_system(out, p, nseg, counts, coord, Q, LJ);
}

int bdb_destroy(bdb_system* s)
{
    if (!s) return BDB_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto& r : s->phases)
        for (auto e : r.ev) cudaEventDestroy(e);
    if (s->stream2) cudaStreamSynchronize(s->stream2);
    if (s->stream3) cudaStreamSynchronize(s->stream3);
    for (auto e : s->la_ev)
        if (e) cudaEventDestroy(e);
    drop_graph(s);
    frames_release(s);
    if (s->stream3) cudaStreamDestroy(s->stream3);
    if (s->stream2) cudaStreamDestroy(s->stream2);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return BDB_OK;
}

int bdb_set_bonded(bdb_system* s, int n_bond, const int* bond_pairs, const double* bond_parms, int n_angle,
                   const int* angle_pairs, const double* angle_parms, int n_angle_cos, const int* angle_cos_pairs,
                   const double* angle_cos_parms, int n_dihe, const int* dihe_pairs, const double* dihe_parms,
                   int n_dihe_angle, const int* dihe_angle_pairs, const double* dihe_angle_parms)
{
    if (!s) return fail(BDB_ERR_ARG, "null system");
    struct T {
        int cnt, members, npar;
        const int* idx;
        const double* par;
        DevBuf<int>* di;
        DevBuf<double>* dp;
        int* store;
    } terms[5] = {
        {n_bond, 2, 3, bond_pairs, bond_parms, &s->bond_pairs, &s->bond_parms, &s->n_bond},
        {n_angle, 3, 2, angle_pairs, angle_parms, &s->angle_pairs, &s->angle_parms, &s->n_angle},
        {n_angle_cos, 3, 2, angle_cos_pairs, angle_cos_parms, &s->angle_cos_pairs, &s->angle_cos_parms, &s->n_angle_cos},
        {n_dihe, 4, 2, dihe_pairs, dihe_parms, &s->dihe_pairs, &s->dihe_parms, &s->n_dihe},
        {n_dihe_angle, 4, 2, dihe_angle_pairs, dihe_angle_parms, &s->dihe_angle_pairs, &s->dihe_angle_parms,
         &s->n_dihe_angle},
    };
    std::vector<int> seg_of(s->n);
    for (size_t g = 0; g < s->segs.size(); ++g)
        for (int i = 0; i < s->segs[g].count; ++i) seg_of[s->segs[g].begin + i] = (int)g;
    for (auto& t : terms) {
        if (t.cnt < 0 || (t.cnt && (!t.idx || !t.par))) return fail(BDB_ERR_ARG, "bonded term arrays");
        for (int k = 0; k < t.cnt * t.members; ++k)
            if (t.idx[k] < 0 || t.idx[k] >= s->n) return fail(BDB_ERR_ARG, "bonded term references a missing bead");
        for (int k = 0; k < t.cnt; ++k)
            for (int m = 1; m < t.members; ++m)
                if (seg_of[t.idx[k * t.members + m]] != seg_of[t.idx[k * t.members]])
                    return fail(BDB_ERR_ARG, "bonded term joins beads of two segments");
    }
    for (auto& t : terms) {
        *t.store = t.cnt;
        if (t.di->alloc(std::max(1, t.cnt * t.members)) || t.dp->alloc(std::max(1, t.cnt * t.npar)))
            return BDB_ERR_NOMEM;
        if (t.cnt) {
            BDB_CUDA(h2d(s, t.di->p, t.idx, sizeof(int) * t.cnt * t.members));
            BDB_CUDA(h2d(s, t.dp->p, t.par, sizeof(double) * t.cnt * t.npar));
        }
    }
    s->have_forces = false;
    drop_graph(s);
    return bonded_setup(s);
}

int bdb_set_coord(bdb_system* s, const double* coord)
{
    if (!s || !coord) return fail(BDB_ERR_ARG, "null argument");
    BDB_CUDA(cudaMemcpyAsync(s->pos.p, coord, sizeof(double) * 4 * s->n, cudaMemcpyHostToDevice, s->stream));
    BDB_CUDA(cudaMemsetAsync(s->cells_built.p, 0, sizeof(int) * s->segs.size(), s->stream));
    s->have_forces = false;
    s->factor_valid = false;
    s->igt_ready = false;   // a pending IGT predictor belongs to the old positions
    return BDB_OK;
}

int bdb_get_coord(bdb_system* s, double* coord)
{
    if (!s || !coord) return fail(BDB_ERR_ARG, "null argument");
    BDB_CUDA(cudaMemcpyAsync(coord, s->pos.p, sizeof(double) * 4 * s->n, cudaMemcpyDeviceToHost, s->stream));
    BDB_CUDA(cudaStreamSynchronize(s->stream));
    return BDB_OK;
}

int bdb_save_state(bdb_system* s)
{
    if (!s) return fail(BDB_ERR_ARG, "null system");
    BDB_CUDA(cudaMemcpyAsync(s->pos_save.p, s->pos.p, sizeof(double4) * s->n, cudaMemcpyDeviceToDevice, s->stream));
    BDB_CUDA(cudaMemcpyAsync(s->F_save.p, s->F.p, sizeof(double) * s->n3, cudaMemcpyDeviceToDevice, s->stream));
    s->saved_step_count = s->step_count;
    s->saved_sim_time = s->sim_time;
    return BDB_OK;
}

int bdb_load_state(bdb_system* s)
{
    if (!s) return fail(BDB_ERR_ARG, "null system");
    BDB_CUDA(cudaMemcpyAsync(s->pos.p, s->pos_save.p, sizeof(double4) * s->n, cudaMemcpyDeviceToDevice, s->stream));
    BDB_CUDA(cudaMemcpyAsync(s->F.p, s->F_save.p, sizeof(double) * s->n3, cudaMemcpyDeviceToDevice, s->stream));
    BDB_CUDA(cudaMemsetAsync(s->cells_built.p, 0, sizeof(int) * s->segs.size(), s->stream));
    s->have_forces = true;
    s->step_count = s->saved_step_count;
    s->sim_time = s->saved_sim_time;
    s->igt_ready = false;   // a pending IGT predictor belongs to the discarded move
    frames_rewind(s, s->step_count);
    return BDB_OK;
}

int bdb_compute_forces(bdb_system* s, double* F, double* E, long long* counts)
{
    if (!s) return fail(BDB_ERR_ARG, "null system");
    BDB_CUDA(cudaMemsetAsync(s->status.p, 0, sizeof(unsigned), s->stream));
    int rc = set_force_time(s, s->sim_time);
    if (!rc) rc = forces_run(s, E != nullptr, counts != nullptr);
    if (rc) return rc;
    if (F) BDB_CUDA(cudaMemcpyAsync(F, s->F.p, sizeof(double) * s->n3, cudaMemcpyDeviceToHost, s->stream));
    if (E) BDB_CUDA(cudaMemcpyAsync(E, s->scal.p + 16, sizeof(double) * (BDB_E_LAST + 1), cudaMemcpyDeviceToHost,
                                    s->stream));
    unsigned long long c[2] = {0, 0};
    if (counts) BDB_CUDA(cudaMemcpyAsync(c, s->counts.p, sizeof(c), cudaMemcpyDeviceToHost, s->stream));
    bool ov = false;
    rc = check_status(s, &ov);
    if (rc) return rc;
    if (counts) {
        counts[0] = (long long)c[0];
        counts[1] = (long long)c[1];
    }
    return ov ? 1 : 0;
}

int bdb_compute_D(bdb_system* s, double* D)
{
    if (!s || !D) return fail(BDB_ERR_ARG, "null argument");
    if (s->segs.size() > 1) return fail(BDB_ERR_UNSUPPORTED, "the full tensor of a batch is not formed (segments are independent)");
    const int n3 = s->n3;
    if (s->p.hydro == BDB_HYDRO_NONE) {
        // compute_D does nothing without hydrodynamics; the tensor is diag_D
        // (diff_tensor.c:477, main_loop.c:161-175)
        std::vector<double4> pos(s->n);
        BDB_CUDA(d2h(s, pos.data(), s->pos.p, sizeof(double4) * s->n));
        memset(D, 0, sizeof(double) * (size_t)n3 * n3);
        for (int r = 0; r < n3; ++r) D[(size_t)r * n3 + r] = s->preDii / pos[r / 3].w;
        return BDB_OK;
    }
    int rc = ensure_matrix(s);
    if (rc) return rc;
    rc = tensor_build(s);
    if (rc) return rc;
    s->factor_valid = false;
    if (s->p.precision == BDB_PREC_FP64) {
        BDB_CUDA(cudaMemcpy2DAsync(D, sizeof(double) * n3, s->M64.p, sizeof(double) * s->npad, sizeof(double) * n3, n3,
                                   cudaMemcpyDeviceToHost, s->stream));
        BDB_CUDA(cudaStreamSynchronize(s->stream));
    } else {
        std::vector<float> tmp((size_t)n3 * n3);
        BDB_CUDA(cudaMemcpy2DAsync(tmp.data(), sizeof(float) * n3, s->M32.p, sizeof(float) * s->npad, sizeof(float) * n3,
                                   n3, cudaMemcpyDeviceToHost, s->stream));
        BDB_CUDA(cudaStreamSynchronize(s->stream));
        for (size_t k = 0; k < tmp.size(); ++k) D[k] = tmp[k];
    }
    // the diagonal of D lives in dD (the matrix diagonal is shared with L)
    std::vector<double> dd(n3);
    BDB_CUDA(d2h(s, dd.data(), s->dD.p, sizeof(double) * n3));
    for (int r = 0; r < n3; ++r) D[(size_t)r * n3 + r] = dd[r];
    return BDB_OK;
}

int bdb_compute_Dij(bdb_system* s, int i, int j, double* tD)
{
    if (!s || !tD || i < 0 || j < 0 || i >= s->n || j >= s->n) return fail(BDB_ERR_ARG, "bad tile index");
    if (s->segs.size() > 1) {
        // beads of different segments do not interact
        auto seg = [&](int b) {
            int g = 0;
            while (g + 1 < (int)s->segs.size() && s->segs[g + 1].begin <= b) ++g;
            return g;
        };
        if (seg(i) != seg(j)) {
            for (int k = 0; k < 9; ++k) tD[k] = 0.0;
            return BDB_OK;
        }
    }
    return tensor_tile_host(s, i, j, tD);
}

int bdb_compute_Rf(bdb_system* s, double* Rf)
{
    if (!s || !Rf) return fail(BDB_ERR_ARG, "null argument");
    int rc;
    if (!s->have_forces && ((rc = set_force_time(s, s->sim_time)) || (rc = forces_run(s, false, false)))) return rc;
    if (s->p.hydro == BDB_HYDRO_CHOLESKY) {
        if (!s->factor_valid && (rc = refresh_factor(s))) return rc;
        rc = stored_matvec(s, false);
    } else {
        rc = tea_run(s, false);
    }
    if (rc) return rc;
    BDB_CUDA(cudaMemcpyAsync(Rf, s->Rf.p, sizeof(double) * s->n3, cudaMemcpyDeviceToHost, s->stream));
    return check_status(s, nullptr);
}

int bdb_compute_r(bdb_system* s, const double* gauss, double* Rs)
{
    if (!s || !Rs) return fail(BDB_ERR_ARG, "null argument");
    int rc;
    BDB_CUDA(cudaMemsetAsync(s->status.p, 0, sizeof(unsigned), s->stream));
    if (!s->have_forces && ((rc = set_force_time(s, s->sim_time)) || (rc = forces_run(s, false, false)))) return rc;
    double* dg = nullptr;
    if (gauss) {
        dg = s->work.p;
        BDB_CUDA(cudaMemcpyAsync(dg, gauss, sizeof(double) * s->n3, cudaMemcpyHostToDevice, s->stream));
    }
    if ((rc = noise_fill(s, dg))) return rc;
    if (s->p.hydro == BDB_HYDRO_CHOLESKY) {
        if (!s->factor_valid && (rc = refresh_factor(s))) return rc;
        rc = stored_matvec(s, true);
    } else {
        rc = tea_run(s, true);
    }
    if (rc) return rc;
    BDB_CUDA(cudaMemcpyAsync(Rs, s->Rs.p, sizeof(double) * s->n3, cudaMemcpyDeviceToHost, s->stream));
    return check_status(s, nullptr);
}

int bdb_step(bdb_system* s, int K, const double* gauss)
{
    if (!s || K < 0) return fail(BDB_ERR_ARG, "bad arguments");
    if (s->p.noise == BDB_NOISE_HOST && !gauss) return fail(BDB_ERR_ARG, "host noise mode needs Gaussians");
    phase_mark(s, P_STEP);
    if (gauss) {
        const size_t need = (size_t)K * s->n3;
        if (s->gbuf.n < need && s->gbuf.alloc(need)) return BDB_ERR_NOMEM;
        BDB_CUDA(cudaMemcpyAsync(s->gbuf.p, gauss, sizeof(double) * need, cudaMemcpyHostToDevice, s->stream));
    }
    BDB_CUDA(cudaMemsetAsync(s->status.p, 0, sizeof(unsigned), s->stream));
    const bool replay = s->graphs && !s->profiling;
    for (int k = 0; k < K; ++k) {
        const double* g = gauss ? s->gbuf.p + (size_t)k * s->n3 : nullptr;
        if (g && k > 0 && replay) {
            // the step graph reads the first slot (already consumed)
            BDB_CUDA(cudaMemcpyAsync(s->gbuf.p, g, sizeof(double) * s->n3, cudaMemcpyDeviceToDevice, s->stream));
            g = s->gbuf.p;
        }
        int rc = one_step(s, g);
        if (!rc) rc = after_step(s, s->p.dt);
        if (rc) return rc;
    }
    phase_mark(s, P_STEP);
    bool ov = false;
    int rc = check_status(s, &ov);
    if (rc) return rc;
    return ov ? 1 : 0;
}

int bdb_refresh(bdb_system* s, int count)
{
    if (!s || count < 0) return fail(BDB_ERR_ARG, "bad arguments");
    if (s->p.hydro != BDB_HYDRO_CHOLESKY) return fail(BDB_ERR_UNSUPPORTED, "no stored tensor: hydro is not cholesky");
    BDB_CUDA(cudaMemsetAsync(s->status.p, 0, sizeof(unsigned), s->stream));
    for (int k = 0; k < count; ++k) {
        const int rc = refresh_factor(s);
        if (rc) return rc;
    }
    return check_status(s, nullptr);
}

int bdb_autotune(bdb_system* s, int enable)
{
    if (!s) return fail(BDB_ERR_ARG, "null system");
    s->autotune = enable != 0;
    return BDB_OK;
}

int bdb_get_tuning(bdb_system* s, int* tea_tile, int* mv_warps_per_sm)
{
    if (!s || !tea_tile || !mv_warps_per_sm) return fail(BDB_ERR_ARG, "null argument");
    *tea_tile = s->tea_tile;
    *mv_warps_per_sm = s->mv_warps;
    return BDB_OK;
}

int bdb_set_tuning(bdb_system* s, int tea_tile, int mv_warps_per_sm)
{
    if (!s) return fail(BDB_ERR_ARG, "null system");
    if (tea_tile != 0 && tea_tile != 16 && tea_tile != 32) return fail(BDB_ERR_ARG, "TEA tile must be 16 or 32");
    if (mv_warps_per_sm < 0 || mv_warps_per_sm > 64) return fail(BDB_ERR_ARG, "matvec warps per SM out of range");
    if (tea_tile && tea_tile != s->tea_tile) {
        s->tea_tile = tea_tile;
        s->tea_meta.release();   // the work list is rebuilt for the new tile at the next TEA call
        drop_graph(s);
    }
    if (mv_warps_per_sm && mv_warps_per_sm != s->mv_warps) {
        s->mv_warps = mv_warps_per_sm;
        drop_graph(s);
    }
    s->tea_tuned = s->mv_tuned = true;   // pinned values are not re-tuned
    return BDB_OK;
}

int bdb_set_wait_limit(bdb_system* s, long long tries)
{
    if (!s) return fail(BDB_ERR_ARG, "null system");
    if (tries > 0xffffffffll) return fail(BDB_ERR_ARG, "wait limit too large");
    s->wait_limit = tries < 0 ? (1u << 22) : (unsigned)tries;
    drop_graph(s);   // the graphs hold the limit their launches were made with
    return BDB_OK;
}

int bdb_get_factor_tuning(bdb_system* s, int* chain_sms)
{
    if (!s || !chain_sms) return fail(BDB_ERR_ARG, "null argument");
    *chain_sms = s->chain_sms;
    return BDB_OK;
}

int bdb_set_factor_tuning(bdb_system* s, int chain_sms)
{
    if (!s) return fail(BDB_ERR_ARG, "null system");
    if (chain_sms < 0 || chain_sms > 4096) return fail(BDB_ERR_ARG, "chain SMs out of range");
    if (chain_sms && chain_sms != s->chain_sms) {
        s->chain_sms = chain_sms;
        drop_graph(s);
    }
    s->factor_tuned = true;   // a pinned value is not re-tuned
    return BDB_OK;
}

int bdb_shard_replicas(int nrep, const int* beads, int nshards, int* shard_of)
{
    if (nrep < 0 || nshards < 1 || (nrep > 0 && (!beads || !shard_of)))
        return fail(BDB_ERR_ARG, "bdb_shard_replicas: bad arguments");
    std::vector<int> order(nrep);
    for (int k = 0; k < nrep; ++k) {
        if (beads[k] < 2) return fail(BDB_ERR_ARG, "bdb_shard_replicas: every replica needs at least two beads");
        order[k] = k;
    }
    auto cost = [&](int k) { return (long long)beads[k] * beads[k] + beads[k]; };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
    std::vector<long long> load(nshards, 0);
    for (int k : order) {
        int best = 0;
        for (int g = 1; g < nshards; ++g)
            if (load[g] < load[best]) best = g;
        shard_of[k] = best;
        load[best] += cost(k);
    }
    return BDB_OK;
}

int bdb_set_time(bdb_system* s, double t)
{
    if (!s) return fail(BDB_ERR_ARG, "null system");
    s->sim_time = t;
    return BDB_OK;
}

int bdb_get_time(bdb_system* s, double* t)
{
    if (!s || !t) return fail(BDB_ERR_ARG, "null argument");
    *t = s->sim_time;
    return BDB_OK;
}

int bdb_set_graphs(bdb_system* s, int mode)
{
    if (!s) return fail(BDB_ERR_ARG, "null system");
    if (mode < 0 || mode > 3) return fail(BDB_ERR_ARG, "graph mode is a mask of 1 (steps) and 2 (refreshes)");
    s->graphs = (mode & 1) != 0;
    s->graph_refresh = (mode & 2) != 0;
    drop_graph(s);
    return BDB_OK;
}

int bdb_set_dt(bdb_system* s, double dt)
{
    if (!s || !(dt > 0.0)) return fail(BDB_ERR_ARG, "time step must be positive");
    if (s->p.dt != dt) {
        drop_graph(s);
        // the noise drawn ahead for the next step was scaled with the old dt
        BDB_CUDA(cudaMemsetAsync(s->ctr.p + 2, 0, sizeof(unsigned long long), s->stream));
    }
    s->p.dt = dt;
    return BDB_OK;
}

int bdb_factor_error(bdb_system* s, double* rel_err)
{
    if (!s || !rel_err) return fail(BDB_ERR_ARG, "null argument");
    if (s->p.hydro != BDB_HYDRO_CHOLESKY) return fail(BDB_ERR_STATE, "no stored factor (hydro is not cholesky)");
    int rc;
    BDB_CUDA(cudaMemsetAsync(s->status.p, 0, sizeof(unsigned), s->stream));
    if ((rc = refresh_factor(s))) return rc;
    if ((rc = check_status(s, nullptr))) return rc;
    return factor_error(s, rel_err);
}

int bdb_profile(bdb_system* s, int enable)
{
    if (!s) return fail(BDB_ERR_ARG, "null system");
    s->profiling = enable != 0;
    return BDB_OK;
}

int bdb_phase_stats(bdb_system* s, const char* phase, double* total_ms, long long* calls)
{
    if (!s || !phase || !total_ms || !calls) return fail(BDB_ERR_ARG, "null argument");
    int ph = -1;
    for (int k = 0; k < P_COUNT; ++k)
        if (!strcmp(phase, kPhaseNames[k])) ph = k;
    if (ph < 0) return fail(BDB_ERR_ARG, "unknown phase");
    BDB_CUDA(cudaStreamSynchronize(s->stream));
    if (s->stream2) BDB_CUDA(cudaStreamSynchronize(s->stream2));
    if (s->stream3) BDB_CUDA(cudaStreamSynchronize(s->stream3));
    auto& r = s->phases[ph];
    double tot = 0;
    for (size_t k = 0; k + 1 < r.used; k += 2) {
        float ms = 0;
        BDB_CUDA(cudaEventElapsedTime(&ms, r.ev[k], r.ev[k + 1]));
        tot += ms;
    }
    *total_ms = tot;
    *calls = (long long)(r.used / 2);
    return BDB_OK;
}

int bdb_reset_stats(bdb_system* s)
{
    if (!s) return fail(BDB_ERR_ARG, "null system");
    BDB_CUDA(cudaStreamSynchronize(s->stream));
    for (auto& r : s->phases) r.used = 0;
    s->launches = 0;
    return BDB_OK;
}

int bdb_launches(bdb_system* s, long long* count)
{
    if (!s || !count) return fail(BDB_ERR_ARG, "null argument");
    *count = s->launches;
    return BDB_OK;
}

void* bdb_stream(bdb_system* s) { return s ? (void*)s->stream : nullptr; }

}  // extern "C"
