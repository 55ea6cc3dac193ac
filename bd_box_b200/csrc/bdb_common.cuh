// Shared definitions of the bdb200 engine: the system object, error
// plumbing, physical constants and the exact-arithmetic helpers used where
// a decision (cutoff, overlap, periodic image) must match BD_BOX's double
// arithmetic bit for bit.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/bdb200.h"

// data.h:207-211 (double build)
#define BDB_KB 0.001986248532617
#define BDB_KB_1_8PI 0.00007903031804378703
#define BDB_KB_1_6PI 0.00010537375739171604
#define BDB_SQRTPI 1.77245385090551602729
#define BDB_M1_SQRTPI 0.5641895835
#define BDB_M_PIF 3.14159265358979323846f
#define BDB_PI_D 3.14159265358979323846

namespace bdb {

void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define BDB_CUDA(call)                                              \
    do {                                                            \
        cudaError_t e_ = (call);                                    \
        if (e_ != cudaSuccess) return ::bdb::cuda_fail(e_, #call);  \
    } while (0)

// Device status word bits, written by kernels, read by the host after a step.
enum : unsigned {
    ST_OVERLAP = 1u,      // overlap / NaN of a force term (retry contract)
    ST_BOND = 2u,         // over-stretched FENE bond (fatal in the reference)
    ST_NOT_SPD = 4u,      // non-positive Cholesky pivot
    ST_TIMEOUT = 8u,      // a bounded wait gave up
    ST_LAUNCH = 16u,      // a kernel found its launch shape wrong and did nothing
};

// A bead segment: one independent system inside a batch.
struct FrameRing;   // asynchronous trajectory frames (frames.cu)

struct Segment {
    int begin;     // first bead
    int count;     // beads
    int pbegin;    // first padded matrix row (stored-D systems)
};

// A TEA / D.F work item: bead tiles (I, J), I >= J, of one segment.
struct TileJob {
    int seg;
    int I, J;
};

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    int alloc(size_t count);
    void release();
    ~DevBuf() { release(); }
};

}  // namespace bdb

struct bdb_system {
    bdb_params p;
    int n = 0;       // beads
    int n3 = 0;      // 3n
    int npad = 0;    // stored-matrix dimension (3n rounded up to the tile)
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr;            // Cholesky: bulk trailing updates
    cudaStream_t stream3 = nullptr;            // Cholesky: the panel chain's side work
    cudaEvent_t la_ev[6] = {};                 // their hand-offs (chol_tc.cu)
    double inv_L[3] = {0, 0, 0};
    double preDii = 0, preDij = 0;

    std::vector<bdb::Segment> segs;
    bdb::DevBuf<bdb::Segment> d_segs;
    bdb::DevBuf<int> d_bead_seg;

    // state
    bdb::DevBuf<double4> pos, pos_save;
    bdb::DevBuf<double> F, F_save, Q;
    bdb::DevBuf<double2> LJ;
    bool have_forces = false;

    // bonded terms (CSR gather)
    int n_bond = 0, n_angle = 0, n_angle_cos = 0, n_dihe = 0, n_dihe_angle = 0;
    bdb::DevBuf<int> bond_pairs, angle_pairs, angle_cos_pairs, dihe_pairs, dihe_angle_pairs;
    bdb::DevBuf<double> bond_parms, angle_parms, angle_cos_parms, dihe_parms, dihe_angle_parms;
    bdb::DevBuf<int> slot_ptr, slot_list;      // bead -> contribution slots
    bdb::DevBuf<double> contrib;               // 3 doubles per slot
    bdb::DevBuf<double> term_energy;           // one per bonded term
    int n_slots = 0, n_terms = 0;
    bdb::DevBuf<int> conn_ptr, conn_list;      // 1-2 bonded neighbours (are_conn)
    bool conn_live = false;

    // cell list
    bdb::DevBuf<unsigned long long> sorted_keys;   // (cell << 24 | local) per bead, per segment sorted
    bdb::DevBuf<int> sorted_idx;
    bdb::DevBuf<double4> grid;                 // per segment: origin xyz, cell size
    bdb::DevBuf<int4> grid_dims;               // per segment: nx, ny, nz, brute flag
    bdb::DevBuf<double4> pos_build;            // positions when the cell list was last sorted
    bdb::DevBuf<int2> cell_range;              // dense per-segment table: [first, end) of each cell
    bdb::DevBuf<long long> cell_off;           // per segment: offset of its table, capacity
    bdb::DevBuf<int> cells_built;              // per segment: 1 once sorted
    bdb::DevBuf<int> cells_resort;             // per segment above the shared-memory sort: re-sort now
    bdb::DevBuf<unsigned long long> big_keys;  // two key buffers of the multi-CTA sort (forces.cu)
    size_t big_npow = 0;                       // their length each: the largest such segment, to a power of 2
    double cell_size = 0;
    double skin = 0;

    // force outputs
    bdb::DevBuf<double> e_part;                // energy partials
    bdb::DevBuf<unsigned> status;              // status word
    bdb::DevBuf<unsigned long long> counts;    // pair counts

    // hydrodynamics
    bdb::DevBuf<double> Rf, Rs, X, dD, work;   // 3n vectors, diag, scratch
    bdb::DevBuf<double> part;                  // TEA / symv partial sums
    bdb::DevBuf<double> eps_part;
    bdb::DevBuf<double> scal;                  // device scalars (eps, beta, ...)
    bdb::DevBuf<bdb::TileJob> jobs;
    bdb::DevBuf<int> tea_next;                 // job counter of the persistent TEA pair kernel
    bdb::DevBuf<float> pscale;                 // mixed Cholesky: FP16 panel scale and 1/scale^2
    bdb::DevBuf<unsigned char> tea_meta;       // TEA segment table + job offsets
    int n_jobs = 0;
    int tea_tile = 32;                         // TEA tile edge (16 or 32 beads)
    int mv_warps = 16;                         // stored matvec: target warps per SM
    int chain_sms = 32;                        // Cholesky: SMs the bulk updates leave to the panel chain
                                               // (set per precision at creation)
    bool autotune = false, tea_tuned = false, mv_tuned = false, factor_tuned = false;
    bdb::DevBuf<double> ewald_tab;             // Ewald lattice tables (rpy_tile.cuh EwaldConst)
    int ewald_nk = 0, ewald_nimg = 0;
    bdb::DevBuf<double> M64;                   // stored D (upper) + L (lower), FP64
    bdb::DevBuf<float> M32;                    // same, FP32 (mixed path)
    // IGT predictor-corrector: the tensor at the predicted positions, the
    // step's starting positions, the two deterministic displacements and
    // diag(D) at the start
    bdb::DevBuf<double> M64b;
    bdb::DevBuf<float> M32b;
    bdb::DevBuf<double4> pos_igt;
    bdb::DevBuf<double> Rf_igt, Rf2_igt, dD_igt;
    bdb::DevBuf<double> fs_igt;                // the predictor's flow displacement (flowing solvent)
    bool igt_ready = false;                    // a predictor awaits its corrector
    bdb::DevBuf<double> panel64;               // Cholesky workspace
    bool factor_valid = false;
    alignas(64) unsigned char tc_map[2048];    // CUtensorMaps: FP16 hi / lo panel buffers (x4), FP32 matrix
    bool tc_map_ok = false;
    bool tc64_ok = false;                      // FP64 tensor-core Cholesky set up
    alignas(64) unsigned char mv_map[384];     // CUtensorMaps for the stored matvec: FP32 matrix, X, F
    const void* mv_map_src[3] = {};            // buffers the maps were encoded for
    int mv_ctas_per_sm = 0;                    // resident CTAs of the TMA matvec kernel per SM
    int sm_count = 148;
    unsigned wait_limit = 1u << 22;            // tries of every bounded device wait (bdb_set_wait_limit)
    int steps_since_refresh = 0;

    // noise: Philox stream index and finished-block count (device)
    bdb::DevBuf<unsigned long long> ctr;

    // CUDA graph of the steady part of a step (noise .. forces), replayed
    // while no refresh is due; rebuilt after anything its launches captured
    // changes (time step, bonded terms)
    cudaGraphExec_t step_graph = nullptr;
    long long graph_launches = 0;
    // the same for steps with caller Gaussians, for the device copy of them
    // at the address it captured (the staging buffer's first slot)
    cudaGraphExec_t step_graph_host = nullptr;
    const double* step_graph_host_src = nullptr;
    long long graph_launches_host = 0;
    long long eager_steps = 0;
    cudaGraphExec_t refresh_graph = nullptr;   // tensor build + factorisation (mixed path)
    long long refresh_launches = 0, eager_refreshes = 0;
    bool graphs = true, graph_refresh = true;
    bool fuse_step = true;                     // Cholesky steps: noise drawn ahead, update in the product's finisher

    // steps taken (bdb_step, bdb_step_igt), simulated time, and the frame
    // ring of bdb_frames_start
    long long step_count = 0;
    double sim_time = 0;
    bdb::FrameRing* frames = nullptr;
    long long saved_step_count = 0;            // bdb_save_state's copy
    double saved_sim_time = 0;

    // elastic-collision recovery (newton.cu): velocities, masses, pair list,
    // scan scalars, and the previous scan's list size (BD_BOX keeps it global)
    bdb::DevBuf<double> nw_vel, nw_mass;
    bdb::DevBuf<int> nw_pairs;
    bdb::DevBuf<unsigned long long> nw_scal;
    int nw_prev_ints = 0;

    // measurement: CUDA-event pairs per phase, kernel launch count
    struct PhaseRec {
        std::vector<cudaEvent_t> ev;   // begin/end pairs
        size_t used = 0;
    };
    PhaseRec phases[16];
    bool profiling = false;
    long long launches = 0;
    bdb::DevBuf<double> gbuf;          // device copy of caller Gaussians
};

namespace bdb {

// ---- exact double arithmetic (no FMA contraction) -------------------------
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// trans_dist_vec (trans.c:111-121): v = v2 - v1, minimum image if periodic,
// evaluated exactly as the reference evaluates it.
__device__ __forceinline__ void dist_vec(const double4& v1, const double4& v2, int periodic,
                                         const double* box, const double* inv_L, double* v)
{
    v[0] = sub(v2.x, v1.x);
    v[1] = sub(v2.y, v1.y);
    v[2] = sub(v2.z, v1.z);
    if (periodic) {
#pragma unroll
        for (int k = 0; k < 3; ++k)
            v[k] = sub(v[k], mul(box[k], floor(add(mul(v[k], inv_L[k]), 0.5))));
    }
}

// sq3v (math_help.c:30-33)
__device__ __forceinline__ double sq3(const double* v)
{
    return add(add(mul(v[0], v[0]), mul(v[1], v[1])), mul(v[2], v[2]));
}

}  // namespace bdb

// kernel entry points used across translation units
namespace bdb {
enum Phase {
    P_STEP, P_REFRESH, P_BUILD, P_FACTOR, P_MATVEC, P_TEA, P_FORCES, P_NOISE, P_UPDATE,
    // kernels of the mixed-precision factorisation, each on its own stream
    P_POTRF, P_TRSM, P_SYRK_COL, P_SYRK_REST, P_COUNT
};
void phase_mark(bdb_system* s, int phase);   // records begin/end events when profiling
void phase_mark_on(bdb_system* s, int phase, cudaStream_t stream);
void drop_graph(bdb_system* s);              // forget the captured step
int after_step(bdb_system* s, double dt);     // count a finished step, record a frame when due
void frames_release(bdb_system* s);           // wait for frame copies in flight, free the ring
void frames_rewind(bdb_system* s, long long step);   // drop frames of steps after `step`
int frames_redo_current(bdb_system* s);       // record the current step's frame again
int build_and_factor(bdb_system* s);         // tensor build + factorisation into the stored matrix, eagerly
int forces_phase(bdb_system* s);             // forces at the current positions (profiled phase)
int check_status(bdb_system* s, bool* overlap);   // read and decode the status word (synchronises)
int forces_setup(bdb_system* s);
int forces_run(bdb_system* s, bool want_energy, bool want_counts);
int set_force_time(bdb_system* s, double t);   // time of the next force evaluations (time-dependent field only)
int bonded_setup(bdb_system* s);
int tensor_build(bdb_system* s);       // stored D into M64/M32 + dD
int tensor_tile_host(bdb_system* s, int i, int j, double* tD);
int factor_run(bdb_system* s);         // Cholesky of the stored D in place
int stored_matvec(bdb_system* s, bool want_rs);   // Rf = D.F (upper), Rs = L.X (lower)
int stored_matvec_step(bdb_system* s);   // mixed path: noise drawn in the product, update in its finisher
int tea_run(bdb_system* s, bool want_rs);         // matrix-free D.F (+ TEA noise)
int noise_fill(bdb_system* s, const double* host_gauss);   // X = unit Gaussians
int update_positions(bdb_system* s, double* fs = nullptr);  // pos += Rf + Rs, periodic wrap
int diag_noise(bdb_system* s);        // hydro none: Rs = X sqrt(2 dt D_ii)
int factor_error(bdb_system* s, double* rel);
int ensure_matrix(bdb_system* s);    // allocate the stored matrix (identity padding)
int engine_step(bdb_system* s);      // one Ermak-McCammon step, device noise

// Copies and fills ordered on the system's stream. The system's streams are
// non-blocking: they do not wait for the legacy default stream, where a plain
// cudaMemcpy / cudaMemset goes, so a fill queued there may land after (and
// erase) what a kernel on the system's stream has written since, and a plain
// device-to-host copy may read before that kernel has finished.
inline cudaError_t h2d(const bdb_system* s, void* dst, const void* src, size_t bytes)
{
    // a pageable source is staged before the call returns
    return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s->stream) : cudaSuccess;
}
inline cudaError_t d2h(const bdb_system* s, void* dst, const void* src, size_t bytes)
{
    if (!bytes) return cudaSuccess;
    const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s->stream);
    return e != cudaSuccess ? e : cudaStreamSynchronize(s->stream);
}
inline cudaError_t dzero(const bdb_system* s, void* dst, size_t bytes)
{
    return bytes ? cudaMemsetAsync(dst, 0, bytes, s->stream) : cudaSuccess;
}
}  // namespace bdb
