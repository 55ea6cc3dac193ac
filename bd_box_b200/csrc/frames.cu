// Run state out of the device: asynchronous trajectory frames, and (at the
// end of this file) checkpoint images for resume.
//
// Asynchronous trajectory frames: the positions of every `every`-th step go
// to a ring of pinned host buffers by cudaMemcpyAsync on the engine's
// stream, so the step loop (and its graph replays) never waits for output.
// BD_BOX writes its XYZ/DCD frames from the host copy of coord after each
// saved step (output.c:64-100, save_output :250-257, called from
// main_loop.c:97-116); here the host takes finished frames when it likes.
//
// A frame whose copy has not finished stays in the ring. When the ring is
// full, recording a new frame first waits for the oldest one and moves it to
// a host-side queue, so no frame is ever dropped.
//
// With energies on, a saved step also runs the energy variant of the force
// pass at the new positions (the forces it writes are the ones the step
// already has) and copies E[0..BDB_E_LAST] with the frame: BD_BOX forms E
// only on the steps it writes to the energy file (main_loop.c:102, 112).
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <deque>
#include <vector>

#include "bdb_common.cuh"

namespace bdb {

static constexpr int NE = BDB_E_LAST + 1;   // energies per frame

struct Frame {
    long long step;
    double time;
    std::vector<double> coord;   // 4n: x, y, z, radius
    std::vector<double> E;       // NE, or empty without energies
};

struct FrameRing {
    int every = 1, cap = 0;
    bool energy = false;
    long long start = 0;
    size_t frame_doubles = 0;
    double* host = nullptr;      // pinned: cap frames
    double* host_e = nullptr;    // pinned: cap x NE energies (with energies on)
    std::vector<cudaEvent_t> ev;
    std::vector<long long> step;
    std::vector<double> time;
    int head = 0, count = 0;     // oldest slot, frames in the ring
    std::deque<Frame> spill;     // frames moved out of a full ring, oldest first
};

void frames_release(bdb_system* s)
{
    FrameRing* f = s->frames;
    if (!f) return;
    for (int k = 0; k < f->count; ++k) cudaEventSynchronize(f->ev[(f->head + k) % f->cap]);
    for (auto e : f->ev)
        if (e) cudaEventDestroy(e);
    if (f->host) cudaFreeHost(f->host);
    if (f->host_e) cudaFreeHost(f->host_e);
    delete f;
    s->frames = nullptr;
}

// move the ring's oldest frame to the host-side queue (its copy must be done)
static int spill_oldest(FrameRing* f)
{
    const int slot = f->head;
    BDB_CUDA(cudaEventSynchronize(f->ev[slot]));
    Frame fr;
    fr.step = f->step[slot];
    fr.time = f->time[slot];
    fr.coord.assign(f->host + slot * f->frame_doubles, f->host + (slot + 1) * f->frame_doubles);
    if (f->energy) fr.E.assign(f->host_e + slot * NE, f->host_e + (slot + 1) * NE);
    f->spill.push_back(std::move(fr));
    f->head = (f->head + 1) % f->cap;
    --f->count;
    return BDB_OK;
}

static int record(bdb_system* s)
{
    FrameRing* f = s->frames;
    if (f->count == f->cap) {
        int rc = spill_oldest(f);
        if (rc) return rc;
    }
    const int slot = (f->head + f->count) % f->cap;
    BDB_CUDA(cudaMemcpyAsync(f->host + slot * f->frame_doubles, s->pos.p, sizeof(double) * f->frame_doubles,
                             cudaMemcpyDeviceToHost, s->stream));
    if (f->energy) {
        int rc = forces_run(s, true, false);
        if (rc) return rc;
        s->have_forces = true;
        BDB_CUDA(cudaMemcpyAsync(f->host_e + slot * NE, s->scal.p + 16, sizeof(double) * NE, cudaMemcpyDeviceToHost,
                                 s->stream));
    }
    BDB_CUDA(cudaEventRecord(f->ev[slot], s->stream));
    f->step[slot] = s->step_count;
    f->time[slot] = s->sim_time;
    ++f->count;
    return BDB_OK;
}

// drop the frames of steps after `step` (a step taken back by
// bdb_load_state); their copies may still be in flight, which is harmless:
// the next copy into a freed slot is ordered after them on the same stream
void frames_rewind(bdb_system* s, long long step)
{
    FrameRing* f = s->frames;
    if (!f) return;
    while (f->count > 0 && f->step[(f->head + f->count - 1) % f->cap] > step) --f->count;
    if (f->count == 0)
        while (!f->spill.empty() && f->spill.back().step > step) f->spill.pop_back();
}

// the current step's frame again, after its positions changed (the
// elastic-collision recovery of an accepted step)
int frames_redo_current(bdb_system* s)
{
    FrameRing* f = s->frames;
    if (!f || (s->step_count - f->start) % f->every) return BDB_OK;
    frames_rewind(s, s->step_count - 1);
    return record(s);
}

// after every completed step of bdb_step / bdb_step_igt
int after_step(bdb_system* s, double dt)
{
    ++s->step_count;
    s->sim_time += dt;
    FrameRing* f = s->frames;
    if (!f || (s->step_count - f->start) % f->every) return BDB_OK;
    return record(s);
}

}  // namespace bdb

using namespace bdb;

extern "C" {

int bdb_frames_start(bdb_system* s, int every, int capacity, int with_energy)
{
    if (!s) return fail(BDB_ERR_ARG, "null system");
    if (every < 1 || capacity < 1) return fail(BDB_ERR_ARG, "bdb_frames_start: every and capacity must be >= 1");
    frames_release(s);
    FrameRing* f = new FrameRing;
    s->frames = f;
    f->every = every;
    f->cap = capacity;
    f->energy = with_energy != 0;
    f->start = s->step_count;
    f->frame_doubles = (size_t)4 * s->n;
    f->ev.assign(capacity, nullptr);
    f->step.assign(capacity, 0);
    f->time.assign(capacity, 0.0);
    cudaError_t e = cudaMallocHost(&f->host, sizeof(double) * f->frame_doubles * capacity);
    if (e == cudaSuccess && f->energy) e = cudaMallocHost(&f->host_e, sizeof(double) * NE * capacity);
    for (int k = 0; k < capacity && e == cudaSuccess; ++k) e = cudaEventCreateWithFlags(&f->ev[k], cudaEventDisableTiming);
    if (e != cudaSuccess) {
        frames_release(s);
        return cuda_fail(e, "bdb_frames_start");
    }
    // the starting state is the first frame (main_loop.c:93-97 saves step 0)
    return record(s);
}

int bdb_frames_take(bdb_system* s, int max_frames, long long* steps, double* times, double* coord, double* energies,
                    int* nframes)
{
    if (!s || !nframes || max_frames < 0) return fail(BDB_ERR_ARG, "bad arguments");
    *nframes = 0;
    FrameRing* f = s->frames;
    if (!f) return fail(BDB_ERR_ARG, "bdb_frames_take: frames were not started");
    if (max_frames > 0 && (!steps || !times || !coord)) return fail(BDB_ERR_ARG, "null output array");
    const bool want_e = f->energy && energies;
    // finished frames, oldest first: the queue, then the ring up to the
    // first copy still in flight
    const size_t fd = f->frame_doubles;
    int n = 0;
    while (n < max_frames && !f->spill.empty()) {
        Frame& fr = f->spill.front();
        steps[n] = fr.step;
        times[n] = fr.time;
        std::memcpy(coord + n * fd, fr.coord.data(), sizeof(double) * fd);
        if (want_e) std::memcpy(energies + n * NE, fr.E.data(), sizeof(double) * NE);
        f->spill.pop_front();
        ++n;
    }
    while (n < max_frames && f->count > 0) {
        const int slot = f->head;
        const cudaError_t q = cudaEventQuery(f->ev[slot]);
        if (q == cudaErrorNotReady) break;
        if (q != cudaSuccess) return cuda_fail(q, "bdb_frames_take");
        steps[n] = f->step[slot];
        times[n] = f->time[slot];
        std::memcpy(coord + n * fd, f->host + slot * fd, sizeof(double) * fd);
        if (want_e) std::memcpy(energies + n * NE, f->host_e + slot * NE, sizeof(double) * NE);
        f->head = (f->head + 1) % f->cap;
        --f->count;
        ++n;
    }
    *nframes = n;
    return BDB_OK;
}

int bdb_frames_pending(bdb_system* s, int* nframes)
{
    if (!s || !nframes) return fail(BDB_ERR_ARG, "bad arguments");
    FrameRing* f = s->frames;
    *nframes = f ? (int)f->spill.size() + f->count : 0;
    return BDB_OK;
}

int bdb_frames_flush(bdb_system* s)
{
    if (!s) return fail(BDB_ERR_ARG, "null system");
    FrameRing* f = s->frames;
    if (!f) return BDB_OK;
    for (int k = 0; k < f->count; ++k) BDB_CUDA(cudaEventSynchronize(f->ev[(f->head + k) % f->cap]));
    return BDB_OK;
}

int bdb_frames_stop(bdb_system* s)
{
    if (!s) return fail(BDB_ERR_ARG, "null system");
    frames_release(s);
    return BDB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Checkpoints: the state a resumed run needs, as a flat host image.

namespace bdb {

struct CheckpointHeader {
    uint64_t magic;              // "BDBCKPT1"
    int64_t n;
    int64_t step_count;
    double sim_time;
    int64_t steps_since_refresh;
    uint64_t philox_stream;
    double dt;
};

static constexpr uint64_t CKPT_MAGIC = 0x3154504b43424442ull;   // "BDBCKPT1" little-endian

}  // namespace bdb

extern "C" {

size_t bdb_checkpoint_size(bdb_system* s)
{
    return s ? sizeof(CheckpointHeader) + sizeof(double4) * (size_t)s->n : 0;
}

int bdb_checkpoint_save(bdb_system* s, void* buf, size_t bytes)
{
    if (!s || !buf) return fail(BDB_ERR_ARG, "null argument");
    if (bytes < bdb_checkpoint_size(s)) return fail(BDB_ERR_ARG, "checkpoint buffer too small");
    CheckpointHeader h;
    h.magic = CKPT_MAGIC;
    h.n = s->n;
    h.step_count = s->step_count;
    h.sim_time = s->sim_time;
    h.steps_since_refresh = s->steps_since_refresh;
    h.dt = s->p.dt;
    unsigned long long stream = 0;
    BDB_CUDA(cudaMemcpyAsync(&stream, s->ctr.p, sizeof stream, cudaMemcpyDeviceToHost, s->stream));
    unsigned char* out = static_cast<unsigned char*>(buf);
    BDB_CUDA(cudaMemcpyAsync(out + sizeof h, s->pos.p, sizeof(double4) * s->n, cudaMemcpyDeviceToHost, s->stream));
    BDB_CUDA(cudaStreamSynchronize(s->stream));
    h.philox_stream = stream;
    std::memcpy(out, &h, sizeof h);
    return BDB_OK;
}

int bdb_checkpoint_load(bdb_system* s, const void* buf, size_t bytes)
{
    if (!s || !buf) return fail(BDB_ERR_ARG, "null argument");
    CheckpointHeader h;
    if (bytes < sizeof h) return fail(BDB_ERR_ARG, "checkpoint image too small");
    std::memcpy(&h, buf, sizeof h);
    if (h.magic != CKPT_MAGIC) return fail(BDB_ERR_ARG, "not a checkpoint image");
    if (h.n != s->n || bytes < bdb_checkpoint_size(s)) return fail(BDB_ERR_ARG, "checkpoint of another bead count");
    const unsigned char* in = static_cast<const unsigned char*>(buf);
    BDB_CUDA(cudaMemcpyAsync(s->pos.p, in + sizeof h, sizeof(double4) * s->n, cudaMemcpyHostToDevice, s->stream));
    // the stream index, the block count, no noise drawn ahead
    const unsigned long long ctr[3] = {h.philox_stream, 0ull, 0ull};
    BDB_CUDA(cudaMemcpyAsync(s->ctr.p, ctr, sizeof ctr, cudaMemcpyHostToDevice, s->stream));
    BDB_CUDA(cudaMemsetAsync(s->cells_built.p, 0, sizeof(int) * s->segs.size(), s->stream));
    BDB_CUDA(cudaStreamSynchronize(s->stream));   // ctr is a stack array
    s->step_count = h.step_count;
    s->sim_time = h.sim_time;
    s->steps_since_refresh = (int)h.steps_since_refresh;
    if (s->p.dt != h.dt) {
        s->p.dt = h.dt;
        drop_graph(s);
    }
    s->have_forces = false;     // recomputed at the next step
    s->factor_valid = false;    // the stored tensor and its factor are rebuilt at the next step
    s->igt_ready = false;       // a pending IGT predictor belongs to the replaced state
    return BDB_OK;
}

}  // extern "C"
