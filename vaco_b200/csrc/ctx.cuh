// ctx.cuh -- the vaco_av1_ctx object behind the C ABI (internal).
#pragma once

#include <map>
#include <string>

#include "common.cuh"

#include <vector>

namespace vaco {
inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }
}  // namespace vaco

struct vaco_av1_ctx {
    using size_t = ::size_t;
    int device = 0;
    cudaStream_t stream = nullptr;
    vaco::DeviceStatus* status = nullptr;     // device
    unsigned long long* status_host = nullptr;  // pinned
    int last_cuda_error = 0;
    uint64_t launches = 0;
    // deferred status (vaco_av1_ctx_set_deferred_status): chain calls on
    // device pointers enqueue and return; vaco_av1_ctx_flush reads the word
    bool deferred = false;
    // stage timing (vaco_av1_ctx_set_stage_timing): five events per frame,
    // from a ring of kMarkRing frames so that frames enqueued under deferred
    // status are all timed; a frame's events are read once its last one has
    // completed.
    static constexpr int kMarkRing = 128;
    bool timing = false;
    int timing_every = 1;        // time one frame in this many
    uint64_t timing_count = 0;   // frames seen while timing
    bool timing_this = false;    // the current frame is timed
    cudaEvent_t marks[kMarkRing][5] = {};
    uint64_t mark_head = 0, mark_tail = 0;  // frames recorded / frames read
    double stage_ms[4] = {0, 0, 0, 0};
    uint64_t timed_frames = 0;

    void read_marks(int slot) {
        for (int i = 0; i < 4; ++i) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, marks[slot][i], marks[slot][i + 1]) == cudaSuccess) stage_ms[i] += ms;
        }
        ++timed_frames;
    }
    void mark(int i, cudaStream_t s) {
        if (!timing) return;
        if (i == 0) timing_this = timing_count++ % (uint64_t)timing_every == 0;
        if (!timing_this) return;
        if (i == 0 && mark_head - mark_tail == kMarkRing) {
            // the ring is full: wait for the oldest frame and read it
            const int old = (int)(mark_tail % kMarkRing);
            cudaEventSynchronize(marks[old][4]);
            read_marks(old);
            ++mark_tail;
        }
        cudaEventRecord(marks[mark_head % kMarkRing][i], s);
        if (i == 4) ++mark_head;
    }
    // Called after the stream has been synchronized.
    void collect_marks() {
        for (; mark_tail < mark_head; ++mark_tail) read_marks((int)(mark_tail % kMarkRing));
    }
    struct Buf {
        void* p = nullptr;
        size_t n = 0;
    };
    // Scratch sets: 0 for the synchronous entry points, 1 + k for slot k of
    // the pipelined host entry points (each slot's frame keeps its own
    // buffers while the next ones are copied in).
    static constexpr int kPipeSlots = 3;
    static constexpr int kScratchSets = 1 + kPipeSlots;
    Buf bufs[kScratchSets][40];
    int scratch_set = 0;

    // pipelined host entry points (vaco_av1_postfilter_frame_host_submit / _wait)
    struct PipeSlot {
        bool busy = false;
        uint64_t ticket = 0;
        cudaEvent_t staged = nullptr, filtered = nullptr, done = nullptr;
        vaco::DeviceStatus* status = nullptr;       // device
        unsigned long long* status_host = nullptr;  // pinned
    };
    PipeSlot pipe[kPipeSlots];
    cudaStream_t copy_in = nullptr, copy_out = nullptr;
    uint64_t next_ticket = 1;

    // film grain (grain.cu): workspace sets whose template kernels run on
    // their own streams, so the templates of consecutive frames (which depend
    // only on the parameters) overlap each other and the frames' other work
    static constexpr int kGrainSets = 8;
    struct GrainSet {
        cudaStream_t stream = nullptr;
        cudaEvent_t ready = nullptr;  // the set's templates are written
        cudaEvent_t free = nullptr;   // the last apply that read the set has run
        bool used = false;
    };
    GrainSet grain[kGrainSets];
    uint64_t grain_next = 0;

    // batched form (batch.cu)
    vaco_av1_tuning tuning = {3, 4, 1, 1, 256, 1};
    unsigned char* batch_table_host = nullptr;   // pinned staging of the per-batch tables
    size_t batch_table_host_bytes = 0;
    unsigned long long* batch_status_host = nullptr;  // pinned copy of the per-frame status words
    size_t batch_status_host_count = 0;
    std::map<std::string, cudaGraphExec_t> graphs;   // by batch composition (and scratch generation)
    unsigned long long scratch_generation = 0;       // bumps whenever a scratch slot is reallocated
    int sm_count = 0;

    void* scratch(int slot, size_t bytes) {
        Buf& b = bufs[scratch_set][slot];
        if (b.n >= bytes && b.p) return b.p;
        // Work enqueued without a host sync (deferred status) may still use
        // the old buffer: let it finish before the buffer goes.
        if (b.p) {
            cudaDeviceSynchronize();
            cudaFree(b.p);
        }
        b.p = nullptr;
        b.n = 0;
        size_t n = vaco::align_up(bytes < 256 ? 256 : bytes, 256);
        if (cudaMalloc(&b.p, n) != cudaSuccess) return nullptr;
        b.n = n;
        ++scratch_generation;
        return b.p;
    }
};

// Scratch slots
enum Slot {
    S_PRE0 = 0, S_PRE1, S_PRE2,       // deblocked (pre-CDEF) planes
    S_CDEF0, S_CDEF1, S_CDEF2,        // CDEF output planes
    S_UPRE0, S_UPRE1, S_UPRE2,        // upscaled pre-CDEF planes
    S_UCDEF0, S_UCDEF1, S_UCDEF2,     // upscaled CDEF planes
    S_H_IN0, S_H_IN1, S_H_IN2,        // host-entry staging (inputs)
    S_H_OUT0, S_H_OUT1, S_H_OUT2,     // host-entry staging (outputs)
    S_H_SIDE0, S_H_SIDE1, S_H_SIDE2, S_H_SIDE3, S_H_SIDE4, S_H_SIDE5,
    S_BATCH_ARENA, S_BATCH_TABLE,      // batched form: intermediates, per-batch tables
    S_EMIT0, S_EMIT1, S_EMIT2,         // host-entry emission: packed frame planes
    S_GRAIN0,                          // film grain workspace sets S_GRAIN0 .. + kGrainSets - 1
    S_GRAIN_END = S_GRAIN0 + vaco_av1_ctx::kGrainSets,
};
static_assert(S_GRAIN_END <= (int)(sizeof(vaco_av1_ctx::bufs[0]) / sizeof(vaco_av1_ctx::Buf)),
              "every scratch slot needs a buffer in each set");


namespace vaco {
// Asynchronous halves of vaco_av1_postfilter_batch_dev (batch.cu).
struct BatchPending {
    int n = 0;
    std::vector<unsigned long long> host_keys;
    std::vector<int> queued;  // frames whose device status word is live
};
int32_t batch_enqueue(vaco_av1_ctx* ctx, cudaStream_t s, const vaco_av1_frame_job* jobs, int n, BatchPending* pending);
int32_t batch_collect(vaco_av1_ctx* ctx, const BatchPending& pending, int32_t* statuses, int32_t* msgs);
}  // namespace vaco
