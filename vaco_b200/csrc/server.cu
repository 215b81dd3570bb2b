// server.cu -- the served form: continuous batching of frames from many
// decoder streams (no counterpart in vaco, which filters each frame inside its
// own decode_frame call, crates/codec/vaco-codec-av1/src/decode.rs:553-559).
//
// Model:
//   - A stream is admitted with its geometry and a number of frame slots; the
//     slots' pictures, side information and restoration units are allocated
//     once in device memory and stay resident (the decoder writes into them).
//     Admission fails when the memory budget cannot hold them.
//   - submit() queues a slot with its frame-level parameters and returns a
//     ticket without blocking.
//   - One worker thread owns `inflight_batches` launch slots, each with its own
//     context (scratch arena, pinned tables) and CUDA stream.  Whenever a
//     launch slot is free and frames are pending, it packs the pending frames
//     (FIFO, up to max_batch_frames and the slot's scratch share) into one
//     batched launch set (batch.cu) and records an event; frames submitted
//     meanwhile wait for the next free launch slot, so consecutive launch sets
//     overlap on the device.
//   - Completion is detected by polling the events (host side only: no device
//     wait of any kind), after which tickets carry the frame's status and its
//     submit-to-completion latency.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "ctx.cuh"
#include "kernels.cuh"

using namespace vaco;
using Clock = std::chrono::steady_clock;

namespace {

struct SlotBuffers {
    vaco_av1_frame_job job;  // device pointers of this frame slot
    std::vector<void*> allocations;
    bool in_flight = false;
    cudaEvent_t uploaded = nullptr;  // recorded after a submit_host's input copies
};

struct StreamState {
    bool open = false;
    vaco_av1_frame_info info{};
    int lr_unit_size[3] = {0, 0, 0};
    std::vector<SlotBuffers> slots;
    int64_t bytes = 0;
    int64_t scratch_estimate = 0;  // batch scratch one frame of this stream needs
};

struct Pending {
    uint64_t ticket;
    int stream, slot;
    vaco_av1_frame_job job;
    int64_t scratch;
    Clock::time_point submitted;
    cudaEvent_t upload = nullptr;  // the launch waits for it (submit_host)
};

struct TicketState {
    bool done = false;
    int32_t status = VACO_AV1_OK, msg = 0;
    double latency_ms = 0;
};

struct LaunchSlot {
    vaco_av1_ctx* ctx = nullptr;
    cudaEvent_t done = nullptr;
    bool busy = false;
    std::vector<Pending> jobs;
    std::vector<vaco_av1_frame_job> table;
    BatchPending pending;
};

// Default bound of the server's host waits (a slot's backpressure in submit,
// a stream's in-flight frames in close_stream), in 1 ms polls.
constexpr int kDefaultWaitPolls = 10000;

size_t plane_bytes(int w, int h) { return align_up((size_t)align_up((size_t)std::max(w, 1), 64) * std::max(h, 1) * 2, 256); }

}  // namespace

struct vaco_av1_server {
    vaco_av1_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Pending> pending;
    std::unordered_map<uint64_t, TicketState> tickets;
    std::vector<StreamState> streams;
    std::vector<LaunchSlot> launch;
    uint64_t next_ticket = 1;
    int64_t resident = 0, stream_budget = 0, scratch_share = 0;
    // host->device copies of submit_host, spread over a few copy streams (by
    // slot) so one frame's copies overlap the set-up of another's
    static constexpr int kUploadStreams = 4;
    cudaStream_t upload_streams[kUploadStreams] = {};
    int wait_polls = kDefaultWaitPolls;      // bound of submit / close_stream waits
    vaco_av1_server_stats stats{};
    bool stop = false;
    std::thread worker;

    void finish(LaunchSlot& ls, cudaError_t err) {
        std::vector<int32_t> st(ls.jobs.size()), ms(ls.jobs.size());
        if (err == cudaSuccess) {
            batch_collect(ls.ctx, ls.pending, st.data(), ms.data());
        } else {
            std::fill(st.begin(), st.end(), (int32_t)VACO_AV1_DEVICE_ERROR);
            std::fill(ms.begin(), ms.end(), (int32_t)VACO_AV1_MSG_CUDA);
        }
        const auto now = Clock::now();
        for (size_t i = 0; i < ls.jobs.size(); ++i) {
            const Pending& p = ls.jobs[i];
            auto it = tickets.find(p.ticket);
            if (it != tickets.end()) {
                it->second.done = true;
                it->second.status = st[i];
                it->second.msg = ms[i];
                it->second.latency_ms = std::chrono::duration<double, std::milli>(now - p.submitted).count();
            }
            if (p.stream < (int)streams.size() && p.slot < (int)streams[p.stream].slots.size())
                streams[p.stream].slots[p.slot].in_flight = false;
            ++stats.completed;
            if (st[i] != VACO_AV1_OK) ++stats.failed;
        }
        ls.jobs.clear();
        ls.busy = false;
        cv_done.notify_all();
    }

    void run() {
        cudaSetDevice(cfg.device);
        std::unique_lock<std::mutex> lk(mu);
        while (!stop) {
            bool progressed = false;
            for (LaunchSlot& ls : launch) {
                if (!ls.busy) continue;
                const cudaError_t q = cudaEventQuery(ls.done);
                if (q == cudaErrorNotReady) continue;
                finish(ls, q);
                progressed = true;
            }
            for (LaunchSlot& ls : launch) {
                if (ls.busy || pending.empty()) continue;
                // pack pending frames FIFO within the batch size and scratch share
                int64_t scratch = 0;
                while (!pending.empty() && (int)ls.jobs.size() < cfg.max_batch_frames &&
                       (ls.jobs.empty() || scratch + pending.front().scratch <= scratch_share)) {
                    scratch += pending.front().scratch;
                    ls.jobs.push_back(pending.front());
                    pending.pop_front();
                }
                ls.table.resize(ls.jobs.size());
                for (size_t i = 0; i < ls.jobs.size(); ++i) ls.table[i] = ls.jobs[i].job;
                // the launch slot belongs to this thread: submitters may proceed meanwhile
                lk.unlock();
                // frames submitted with their inputs: the launch follows their copies
                cudaError_t we = cudaSuccess;
                for (const Pending& j : ls.jobs)
                    if (j.upload && we == cudaSuccess) we = cudaStreamWaitEvent(ls.ctx->stream, j.upload, 0);
                int32_t st = we == cudaSuccess ? batch_enqueue(ls.ctx, ls.ctx->stream, ls.table.data(),
                                                               (int)ls.table.size(), &ls.pending)
                                               : VACO_AV1_DEVICE_ERROR;
                cudaError_t e = st == VACO_AV1_OK ? cudaEventRecord(ls.done, ls.ctx->stream) : cudaErrorUnknown;
                lk.lock();
                ++stats.batches;
                stats.max_batch = std::max<uint64_t>(stats.max_batch, ls.jobs.size());
                if (e != cudaSuccess) {
                    finish(ls, e);
                } else {
                    ls.busy = true;
                }
                progressed = true;
            }
            if (!progressed) {
                bool any_busy = false;
                for (const LaunchSlot& ls : launch) any_busy = any_busy || ls.busy;
                // bounded host waits: poll in-flight events often, idle longer
                cv_work.wait_for(lk, any_busy ? std::chrono::microseconds(20) : std::chrono::milliseconds(5));
            }
        }
        // drain: wait (bounded per poll) for in-flight work before exiting
        for (LaunchSlot& ls : launch)
            if (ls.busy) finish(ls, cudaEventSynchronize(ls.done));
    }
};

namespace {

void free_stream(StreamState& s) {
    for (SlotBuffers& b : s.slots) {
        for (void* p : b.allocations) cudaFree(p);
        if (b.uploaded) cudaEventDestroy(b.uploaded);
    }
    s.slots.clear();
    s.open = false;
}

}  // namespace

extern "C" int32_t vaco_av1_server_create(const vaco_av1_server_config* config, vaco_av1_server** out) {
    if (!config || !out || config->max_batch_frames < 1 || config->inflight_batches < 1 ||
        config->inflight_batches > 8 || config->memory_budget_bytes <= 0 || config->host_wait_ms < 0)
        return VACO_AV1_INVALID_DATA;
    *out = nullptr;
    if (cudaSetDevice(config->device) != cudaSuccess) return VACO_AV1_DEVICE_ERROR;
    vaco_av1_server* s = new vaco_av1_server();
    s->cfg = *config;
    if (config->host_wait_ms > 0) s->wait_polls = config->host_wait_ms;
    // a quarter of the budget is reserved for batch scratch, shared by the launch slots
    const int64_t scratch_total = config->memory_budget_bytes / 4;
    s->scratch_share = scratch_total / config->inflight_batches;
    s->stream_budget = config->memory_budget_bytes - scratch_total;
    s->stats.scratch_bytes = scratch_total;
    s->launch.resize(config->inflight_batches);
    for (cudaStream_t& us : s->upload_streams)
        if (cudaStreamCreateWithFlags(&us, cudaStreamNonBlocking) != cudaSuccess) {
            vaco_av1_server_destroy(s);
            return VACO_AV1_DEVICE_ERROR;
        }
    for (LaunchSlot& ls : s->launch) {
        if (vaco_av1_ctx_create(config->device, &ls.ctx) != VACO_AV1_OK ||
            cudaEventCreateWithFlags(&ls.done, cudaEventDisableTiming) != cudaSuccess) {
            vaco_av1_server_destroy(s);
            return VACO_AV1_DEVICE_ERROR;
        }
        ls.ctx->tuning.use_graphs = 0;  // compositions vary from launch to launch
        // Reserve the slot's scratch share up front so no launch stalls on an
        // allocation under load (the batch arena otherwise grows on demand).
        if (!ls.ctx->scratch(S_BATCH_ARENA, (size_t)s->scratch_share)) {
            vaco_av1_server_destroy(s);
            return VACO_AV1_DEVICE_ERROR;
        }
    }
    s->worker = std::thread([s] { s->run(); });
    *out = s;
    return VACO_AV1_OK;
}

extern "C" void vaco_av1_server_destroy(vaco_av1_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->cfg.device);
    for (LaunchSlot& ls : s->launch) {
        if (ls.done) cudaEventDestroy(ls.done);
        if (ls.ctx) vaco_av1_ctx_destroy(ls.ctx);
    }
    for (StreamState& st : s->streams) free_stream(st);
    for (cudaStream_t us : s->upload_streams)
        if (us) cudaStreamDestroy(us);
    delete s;
}

extern "C" int32_t vaco_av1_server_open_stream(vaco_av1_server* s, const vaco_av1_frame_info* info,
                                               const int32_t* lr_unit_size, int32_t buffers, int32_t* stream_id,
                                               int32_t* msg) {
    if (msg) *msg = 0;
    if (!s || !info || !stream_id || buffers < 1 || buffers > 64) return VACO_AV1_INVALID_DATA;
    const vaco_av1_frame_info& i = *info;
    if (i.mi_rows <= 0 || i.mi_cols <= 0 || i.coded_width <= 0 || i.coded_height <= 0 ||
        i.mi_cols != 2 * ((i.coded_width + 7) >> 3) || i.mi_rows != 2 * ((i.coded_height + 7) >> 3) ||
        i.upscaled_width < i.coded_width || !av1_subsampling_ok(i.subsampling_x, i.subsampling_y)) {
        if (msg) *msg = VACO_AV1_MSG_FRAME_GEOMETRY;
        return VACO_AV1_INVALID_DATA;
    }
    const int np = i.monochrome ? 1 : 3;
    const int ssx = i.subsampling_x, ssy = i.subsampling_y;
    // per-slot byte layout
    struct Part {
        size_t bytes;
    };
    int64_t slot_bytes = 0;
    size_t in_bytes[3] = {0, 0, 0}, out_bytes[3] = {0, 0, 0};
    int unit_counts[3] = {0, 0, 0};
    for (int k = 0; k < np; ++k) {
        const int sx = k ? ssx : 0, sy = k ? ssy : 0;
        in_bytes[k] = plane_bytes((i.mi_cols * 4) >> sx, (i.mi_rows * 4) >> sy);
        out_bytes[k] = plane_bytes(i.upscaled_width >> sx, i.coded_height >> sy);
        const int u = lr_unit_size ? lr_unit_size[k] : 0;
        if (u > 0) {
            const int w = i.upscaled_width >> sx, h = i.coded_height >> sy;
            unit_counts[k] = std::max((w + u / 2) / u, 1) * std::max((h + u / 2) / u, 1);
        }
        slot_bytes += in_bytes[k] + out_bytes[k] + align_up(sizeof(vaco_av1_lr_unit) * unit_counts[k] + 1, 256);
    }
    const size_t cells = (size_t)i.mi_rows * i.mi_cols;
    const size_t ccells = (size_t)((i.mi_rows + ssy) >> ssy) * ((i.mi_cols + ssx) >> ssx);
    const size_t nidx = (size_t)((i.mi_rows + 15) / 16) * ((i.mi_cols + 15) / 16);
    slot_bytes += align_up(cells, 256) * 2 + align_up(ccells, 256) + align_up(cells * 4, 256) + align_up(nidx * 4, 256);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->resident + slot_bytes * buffers > s->stream_budget) {
        if (msg) *msg = VACO_AV1_MSG_QUEUE_FULL;
        return VACO_AV1_LIMIT_EXCEEDED;
    }
    cudaSetDevice(s->cfg.device);
    StreamState st;
    st.open = true;
    st.info = i;
    for (int k = 0; k < 3; ++k) st.lr_unit_size[k] = k < np && lr_unit_size ? lr_unit_size[k] : 0;
    st.bytes = slot_bytes * buffers;
    // batch scratch of one frame: CDEF planes, boundary rows, superres copies
    int64_t scratch = 0;
    for (int k = 0; k < np; ++k) scratch += 3 * (int64_t)std::max(in_bytes[k], out_bytes[k]);
    st.scratch_estimate = scratch;
    auto alloc = [&](SlotBuffers& b, size_t bytes) -> void* {
        void* p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(bytes, 256)) != cudaSuccess) return nullptr;
        cudaMemset(p, 0, std::max<size_t>(bytes, 256));
        b.allocations.push_back(p);
        return p;
    };
    st.slots.resize(buffers);
    for (SlotBuffers& b : st.slots) {
        vaco_av1_frame_job& j = b.job;
        memset(&j, 0, sizeof j);
        j.info = i;
        bool ok = true;
        for (int k = 0; k < np && ok; ++k) {
            const int sx = k ? ssx : 0, sy = k ? ssy : 0;
            const int iw = (i.mi_cols * 4) >> sx, ih = (i.mi_rows * 4) >> sy;
            const int ow = i.upscaled_width >> sx, oh = i.coded_height >> sy;
            j.src.planes[k] = static_cast<uint16_t*>(alloc(b, in_bytes[k]));
            j.src.width[k] = iw;
            j.src.height[k] = ih;
            j.src.stride[k] = (int)align_up((size_t)iw, 64);
            j.dst.planes[k] = static_cast<uint16_t*>(alloc(b, out_bytes[k]));
            j.dst.width[k] = ow;
            j.dst.height[k] = oh;
            j.dst.stride[k] = (int)align_up((size_t)std::max(ow, 1), 64);
            if (unit_counts[k]) {
                j.lr_units[k] = static_cast<const vaco_av1_lr_unit*>(alloc(b, sizeof(vaco_av1_lr_unit) * unit_counts[k]));
                j.lr_unit_count[k] = unit_counts[k];
                j.lr_unit_size[k] = st.lr_unit_size[k];
            }
            ok = j.src.planes[k] && j.dst.planes[k] && (!unit_counts[k] || j.lr_units[k]);
        }
        j.tx_luma = static_cast<const uint8_t*>(alloc(b, cells));
        j.tx_chroma = static_cast<const uint8_t*>(alloc(b, std::max<size_t>(ccells, 1)));
        j.skip = static_cast<const uint8_t*>(alloc(b, cells));
        j.lvl_map = static_cast<const uint8_t*>(alloc(b, cells * 4));
        j.cdef_idx = static_cast<const int32_t*>(alloc(b, nidx * 4));
        j.cdef_stride = (i.mi_cols + 15) / 16;
        j.cdef_count = (int32_t)nidx;
        ok = ok && j.tx_luma && j.tx_chroma && j.skip && j.lvl_map && j.cdef_idx &&
             cudaEventCreateWithFlags(&b.uploaded, cudaEventDisableTiming) == cudaSuccess;
        if (!ok) {
            free_stream(st);
            if (msg) *msg = VACO_AV1_MSG_CUDA;
            return VACO_AV1_DEVICE_ERROR;
        }
    }
    s->resident += st.bytes;
    s->stats.resident_bytes = s->resident;
    int id = -1;
    for (size_t k = 0; k < s->streams.size(); ++k)
        if (!s->streams[k].open) {
            id = (int)k;
            break;
        }
    if (id < 0) {
        id = (int)s->streams.size();
        s->streams.emplace_back();
    }
    s->streams[id] = std::move(st);
    *stream_id = id;
    return VACO_AV1_OK;
}

extern "C" int32_t vaco_av1_server_close_stream(vaco_av1_server* s, int32_t id) {
    if (!s) return VACO_AV1_INVALID_DATA;
    std::unique_lock<std::mutex> lk(s->mu);
    if (id < 0 || id >= (int)s->streams.size() || !s->streams[id].open) return VACO_AV1_INVALID_DATA;
    // Wait until none of its slots is in flight: bounded polls, then
    // VACO_AV1_TIMEOUT with the stream left open (its frames still complete
    // and a later close succeeds).
    for (int waited = 0;; ++waited) {
        bool busy = false;
        for (const SlotBuffers& b : s->streams[id].slots) busy = busy || b.in_flight;
        if (!busy) break;
        if (waited >= s->wait_polls) return VACO_AV1_TIMEOUT;
        s->cv_done.wait_for(lk, std::chrono::milliseconds(1));
        if (id >= (int)s->streams.size() || !s->streams[id].open) return VACO_AV1_INVALID_DATA;
    }
    cudaSetDevice(s->cfg.device);
    s->resident -= s->streams[id].bytes;
    s->stats.resident_bytes = s->resident;
    free_stream(s->streams[id]);
    return VACO_AV1_OK;
}

extern "C" int32_t vaco_av1_server_slot(vaco_av1_server* s, int32_t id, int32_t slot, vaco_av1_frame_job* job) {
    if (!s || !job) return VACO_AV1_INVALID_DATA;
    std::lock_guard<std::mutex> lk(s->mu);
    if (id < 0 || id >= (int)s->streams.size() || !s->streams[id].open) return VACO_AV1_INVALID_DATA;
    if (slot < 0 || slot >= (int)s->streams[id].slots.size()) return VACO_AV1_INVALID_DATA;
    *job = s->streams[id].slots[slot].job;
    return VACO_AV1_OK;
}

namespace {

// Waits while slot `slot` of stream `id` is still in flight (backpressure,
// bounded) and reserves it for the caller.  `lk` holds the server mutex.
int32_t reserve_slot(vaco_av1_server* s, std::unique_lock<std::mutex>& lk, int32_t id, int32_t slot) {
    if (id < 0 || id >= (int)s->streams.size() || !s->streams[id].open) return VACO_AV1_INVALID_DATA;
    if (slot < 0 || slot >= (int)s->streams[id].slots.size()) return VACO_AV1_INVALID_DATA;
    for (int waited = 0; s->streams[id].slots[slot].in_flight; ++waited) {
        if (waited >= s->wait_polls) return VACO_AV1_TIMEOUT;
        s->cv_done.wait_for(lk, std::chrono::milliseconds(1));
        if (id >= (int)s->streams.size() || !s->streams[id].open) return VACO_AV1_INVALID_DATA;
    }
    s->streams[id].slots[slot].in_flight = true;
    return VACO_AV1_OK;
}

// Queues a reserved slot with the frame-level parameters of `params`; the
// launch that takes it first waits for `upload` when that is set.  `lk`
// holds the server mutex.
uint64_t queue_slot(vaco_av1_server* s, int32_t id, int32_t slot, const vaco_av1_frame_job* params,
                    cudaEvent_t upload) {
    StreamState& st = s->streams[id];
    Pending p;
    p.ticket = s->next_ticket++;
    p.stream = id;
    p.slot = slot;
    p.job = st.slots[slot].job;
    p.job.deblock = params->deblock;
    p.job.cdef = params->cdef;
    for (int k = 0; k < 3; ++k) {
        p.job.lr_type[k] = st.lr_unit_size[k] ? params->lr_type[k] : VACO_AV1_FRAME_LR_NONE;
        if (!p.job.lr_type[k]) {
            p.job.lr_units[k] = nullptr;
            p.job.lr_unit_count[k] = 0;
        }
    }
    if (!params->lvl_map) p.job.lvl_map = nullptr;
    p.scratch = st.scratch_estimate;
    p.submitted = Clock::now();
    p.upload = upload;
    s->tickets.emplace(p.ticket, TicketState{});
    s->pending.push_back(p);
    ++s->stats.submitted;
    s->cv_work.notify_one();
    return p.ticket;
}

// Enqueues the copies of a host frame (planes, restoration units, side
// information) into the device buffers `d` of a slot on `stream`.
cudaError_t enqueue_upload(const vaco_av1_frame_job& d, const vaco_av1_frame_job* host, cudaStream_t stream) {
    const vaco_av1_frame_info& i = d.info;
    const int np = i.monochrome ? 1 : 3;
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < np && e == cudaSuccess; ++k) {
        if (d.src.width[k] > 0 && d.src.height[k] > 0)
            e = cudaMemcpy2DAsync(d.src.planes[k], (size_t)d.src.stride[k] * 2, host->src.planes[k],
                                  (size_t)host->src.stride[k] * 2, (size_t)d.src.width[k] * 2, d.src.height[k],
                                  cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess && d.lr_units[k] && host->lr_units[k] && host->lr_unit_count[k] == d.lr_unit_count[k])
            e = cudaMemcpyAsync(const_cast<vaco_av1_lr_unit*>(d.lr_units[k]), host->lr_units[k],
                                sizeof(vaco_av1_lr_unit) * d.lr_unit_count[k], cudaMemcpyHostToDevice, stream);
    }
    const size_t cells = (size_t)i.mi_rows * i.mi_cols;
    const size_t ccells = (size_t)((i.mi_rows + i.subsampling_y) >> i.subsampling_y) *
                          ((i.mi_cols + i.subsampling_x) >> i.subsampling_x);
    auto up = [&](const void* dst, const void* src, size_t bytes) {
        if (e == cudaSuccess && src && bytes)
            e = cudaMemcpyAsync(const_cast<void*>(dst), src, bytes, cudaMemcpyHostToDevice, stream);
    };
    up(d.tx_luma, host->tx_luma, cells);
    if (np > 1) up(d.tx_chroma, host->tx_chroma, ccells);
    up(d.skip, host->skip, cells);
    up(d.lvl_map, host->lvl_map, cells * 4);
    if (host->cdef_idx && host->cdef_count == d.cdef_count)
        up(d.cdef_idx, host->cdef_idx, sizeof(int32_t) * d.cdef_count);
    return e;
}

// A host frame must match the slot's geometry and carry every plane.
bool host_frame_fits(const vaco_av1_frame_job& d, const vaco_av1_frame_job* host) {
    const vaco_av1_frame_info& i = d.info;
    if (host->info.mi_rows != i.mi_rows || host->info.mi_cols != i.mi_cols || host->info.bit_depth != i.bit_depth)
        return false;
    const int np = i.monochrome ? 1 : 3;
    for (int k = 0; k < np; ++k)
        if (!host->src.planes[k] || host->src.stride[k] < d.src.width[k]) return false;
    return true;
}

}  // namespace

extern "C" int32_t vaco_av1_server_submit(vaco_av1_server* s, int32_t id, int32_t slot, const vaco_av1_frame_job* params,
                                          uint64_t* ticket) {
    if (!s || !params || !ticket) return VACO_AV1_INVALID_DATA;
    std::unique_lock<std::mutex> lk(s->mu);
    const int32_t st = reserve_slot(s, lk, id, slot);
    if (st != VACO_AV1_OK) return st;
    *ticket = queue_slot(s, id, slot, params, nullptr);
    return VACO_AV1_OK;
}

extern "C" int32_t vaco_av1_server_submit_host(vaco_av1_server* s, int32_t id, int32_t slot,
                                               const vaco_av1_frame_job* host, uint64_t* ticket) {
    if (!s || !host || !ticket) return VACO_AV1_INVALID_DATA;
    std::unique_lock<std::mutex> lk(s->mu);
    int32_t st = reserve_slot(s, lk, id, slot);
    if (st != VACO_AV1_OK) return st;
    const vaco_av1_frame_job d = s->streams[id].slots[slot].job;
    const cudaEvent_t ev = s->streams[id].slots[slot].uploaded;
    if (!host_frame_fits(d, host)) {
        s->streams[id].slots[slot].in_flight = false;
        s->cv_done.notify_all();
        return VACO_AV1_INVALID_DATA;
    }
    // The reserved slot keeps close_stream and other submits away while the
    // copies are enqueued without the lock.
    lk.unlock();
    cudaSetDevice(s->cfg.device);
    const cudaStream_t us = s->upload_streams[(id + slot) % vaco_av1_server::kUploadStreams];
    cudaError_t e = enqueue_upload(d, host, us);
    if (e == cudaSuccess) e = cudaEventRecord(ev, us);
    lk.lock();
    if (e != cudaSuccess) {
        s->streams[id].slots[slot].in_flight = false;
        s->cv_done.notify_all();
        return VACO_AV1_DEVICE_ERROR;
    }
    *ticket = queue_slot(s, id, slot, host, ev);
    return VACO_AV1_OK;
}

extern "C" int32_t vaco_av1_server_wait(vaco_av1_server* s, uint64_t ticket, int32_t timeout_ms, int32_t* msg,
                                        double* latency_ms) {
    if (!s) return VACO_AV1_INVALID_DATA;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return VACO_AV1_INVALID_DATA;
    auto ready = [&] { return s->tickets[ticket].done; };
    if (timeout_ms < 0) {
        while (!ready()) s->cv_done.wait_for(lk, std::chrono::milliseconds(10));
    } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
        if (msg) *msg = VACO_AV1_MSG_TIMEOUT;
        return VACO_AV1_TIMEOUT;
    }
    const TicketState t = s->tickets[ticket];
    s->tickets.erase(ticket);
    if (msg) *msg = t.msg;
    if (latency_ms) *latency_ms = t.latency_ms;
    return t.status;
}

extern "C" int32_t vaco_av1_server_get_stats(vaco_av1_server* s, vaco_av1_server_stats* stats) {
    if (!s || !stats) return VACO_AV1_INVALID_DATA;
    std::lock_guard<std::mutex> lk(s->mu);
    *stats = s->stats;
    return VACO_AV1_OK;
}

namespace {

// Copies one plane between a host picture (pitch in samples) and a device plane.
cudaError_t copy_plane(void* dst, size_t dpitch, const void* src, size_t spitch, int w, int h, cudaMemcpyKind kind) {
    if (w <= 0 || h <= 0) return cudaSuccess;
    return cudaMemcpy2D(dst, dpitch * 2, src, spitch * 2, (size_t)w * 2, h, kind);
}

}  // namespace

extern "C" int32_t vaco_av1_server_upload(vaco_av1_server* s, int32_t id, int32_t slot, const vaco_av1_frame_job* host) {
    if (!s || !host) return VACO_AV1_INVALID_DATA;
    vaco_av1_frame_job d;
    if (vaco_av1_server_slot(s, id, slot, &d) != VACO_AV1_OK) return VACO_AV1_INVALID_DATA;
    if (!host_frame_fits(d, host)) return VACO_AV1_INVALID_DATA;
    cudaSetDevice(s->cfg.device);
    cudaError_t e = enqueue_upload(d, host, s->upload_streams[0]);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->upload_streams[0]);
    return e == cudaSuccess ? VACO_AV1_OK : VACO_AV1_DEVICE_ERROR;
}

extern "C" int32_t vaco_av1_server_download(vaco_av1_server* s, int32_t id, int32_t slot, const vaco_av1_picture* host) {
    if (!s || !host) return VACO_AV1_INVALID_DATA;
    vaco_av1_frame_job d;
    if (vaco_av1_server_slot(s, id, slot, &d) != VACO_AV1_OK) return VACO_AV1_INVALID_DATA;
    cudaSetDevice(s->cfg.device);
    const int np = d.info.monochrome ? 1 : 3;
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < np && e == cudaSuccess; ++k) {
        if (!host->planes[k] || host->width[k] != d.dst.width[k] || host->height[k] != d.dst.height[k])
            return VACO_AV1_INVALID_DATA;
        e = copy_plane(host->planes[k], host->stride[k], d.dst.planes[k], d.dst.stride[k], d.dst.width[k],
                       d.dst.height[k], cudaMemcpyDeviceToHost);
    }
    return e == cudaSuccess ? VACO_AV1_OK : VACO_AV1_DEVICE_ERROR;
}

extern "C" int32_t vaco_av1_server_submit_many(vaco_av1_server* s, int32_t n, const int32_t* stream_ids,
                                               const int32_t* slots, const vaco_av1_frame_job* params,
                                               uint64_t* tickets) {
    if (!s || n < 0 || (n > 0 && (!stream_ids || !slots || !params || !tickets))) return VACO_AV1_INVALID_DATA;
    for (int32_t i = 0; i < n; ++i) {
        const int32_t st = vaco_av1_server_submit(s, stream_ids[i], slots[i], params + i, tickets + i);
        if (st != VACO_AV1_OK) return st;
    }
    return VACO_AV1_OK;
}

extern "C" int32_t vaco_av1_server_wait_many(vaco_av1_server* s, int32_t n, const uint64_t* tickets,
                                             int32_t timeout_ms, int32_t* statuses, int32_t* msgs,
                                             double* latency_ms) {
    if (!s || n < 0 || (n > 0 && !tickets)) return VACO_AV1_INVALID_DATA;
    int32_t first = VACO_AV1_OK;
    for (int32_t i = 0; i < n; ++i) {
        int32_t msg = 0;
        double lat = 0;
        const int32_t st = vaco_av1_server_wait(s, tickets[i], timeout_ms, &msg, &lat);
        if (statuses) statuses[i] = st;
        if (msgs) msgs[i] = msg;
        if (latency_ms) latency_ms[i] = lat;
        if (first == VACO_AV1_OK && st != VACO_AV1_OK) first = st;
    }
    return first;
}
