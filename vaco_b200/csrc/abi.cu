// abi.cu -- the C ABI of include/vaco_av1_gpu.h.
//
// Host-side argument checks reproduce vaco's own validation order; data
// checks run on the device and land in the context's status word (see
// common.cuh).  A status word key orders errors by (stage, position), so a
// host-detected problem in a later stage never hides a device-detected one
// in an earlier stage: host errors are folded into the same ordering.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>

#include "common.cuh"
#include "ctx.cuh"
#include "kernels.cuh"

using namespace vaco;

namespace {

const char* const kMessages[VACO_AV1_MSG_COUNT] = {
    "",
    "CDEF bit depth must be 8, 10, or 12",
    "CDEF sample exceeds bit depth",
    "invalid CDEF block parameters",
    "CDEF strength index exceeds table",
    "AV1 superres bit depth must be 8, 10, or 12",
    "invalid AV1 superres plane geometry",
    "AV1 superres sample exceeds bit depth",
    "AV1 restoration plane geometry or bit depth",
    "AV1 restoration unit count",
    "AV1 restoration coefficient out of range",
    "AV1 restoration sample exceeds bit depth",
    "AV1 active restoration has no unit size",
    "invalid AV1 deblocking parameters",
    "AV1 deblocking sample exceeds bit depth",
    "AV1 frame geometry does not match its pictures",
    "required argument is NULL",
    "CUDA runtime error",
    "request exceeds the fixed scratch size",
    "job admission refused: queue or memory budget full",
    "bounded device wait timed out",
    "vaco-codec-av1: unsupported pixel format",
    "invalid AV1 film grain parameters",
    "AV1 film grain sample exceeds bit depth",
    "AV1 superres missing U plane",
    "AV1 superres missing V plane",
};

unsigned long long make_key(unsigned stage, unsigned long long position, unsigned msg) {
    return ((unsigned long long)stage << 60) | ((position & ((1ull << 52) - 1)) << 8) | msg;
}

// LR key positions: plane, then the check vaco's restore_plane runs first.
enum LrCheck : unsigned { LR_NO_UNIT_SIZE = 0, LR_GEOM = 1, LR_COUNT = 2, LR_COEFF = 3, LR_SAMPLE = 4 };
unsigned long long lr_position(int plane, unsigned check, unsigned long long index) {
    return ((unsigned long long)plane << 44) | ((unsigned long long)check << 40) | index;
}

bool bd_valid(int bd) { return bd == 8 || bd == 10 || bd == 12; }


}  // namespace

namespace {

int32_t set_msg(int32_t* msg, int m) {
    if (msg) *msg = m;
    return m;
}

int32_t cuda_fail(vaco_av1_ctx* ctx, cudaError_t e, int32_t* msg) {
    if (ctx) ctx->last_cuda_error = (int)e;
    set_msg(msg, VACO_AV1_MSG_CUDA);
    return VACO_AV1_DEVICE_ERROR;
}

int32_t invalid(int32_t* msg, int m) {
    set_msg(msg, m);
    return m == VACO_AV1_MSG_NULL_ARGUMENT || m == VACO_AV1_MSG_FRAME_GEOMETRY ? VACO_AV1_INVALID_DATA
                                                                                : VACO_AV1_INVALID_DATA;
}

cudaError_t reset_status(vaco_av1_ctx* ctx, cudaStream_t s) {
    return cudaMemsetAsync(ctx->status, 0xFF, sizeof(DeviceStatus), s);
}

// Read the status word back (one small D2H copy + stream sync) and fold in
// the earliest host-detected error `host_key`.
int32_t finish(vaco_av1_ctx* ctx, cudaStream_t s, unsigned long long host_key, int32_t* msg) {
    cudaError_t e = cudaMemcpyAsync(ctx->status_host, ctx->status, sizeof(unsigned long long),
                                    cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    ctx->collect_marks();
    unsigned long long key = *ctx->status_host;
    if (host_key < key) key = host_key;
    if (key == kNoError) {
        set_msg(msg, VACO_AV1_MSG_NONE);
        return VACO_AV1_OK;
    }
    set_msg(msg, (int)(key & 0xFF));
    return VACO_AV1_INVALID_DATA;
}

DevPlaneC cplane(const vaco_av1_picture& p, int k) {
    return DevPlaneC{p.planes[k], p.width[k], p.height[k], p.stride[k]};
}
DevPlane mplane(const vaco_av1_picture& p, int k) {
    return DevPlane{p.planes[k], p.width[k], p.height[k], p.stride[k]};
}

// Reconstruction picture extents: luma mi_cols*4 x mi_rows*4, chroma >> ss.
bool padded_picture_ok(const vaco_av1_picture* p, const vaco_av1_frame_info* info) {
    if (!p) return false;
    int np = info->monochrome ? 1 : 3;
    for (int k = 0; k < np; ++k) {
        int sx = k ? info->subsampling_x : 0, sy = k ? info->subsampling_y : 0;
        if (!p->planes[k]) return false;
        if (p->width[k] != (info->mi_cols * 4) >> sx || p->height[k] != (info->mi_rows * 4) >> sy) return false;
        if (p->stride[k] < p->width[k]) return false;
    }
    return true;
}

bool info_ok(const vaco_av1_frame_info* info) {
    if (!info) return false;
    if (info->mi_rows <= 0 || info->mi_cols <= 0 || info->mi_rows > (1 << 15) || info->mi_cols > (1 << 15))
        return false;
    if (info->subsampling_x < 0 || info->subsampling_x > 1 || info->subsampling_y < 0 || info->subsampling_y > 1)
        return false;
    return true;
}

// Copy a host picture into device scratch (pitch = width rounded to 64).
bool stage_picture_in(vaco_av1_ctx* ctx, const vaco_av1_picture* host, int np, int first_slot,
                      vaco_av1_picture* dev, cudaStream_t s, cudaError_t* err) {
    *dev = vaco_av1_picture{};
    for (int k = 0; k < np; ++k) {
        int w = host->width[k], h = host->height[k];
        int pitch = (int)align_up((size_t)(w > 0 ? w : 1), 64);
        void* d = ctx->scratch(first_slot + k, (size_t)pitch * (h > 0 ? h : 1) * 2);
        if (!d) {
            *err = cudaErrorMemoryAllocation;
            return false;
        }
        dev->planes[k] = (uint16_t*)d;
        dev->width[k] = w;
        dev->height[k] = h;
        dev->stride[k] = pitch;
        if (w > 0 && h > 0 && host->planes[k]) {
            *err = cudaMemcpy2DAsync(d, (size_t)pitch * 2, host->planes[k], (size_t)host->stride[k] * 2,
                                     (size_t)w * 2, h, cudaMemcpyHostToDevice, s);
            if (*err != cudaSuccess) return false;
        }
    }
    return true;
}

bool alloc_picture(vaco_av1_ctx* ctx, const vaco_av1_picture* like, int np, int first_slot, vaco_av1_picture* dev,
                   cudaError_t* err) {
    *dev = vaco_av1_picture{};
    for (int k = 0; k < np; ++k) {
        int w = like->width[k], h = like->height[k];
        int pitch = (int)align_up((size_t)(w > 0 ? w : 1), 64);
        void* d = ctx->scratch(first_slot + k, (size_t)pitch * (h > 0 ? h : 1) * 2);
        if (!d) {
            *err = cudaErrorMemoryAllocation;
            return false;
        }
        dev->planes[k] = (uint16_t*)d;
        dev->width[k] = w;
        dev->height[k] = h;
        dev->stride[k] = pitch;
    }
    return true;
}

cudaError_t copy_picture_out(const vaco_av1_picture* dev, const vaco_av1_picture* host, int np, cudaStream_t s) {
    for (int k = 0; k < np; ++k) {
        int w = host->width[k], h = host->height[k];
        if (w <= 0 || h <= 0) continue;
        cudaError_t e = cudaMemcpy2DAsync(host->planes[k], (size_t)host->stride[k] * 2, dev->planes[k],
                                          (size_t)dev->stride[k] * 2, (size_t)w * 2, h, cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <class T>
const T* stage_array(vaco_av1_ctx* ctx, int slot, const T* host, size_t count, cudaStream_t s, cudaError_t* err) {
    if (!host || count == 0) return nullptr;
    void* d = ctx->scratch(slot, count * sizeof(T));
    if (!d) {
        *err = cudaErrorMemoryAllocation;
        return nullptr;
    }
    *err = cudaMemcpyAsync(d, host, count * sizeof(T), cudaMemcpyHostToDevice, s);
    return (const T*)d;
}

// ---------------------------------------------------------------- stage runners (device pointers)

// Deblocking: src -> dst (copy + checks + both passes).  Returns host key.
unsigned long long run_deblock(vaco_av1_ctx* ctx, cudaStream_t s, const vaco_av1_picture& src,
                               const vaco_av1_picture& dst, const vaco_av1_frame_info& info, const uint8_t* tx_luma,
                               const uint8_t* tx_chroma, const uint8_t* lvl_map,
                               const vaco_av1_deblock_params& params, cudaError_t* err) {
    const int np = info.monochrome ? 1 : 3;
    bool params_ok = bd_valid(info.bit_depth) && params.sharpness <= 7;
    for (int k = 0; k < 4; ++k) params_ok = params_ok && params.levels[k] <= 63;
    if (!params_ok || !tx_luma || (np > 1 && !tx_chroma)) {
        return make_key(STAGE_DEBLOCK, 0, params_ok ? VACO_AV1_MSG_NULL_ARGUMENT : VACO_AV1_MSG_DB_PARAMS);
    }
    DevPlaneC sp[3];
    DevPlane dp[3];
    for (int k = 0; k < np; ++k) {
        sp[k] = cplane(src, k);
        dp[k] = mplane(dst, k);
    }
    const int ssx = info.subsampling_x, ssy = info.subsampling_y;
    long n_luma = (long)info.mi_rows * info.mi_cols;
    long n_chroma = np > 1 ? (long)((info.mi_rows + ssy) >> ssy) * ((info.mi_cols + ssx) >> ssx) : 0;
    *err = launch_deblock_prepare(sp, dp, np, info.bit_depth, tx_luma, n_luma, tx_chroma, n_chroma, lvl_map,
                                  ctx->status, s);
    ctx->launches += 1 + np;
    if (*err != cudaSuccess) return kNoError;
    DeblockLaunch L;
    for (int k = 0; k < 3; ++k) L.pic[k] = k < np ? dp[k] : DevPlane{nullptr, 0, 0, 0};
    L.num_planes = np;
    L.ssx = ssx;
    L.ssy = ssy;
    L.bit_depth = info.bit_depth;
    L.mi_rows = info.mi_rows;
    L.mi_cols = info.mi_cols;
    L.coded_width = info.coded_width;
    L.coded_height = info.coded_height;
    L.tx_luma = tx_luma;
    L.tx_chroma = tx_chroma;
    L.lvl_map = lvl_map;
    for (int k = 0; k < 4; ++k) L.levels[k] = params.levels[k];
    L.sharpness = params.sharpness;
    *err = launch_deblock_passes(L, s);
    if (!(params.levels[0] == 0 && params.levels[1] == 0)) ctx->launches += 2;
    return kNoError;
}

unsigned long long run_cdef(vaco_av1_ctx* ctx, cudaStream_t s, const vaco_av1_picture& src,
                            const vaco_av1_picture& dst, const vaco_av1_frame_info& info, const uint8_t* skip,
                            const int32_t* cdef_idx, int cdef_stride, int cdef_count,
                            const vaco_av1_cdef_params& params, cudaError_t* err) {
    const int np = info.monochrome ? 1 : 3;
    bool all_zero = true;
    for (int k = 0; k < 8; ++k)
        all_zero = all_zero && params.y_primary[k] == 0 && params.y_secondary[k] == 0 && params.uv_primary[k] == 0 &&
                   params.uv_secondary[k] == 0;
    if (!params.enabled || all_zero) {
        // apply_cdef returns before touching the picture (decode.rs:741-748).
        for (int k = 0; k < np; ++k) {
            *err = cudaMemcpy2DAsync(dst.planes[k], (size_t)dst.stride[k] * 2, src.planes[k],
                                     (size_t)src.stride[k] * 2, (size_t)src.width[k] * 2, src.height[k],
                                     cudaMemcpyDeviceToDevice, s);
            if (*err != cudaSuccess) return kNoError;
        }
        return kNoError;
    }
    if (!skip || (!cdef_idx && cdef_count > 0)) return make_key(STAGE_CDEF, 0, VACO_AV1_MSG_NULL_ARGUMENT);
    CdefLaunch L;
    L.src = src;
    L.dst = dst;
    L.info = info;
    L.skip = skip;
    L.cdef_idx = cdef_idx;
    L.cdef_stride = cdef_stride;
    L.cdef_count = cdef_idx ? cdef_count : 0;
    L.params = params;
    L.status = ctx->status;
    *err = launch_cdef_frame(L, s);
    ctx->launches += 1;
    return kNoError;
}

}  // namespace

// ======================================================================= C ABI

extern "C" {

const char* vaco_av1_message(int32_t msg) {
    if (msg < 0 || msg >= VACO_AV1_MSG_COUNT) return "";
    return kMessages[msg];
}

int32_t vaco_av1_ctx_create(int32_t device, vaco_av1_ctx** out) {
    if (!out) return VACO_AV1_INVALID_DATA;
    *out = nullptr;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return VACO_AV1_DEVICE_ERROR;
    vaco_av1_ctx* c = new (std::nothrow) vaco_av1_ctx();
    if (!c) return VACO_AV1_DEVICE_ERROR;
    c->device = device;
    e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&c->status, sizeof(DeviceStatus));
    if (e == cudaSuccess) e = cudaMallocHost(&c->status_host, sizeof(unsigned long long));
    if (e != cudaSuccess) {
        vaco_av1_ctx_destroy(c);
        return VACO_AV1_DEVICE_ERROR;
    }
    *out = c;
    return VACO_AV1_OK;
}

void vaco_av1_ctx_destroy(vaco_av1_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto& slot : ctx->pipe)
        if (slot.done) cudaEventSynchronize(slot.done);
    for (auto& set : ctx->bufs)
        for (auto& b : set)
            if (b.p) cudaFree(b.p);
    for (auto& slot : ctx->pipe) {
        for (cudaEvent_t ev : {slot.staged, slot.filtered, slot.done})
            if (ev) cudaEventDestroy(ev);
        if (slot.status) cudaFree(slot.status);
        if (slot.status_host) cudaFreeHost(slot.status_host);
    }
    for (auto& g : ctx->grain) {
        if (g.stream) cudaStreamSynchronize(g.stream);
        for (cudaEvent_t ev : {g.ready, g.free})
            if (ev) cudaEventDestroy(ev);
        if (g.stream) cudaStreamDestroy(g.stream);
    }
    if (ctx->copy_in) cudaStreamDestroy(ctx->copy_in);
    if (ctx->copy_out) cudaStreamDestroy(ctx->copy_out);
    if (ctx->status) cudaFree(ctx->status);
    if (ctx->status_host) cudaFreeHost(ctx->status_host);
    for (auto& frame : ctx->marks)
        for (auto& ev : frame)
            if (ev) cudaEventDestroy(ev);
    for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.second);
    if (ctx->batch_table_host) cudaFreeHost(ctx->batch_table_host);
    if (ctx->batch_status_host) cudaFreeHost(ctx->batch_status_host);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

int32_t vaco_av1_ctx_last_cuda_error(const vaco_av1_ctx* ctx) { return ctx ? ctx->last_cuda_error : 0; }
uint64_t vaco_av1_ctx_launch_count(const vaco_av1_ctx* ctx) { return ctx ? ctx->launches : 0; }

int32_t vaco_av1_ctx_set_deferred_status(vaco_av1_ctx* ctx, int32_t enable) {
    if (!ctx) return VACO_AV1_INVALID_DATA;
    cudaSetDevice(ctx->device);
    // Start from a clean word; the caller has no work of this context in flight.
    if (cudaDeviceSynchronize() != cudaSuccess || cudaMemset(ctx->status, 0xFF, sizeof(DeviceStatus)) != cudaSuccess)
        return VACO_AV1_DEVICE_ERROR;
    ctx->deferred = enable != 0;
    return VACO_AV1_OK;
}

int32_t vaco_av1_ctx_flush(vaco_av1_ctx* ctx, void* stream, int32_t* msg) {
    if (!ctx) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    cudaSetDevice(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    const int32_t st = finish(ctx, s, kNoError, msg);
    if (st == VACO_AV1_DEVICE_ERROR) return st;
    cudaError_t e = reset_status(ctx, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    return st;
}

int32_t vaco_av1_ctx_set_stage_timing(vaco_av1_ctx* ctx, int32_t enable) {
    if (!ctx) return VACO_AV1_INVALID_DATA;
    cudaSetDevice(ctx->device);
    if (enable) {
        for (auto& frame : ctx->marks)
            for (auto& ev : frame)
                if (!ev && cudaEventCreate(&ev) != cudaSuccess) return VACO_AV1_DEVICE_ERROR;
    }
    // Frames still being timed are dropped: wait for them before the reset.
    if (ctx->mark_head != ctx->mark_tail) cudaDeviceSynchronize();
    ctx->timing = enable > 0;
    ctx->timing_every = enable > 0 ? enable : 1;
    ctx->timing_count = 0;
    ctx->mark_head = ctx->mark_tail = 0;
    for (double& v : ctx->stage_ms) v = 0;
    ctx->timed_frames = 0;
    return VACO_AV1_OK;
}

int32_t vaco_av1_ctx_stage_ms(const vaco_av1_ctx* ctx, double* ms4, uint64_t* frames) {
    if (!ctx) return VACO_AV1_INVALID_DATA;
    if (ms4)
        for (int i = 0; i < 4; ++i) ms4[i] = ctx->stage_ms[i];
    if (frames) *frames = ctx->timed_frames;
    return VACO_AV1_OK;
}

// ---------------------------------------------------------------- CDEF block API

int32_t vaco_av1_cdef_find_direction_dev(vaco_av1_ctx* ctx, void* stream, const uint16_t* blocks, int32_t n,
                                         int32_t bit_depth, uint8_t* directions, uint32_t* variances,
                                         int32_t* msg) {
    if (!ctx || (n > 0 && (!blocks || !directions || !variances))) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    cudaStream_t s = (cudaStream_t)stream;
    cudaSetDevice(ctx->device);
    cudaError_t e = reset_status(ctx, s);
    if (e == cudaSuccess && n > 0) {
        e = launch_find_direction(blocks, n, bit_depth, directions, variances, ctx->status, s);
        ctx->launches++;
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    return finish(ctx, s, kNoError, msg);
}

int32_t vaco_av1_cdef_find_direction_host(vaco_av1_ctx* ctx, const uint16_t* blocks, int32_t n, int32_t bit_depth,
                                          uint8_t* directions, uint32_t* variances, int32_t* msg) {
    if (!ctx || (n > 0 && (!blocks || !directions || !variances))) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    if (n <= 0) return vaco_av1_cdef_find_direction_dev(ctx, ctx->stream, nullptr, 0, bit_depth, nullptr, nullptr, msg);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaSuccess;
    const uint16_t* d_in = stage_array(ctx, S_H_IN0, blocks, (size_t)n * 64, s, &e);
    uint8_t* d_dir = (uint8_t*)ctx->scratch(S_H_OUT0, (size_t)n);
    uint32_t* d_var = (uint32_t*)ctx->scratch(S_H_OUT1, (size_t)n * 4);
    if (e != cudaSuccess || !d_in || !d_dir || !d_var) return cuda_fail(ctx, e ? e : cudaErrorMemoryAllocation, msg);
    int32_t st = vaco_av1_cdef_find_direction_dev(ctx, s, d_in, n, bit_depth, d_dir, d_var, msg);
    if (st != VACO_AV1_OK) return st;
    e = cudaMemcpyAsync(directions, d_dir, (size_t)n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(variances, d_var, (size_t)n * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    return VACO_AV1_OK;
}

int32_t vaco_av1_cdef_filter_block_dev(vaco_av1_ctx* ctx, void* stream, const uint16_t* inputs,
                                       const vaco_av1_cdef_filter_params* params, int32_t n, uint16_t* outputs,
                                       int32_t* msg) {
    if (!ctx || (n > 0 && (!inputs || !params || !outputs))) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    cudaStream_t s = (cudaStream_t)stream;
    cudaSetDevice(ctx->device);
    cudaError_t e = reset_status(ctx, s);
    if (e == cudaSuccess && n > 0) {
        e = launch_filter_block(inputs, params, n, outputs, ctx->status, s);
        ctx->launches++;
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    return finish(ctx, s, kNoError, msg);
}

int32_t vaco_av1_cdef_filter_block_host(vaco_av1_ctx* ctx, const uint16_t* inputs,
                                        const vaco_av1_cdef_filter_params* params, int32_t n, uint16_t* outputs,
                                        int32_t* msg) {
    if (!ctx || (n > 0 && (!inputs || !params || !outputs))) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    if (n <= 0) return vaco_av1_cdef_filter_block_dev(ctx, ctx->stream, nullptr, nullptr, 0, nullptr, msg);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaSuccess;
    const uint16_t* d_in = stage_array(ctx, S_H_IN0, inputs, (size_t)n * 144, s, &e);
    const vaco_av1_cdef_filter_params* d_p = e == cudaSuccess ? stage_array(ctx, S_H_IN1, params, (size_t)n, s, &e)
                                                             : nullptr;
    uint16_t* d_out = (uint16_t*)ctx->scratch(S_H_OUT0, (size_t)n * 64 * 2);
    if (e != cudaSuccess || !d_in || !d_p || !d_out) return cuda_fail(ctx, e ? e : cudaErrorMemoryAllocation, msg);
    int32_t st = vaco_av1_cdef_filter_block_dev(ctx, s, d_in, d_p, n, d_out, msg);
    if (st != VACO_AV1_OK) return st;
    e = cudaMemcpyAsync(outputs, d_out, (size_t)n * 64 * 2, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    return VACO_AV1_OK;
}

// ---------------------------------------------------------------- CDEF frame

int32_t vaco_av1_cdef_picture_dev(vaco_av1_ctx* ctx, void* stream, const vaco_av1_picture* src,
                                  const vaco_av1_picture* dst, const vaco_av1_frame_info* info, const uint8_t* skip,
                                  const int32_t* cdef_idx, int32_t cdef_stride, int32_t cdef_count,
                                  const vaco_av1_cdef_params* params, int32_t* msg) {
    if (!ctx || !src || !dst || !info || !params) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    if (!info_ok(info) || !padded_picture_ok(src, info) || !padded_picture_ok(dst, info))
        return invalid(msg, VACO_AV1_MSG_FRAME_GEOMETRY);
    cudaStream_t s = (cudaStream_t)stream;
    cudaSetDevice(ctx->device);
    cudaError_t e = reset_status(ctx, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    unsigned long long hk = run_cdef(ctx, s, *src, *dst, *info, skip, cdef_idx, cdef_stride, cdef_count, *params, &e);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    return finish(ctx, s, hk, msg);
}

int32_t vaco_av1_cdef_picture_host(vaco_av1_ctx* ctx, const vaco_av1_picture* src, const vaco_av1_picture* dst,
                                   const vaco_av1_frame_info* info, const uint8_t* skip, const int32_t* cdef_idx,
                                   int32_t cdef_stride, int32_t cdef_count, const vaco_av1_cdef_params* params,
                                   int32_t* msg) {
    if (!ctx || !src || !dst || !info || !params) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    if (!info_ok(info) || !padded_picture_ok(src, info) || !padded_picture_ok(dst, info))
        return invalid(msg, VACO_AV1_MSG_FRAME_GEOMETRY);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const int np = info->monochrome ? 1 : 3;
    cudaError_t e = cudaSuccess;
    vaco_av1_picture dsrc, ddst;
    if (!stage_picture_in(ctx, src, np, S_H_IN0, &dsrc, s, &e)) return cuda_fail(ctx, e, msg);
    if (!alloc_picture(ctx, dst, np, S_H_OUT0, &ddst, &e)) return cuda_fail(ctx, e, msg);
    const uint8_t* d_skip = stage_array(ctx, S_H_SIDE0, skip, (size_t)info->mi_rows * info->mi_cols, s, &e);
    const int32_t* d_idx =
        e == cudaSuccess ? stage_array(ctx, S_H_SIDE1, cdef_idx, (size_t)(cdef_count > 0 ? cdef_count : 0), s, &e)
                         : nullptr;
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    int32_t st = vaco_av1_cdef_picture_dev(ctx, s, &dsrc, &ddst, info, d_skip, d_idx, cdef_stride, cdef_count, params,
                                           msg);
    if (st != VACO_AV1_OK) return st;
    e = copy_picture_out(&ddst, dst, np, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    return VACO_AV1_OK;
}

// ---------------------------------------------------------------- superres

int32_t vaco_av1_superres_upscale_plane_dev(vaco_av1_ctx* ctx, void* stream, const uint16_t* input,
                                            int32_t in_width, int32_t in_height, int32_t in_stride,
                                            int32_t visible_width, int32_t output_width, int32_t height,
                                            int32_t bit_depth, uint16_t* output, int32_t out_stride,
                                            int32_t* msg) {
    if (!ctx) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    // validate (superres.rs:128-143)
    if (!bd_valid(bit_depth)) return invalid(msg, VACO_AV1_MSG_SR_BIT_DEPTH);
    if (visible_width <= 0 || output_width <= visible_width || height <= 0 || visible_width > in_width ||
        height > in_height)
        return invalid(msg, VACO_AV1_MSG_SR_GEOMETRY);
    if (!input || !output) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    if (in_stride < in_width || out_stride < output_width) return invalid(msg, VACO_AV1_MSG_FRAME_GEOMETRY);
    cudaStream_t s = (cudaStream_t)stream;
    cudaSetDevice(ctx->device);
    cudaError_t e = reset_status(ctx, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    SuperresPlane p;
    p.in = DevPlaneC{input, in_width, in_height, in_stride};
    p.out = DevPlane{output, output_width, height, out_stride};
    p.visible_width = visible_width;
    p.output_width = output_width;
    p.height = height;
    e = launch_superres(&p, 1, bit_depth, ctx->status, STAGE_SUPERRES, s);
    ctx->launches++;
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    return finish(ctx, s, kNoError, msg);
}

int32_t vaco_av1_superres_upscale_plane_host(vaco_av1_ctx* ctx, const uint16_t* input, int32_t in_width,
                                             int32_t in_height, int32_t visible_width, int32_t output_width,
                                             int32_t height, int32_t bit_depth, uint16_t* output, int32_t* msg) {
    if (!ctx) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    if (!bd_valid(bit_depth)) return invalid(msg, VACO_AV1_MSG_SR_BIT_DEPTH);
    if (visible_width <= 0 || output_width <= visible_width || height <= 0 || visible_width > in_width ||
        height > in_height)
        return invalid(msg, VACO_AV1_MSG_SR_GEOMETRY);
    if (!input || !output) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaSuccess;
    vaco_av1_picture hin{}, din, hout{}, dout;
    hin.planes[0] = const_cast<uint16_t*>(input);
    hin.width[0] = in_width;
    hin.height[0] = in_height;
    hin.stride[0] = in_width;
    hout.planes[0] = output;
    hout.width[0] = output_width;
    hout.height[0] = height;
    hout.stride[0] = output_width;
    if (!stage_picture_in(ctx, &hin, 1, S_H_IN0, &din, s, &e)) return cuda_fail(ctx, e, msg);
    if (!alloc_picture(ctx, &hout, 1, S_H_OUT0, &dout, &e)) return cuda_fail(ctx, e, msg);
    int32_t st = vaco_av1_superres_upscale_plane_dev(ctx, s, din.planes[0], in_width, in_height, din.stride[0],
                                                     visible_width, output_width, height, bit_depth, dout.planes[0],
                                                     dout.stride[0], msg);
    if (st != VACO_AV1_OK) return st;
    e = copy_picture_out(&dout, &hout, 1, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    return VACO_AV1_OK;
}

// superres::upscale_picture (src/superres.rs:226-274).  vaco runs
// upscale_plane on Y, then U, then V, so a plane's validation failure only
// surfaces when every earlier plane filtered cleanly.  The planes before the
// first failing one run in one launch; the failure becomes a host key at the
// largest superres position, which any sample error of those planes beats.
int32_t vaco_av1_superres_upscale_picture_dev(vaco_av1_ctx* ctx, void* stream, const vaco_av1_picture* in,
                                              const vaco_av1_picture* out,
                                              const vaco_av1_superres_picture_config* cfg, int32_t* msg) {
    if (!ctx || !in || !out || !cfg) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    if (cfg->subsampling_x < 0 || cfg->subsampling_x > 1 || cfg->subsampling_y < 0 || cfg->subsampling_y > 1)
        return invalid(msg, VACO_AV1_MSG_FRAME_GEOMETRY);
    const int np = cfg->monochrome ? 1 : 3;
    SuperresPlane sp[3];
    int nsp = 0;
    unsigned long long host_key = kNoError;
    for (int k = 0; k < np; ++k) {
        const int sx = k ? cfg->subsampling_x : 0, sy = k ? cfg->subsampling_y : 0;
        // div_ceil on non-negative extents (src/superres.rs:247-250)
        const int vis = cfg->coded_width < 0 ? cfg->coded_width : (cfg->coded_width + (1 << sx) - 1) >> sx;
        const int outw = cfg->upscaled_width < 0 ? cfg->upscaled_width : (cfg->upscaled_width + (1 << sx) - 1) >> sx;
        const int h = cfg->coded_height < 0 ? cfg->coded_height : (cfg->coded_height + (1 << sy) - 1) >> sy;
        int m = VACO_AV1_MSG_NONE;
        if (k > 0 && !in->planes[k])
            m = k == 1 ? VACO_AV1_MSG_SR_MISSING_U : VACO_AV1_MSG_SR_MISSING_V;
        else if (!bd_valid(cfg->bit_depth))
            m = VACO_AV1_MSG_SR_BIT_DEPTH;
        else if (vis <= 0 || outw <= vis || h <= 0 || vis > in->width[k] || h > in->height[k])
            m = VACO_AV1_MSG_SR_GEOMETRY;
        if (m != VACO_AV1_MSG_NONE) {
            host_key = make_key(STAGE_SUPERRES, (1ull << 52) - 1, m);
            break;
        }
        if (!in->planes[k] || !out->planes[k]) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
        if (in->stride[k] < in->width[k] || out->width[k] != outw || out->height[k] != h ||
            out->stride[k] < out->width[k])
            return invalid(msg, VACO_AV1_MSG_FRAME_GEOMETRY);
        SuperresPlane& p = sp[nsp++];
        p.in = cplane(*in, k);
        p.out = DevPlane{out->planes[k], outw, h, out->stride[k]};
        p.visible_width = vis;
        p.output_width = outw;
        p.height = h;
    }
    cudaStream_t s = (cudaStream_t)stream;
    cudaSetDevice(ctx->device);
    cudaError_t e = reset_status(ctx, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    if (nsp > 0) {
        e = launch_superres(sp, nsp, cfg->bit_depth, ctx->status, STAGE_SUPERRES, s);
        ctx->launches++;
        if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    }
    return finish(ctx, s, host_key, msg);
}

int32_t vaco_av1_superres_upscale_picture_host(vaco_av1_ctx* ctx, const vaco_av1_picture* in,
                                               const vaco_av1_picture* out,
                                               const vaco_av1_superres_picture_config* cfg, int32_t* msg) {
    if (!ctx || !in || !out || !cfg) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    const int np = cfg->monochrome ? 1 : 3;
    for (int k = 0; k < np; ++k)
        if (in->width[k] < 0 || in->height[k] < 0 || (in->planes[k] && in->stride[k] < in->width[k]) ||
            out->width[k] < 0 || out->height[k] < 0 || (out->width[k] > 0 && out->height[k] > 0 && !out->planes[k]))
            return invalid(msg, VACO_AV1_MSG_FRAME_GEOMETRY);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaSuccess;
    vaco_av1_picture din, dout;
    if (!stage_picture_in(ctx, in, np, S_H_IN0, &din, s, &e)) return cuda_fail(ctx, e, msg);
    if (!alloc_picture(ctx, out, np, S_H_OUT0, &dout, &e)) return cuda_fail(ctx, e, msg);
    for (int k = 0; k < np; ++k)
        if (!in->planes[k]) din.planes[k] = nullptr;  // keeps vaco's missing-plane error
    int32_t st = vaco_av1_superres_upscale_picture_dev(ctx, s, &din, &dout, cfg, msg);
    if (st != VACO_AV1_OK) return st;
    e = copy_picture_out(&dout, out, np, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    return VACO_AV1_OK;
}

// ---------------------------------------------------------------- restoration

static unsigned long long lr_host_checks(int plane, const vaco_av1_lr_plane_config* c, int bw, int bh, int aw, int ah,
                                         int unit_count, int* cols_out, int* rows_out) {
    bool size_ok = c->unit_size == 32 || c->unit_size == 64 || c->unit_size == 128 || c->unit_size == 256;
    if (!bd_valid(c->bit_depth) || !size_ok || c->width <= 0 || c->height <= 0 || c->width > bw ||
        c->width > aw || c->height > bh || c->height > ah || c->width > (1 << 30) || c->height > (1 << 30))
        return make_key(STAGE_LR, lr_position(plane, LR_GEOM, 0), VACO_AV1_MSG_LR_GEOMETRY);
    int cols = (c->width + c->unit_size / 2) / c->unit_size, rows = (c->height + c->unit_size / 2) / c->unit_size;
    cols = cols < 1 ? 1 : cols;
    rows = rows < 1 ? 1 : rows;
    *cols_out = cols;
    *rows_out = rows;
    if ((long)cols * rows != unit_count)
        return make_key(STAGE_LR, lr_position(plane, LR_COUNT, 0), VACO_AV1_MSG_LR_UNIT_COUNT);
    return kNoError;
}

int32_t vaco_av1_restore_plane_dev(vaco_av1_ctx* ctx, void* stream, const uint16_t* before, int32_t before_width,
                                   int32_t before_height, int32_t before_stride, const uint16_t* after,
                                   int32_t after_width, int32_t after_height, int32_t after_stride,
                                   const vaco_av1_lr_plane_config* config, const vaco_av1_lr_unit* units,
                                   int32_t unit_count, uint16_t* output, int32_t out_stride, int32_t* msg) {
    if (!ctx || !config) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    int cols = 0, rows = 0;
    unsigned long long hk = lr_host_checks(0, config, before_width, before_height, after_width, after_height,
                                           unit_count, &cols, &rows);
    if (hk != kNoError) return invalid(msg, (int)(hk & 0xFF));
    if (!before || !after || !output || !units) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    if (before_stride < before_width || after_stride < after_width || out_stride < config->width)
        return invalid(msg, VACO_AV1_MSG_FRAME_GEOMETRY);
    cudaStream_t s = (cudaStream_t)stream;
    cudaSetDevice(ctx->device);
    cudaError_t e = reset_status(ctx, s);
    if (e == cudaSuccess) e = launch_lr_unit_check(units, unit_count, 0, ctx->status, s);
    const int maxv = (1 << config->bit_depth) - 1;
    if (e == cudaSuccess)
        e = launch_range_check(DevPlaneC{before, before_width, before_height, before_stride}, config->width,
                               config->height, maxv, ctx->status, STAGE_LR, lr_position(0, LR_SAMPLE, 0),
                               VACO_AV1_MSG_LR_SAMPLE, s);
    if (e == cudaSuccess)
        e = launch_range_check(DevPlaneC{after, after_width, after_height, after_stride}, config->width,
                               config->height, maxv, ctx->status, STAGE_LR, lr_position(0, LR_SAMPLE, 0),
                               VACO_AV1_MSG_LR_SAMPLE, s);
    // The checks must pass before filtering: restore_plane validates first.
    int32_t st = e == cudaSuccess ? finish(ctx, s, kNoError, msg) : cuda_fail(ctx, e, msg);
    ctx->launches += 3;
    if (st != VACO_AV1_OK) return st;
    LrPlane p;
    p.before = DevPlaneC{before, before_width, before_height, before_stride};
    p.before_rows = DevPlaneC{nullptr, 0, 0, 0};
    p.after = DevPlaneC{after, after_width, after_height, after_stride};
    p.out = DevPlane{output, config->width, config->height, out_stride};
    p.width = config->width;
    p.height = config->height;
    p.unit_size = config->unit_size;
    p.sub_y = config->subsampling_y ? 1 : 0;
    p.units = units;
    p.unit_cols = cols;
    p.unit_rows = rows;
    p.copy_only = 0;
    p.plane_index = 0;
    p.unit_status = nullptr;  // validated by the checks above
    e = launch_restoration(&p, 1, config->bit_depth, s);
    ctx->launches++;
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    return set_msg(msg, VACO_AV1_MSG_NONE), VACO_AV1_OK;
}

int32_t vaco_av1_restore_plane_host(vaco_av1_ctx* ctx, const uint16_t* before, int32_t before_width,
                                    int32_t before_height, const uint16_t* after, int32_t after_width,
                                    int32_t after_height, const vaco_av1_lr_plane_config* config,
                                    const vaco_av1_lr_unit* units, int32_t unit_count, uint16_t* output,
                                    int32_t* msg) {
    if (!ctx || !config) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    int cols = 0, rows = 0;
    unsigned long long hk = lr_host_checks(0, config, before_width, before_height, after_width, after_height,
                                           unit_count, &cols, &rows);
    if (hk != kNoError) return invalid(msg, (int)(hk & 0xFF));
    if (!before || !after || !output || !units) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaSuccess;
    vaco_av1_picture hin{}, din, hout{}, dout;
    hin.planes[0] = const_cast<uint16_t*>(before);
    hin.width[0] = before_width;
    hin.height[0] = before_height;
    hin.stride[0] = before_width;
    hin.planes[1] = const_cast<uint16_t*>(after);
    hin.width[1] = after_width;
    hin.height[1] = after_height;
    hin.stride[1] = after_width;
    hout.planes[0] = output;
    hout.width[0] = config->width;
    hout.height[0] = config->height;
    hout.stride[0] = config->width;
    if (!stage_picture_in(ctx, &hin, 2, S_H_IN0, &din, s, &e)) return cuda_fail(ctx, e, msg);
    if (!alloc_picture(ctx, &hout, 1, S_H_OUT0, &dout, &e)) return cuda_fail(ctx, e, msg);
    const vaco_av1_lr_unit* d_units = stage_array(ctx, S_H_SIDE0, units, (size_t)unit_count, s, &e);
    if (e != cudaSuccess || !d_units) return cuda_fail(ctx, e ? e : cudaErrorMemoryAllocation, msg);
    int32_t st = vaco_av1_restore_plane_dev(ctx, s, din.planes[0], before_width, before_height, din.stride[0],
                                            din.planes[1], after_width, after_height, din.stride[1], config, d_units,
                                            unit_count, dout.planes[0], dout.stride[0], msg);
    if (st != VACO_AV1_OK) return st;
    e = copy_picture_out(&dout, &hout, 1, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    return VACO_AV1_OK;
}

// ---------------------------------------------------------------- deblocking

int32_t vaco_av1_deblock_picture_dev(vaco_av1_ctx* ctx, void* stream, const vaco_av1_picture* src,
                                     const vaco_av1_picture* dst, const vaco_av1_frame_info* info,
                                     const uint8_t* tx_luma, const uint8_t* tx_chroma, const uint8_t* lvl_map,
                                     const vaco_av1_deblock_params* params, int32_t* msg) {
    if (!ctx || !src || !dst || !info || !params) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    if (!info_ok(info) || !padded_picture_ok(src, info) || !padded_picture_ok(dst, info))
        return invalid(msg, VACO_AV1_MSG_FRAME_GEOMETRY);
    cudaStream_t s = (cudaStream_t)stream;
    cudaSetDevice(ctx->device);
    cudaError_t e = reset_status(ctx, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    unsigned long long hk = run_deblock(ctx, s, *src, *dst, *info, tx_luma, tx_chroma, lvl_map, *params, &e);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    return finish(ctx, s, hk, msg);
}

int32_t vaco_av1_deblock_picture_host(vaco_av1_ctx* ctx, const vaco_av1_picture* src, const vaco_av1_picture* dst,
                                      const vaco_av1_frame_info* info, const uint8_t* tx_luma,
                                      const uint8_t* tx_chroma, const uint8_t* lvl_map,
                                      const vaco_av1_deblock_params* params, int32_t* msg) {
    if (!ctx || !src || !dst || !info || !params) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    if (!info_ok(info) || !padded_picture_ok(src, info) || !padded_picture_ok(dst, info))
        return invalid(msg, VACO_AV1_MSG_FRAME_GEOMETRY);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const int np = info->monochrome ? 1 : 3;
    const int ssx = info->subsampling_x, ssy = info->subsampling_y;
    cudaError_t e = cudaSuccess;
    vaco_av1_picture dsrc, ddst;
    if (!stage_picture_in(ctx, src, np, S_H_IN0, &dsrc, s, &e)) return cuda_fail(ctx, e, msg);
    if (!alloc_picture(ctx, dst, np, S_H_OUT0, &ddst, &e)) return cuda_fail(ctx, e, msg);
    size_t n_luma = (size_t)info->mi_rows * info->mi_cols;
    size_t n_chroma = (size_t)((info->mi_rows + ssy) >> ssy) * ((info->mi_cols + ssx) >> ssx);
    const uint8_t* d_txl = stage_array(ctx, S_H_SIDE0, tx_luma, n_luma, s, &e);
    const uint8_t* d_txc = e == cudaSuccess && np > 1 ? stage_array(ctx, S_H_SIDE1, tx_chroma, n_chroma, s, &e) : nullptr;
    const uint8_t* d_lvl = e == cudaSuccess ? stage_array(ctx, S_H_SIDE2, lvl_map, n_luma * 4, s, &e) : nullptr;
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    int32_t st = vaco_av1_deblock_picture_dev(ctx, s, &dsrc, &ddst, info, d_txl, d_txc, d_lvl, params, msg);
    if (st != VACO_AV1_OK) return st;
    e = copy_picture_out(&ddst, dst, np, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    return VACO_AV1_OK;
}

// ---------------------------------------------------------------- whole chain

// check_dst = false: the caller supplies the destination itself (emission).
static bool chain_geometry_ok(const vaco_av1_frame_job* j, bool check_dst = true) {
    const vaco_av1_frame_info& i = j->info;
    if (!info_ok(&i) || !padded_picture_ok(&j->src, &i)) return false;
    if (!av1_subsampling_ok(i.subsampling_x, i.subsampling_y)) return false;
    if (i.coded_width <= 0 || i.coded_height <= 0 || i.coded_width > i.mi_cols * 4 || i.coded_height > i.mi_rows * 4)
        return false;
    if (i.mi_cols != 2 * ((i.coded_width + 7) >> 3) || i.mi_rows != 2 * ((i.coded_height + 7) >> 3)) return false;
    if (i.upscaled_width < i.coded_width) return false;
    const int np = i.monochrome ? 1 : 3;
    if (np > 1 && ((i.subsampling_x && ((i.coded_width | i.upscaled_width) & 1)) ||
                   (i.subsampling_y && (i.coded_height & 1))))
        return false;
    for (int k = 0; k < np; ++k) {
        int sx = k ? i.subsampling_x : 0, sy = k ? i.subsampling_y : 0;
        if (check_dst && (!j->dst.planes[k] || j->dst.width[k] != (i.upscaled_width >> sx) ||
                          j->dst.height[k] != (i.coded_height >> sy) || j->dst.stride[k] < j->dst.width[k]))
            return false;
    }
    return true;
}

// The chain on device pointers.  Deblocking and CDEF run fused
// (dbcdef.cu): the deblocked picture exists only as restoration's compact
// stripe-boundary rows.
static int32_t postfilter_dev_impl(vaco_av1_ctx* ctx, cudaStream_t s, const vaco_av1_frame_job* job, int32_t* msg,
                                   bool defer) {
    const vaco_av1_frame_info& info = job->info;
    const int np = info.monochrome ? 1 : 3;
    const int ssx = info.subsampling_x, ssy = info.subsampling_y;
    const bool superres = info.upscaled_width != info.coded_width;
    bool lr_active = false;
    for (int k = 0; k < np; ++k) lr_active = lr_active || job->lr_type[k] != VACO_AV1_FRAME_LR_NONE;
    // With deferred status the word keeps accumulating until the next flush.
    cudaError_t e = defer ? cudaSuccess : reset_status(ctx, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);

    vaco_av1_picture cdef;
    if (!alloc_picture(ctx, &job->src, np, S_CDEF0, &cdef, &e)) return cuda_fail(ctx, e, msg);
    // Compact pre-CDEF stripe-boundary rows (only restoration reads them).
    vaco_av1_picture rows_like{}, pre_rows{};
    DevPlane pre_rows_dp[3] = {};
    if (lr_active) {
        for (int k = 0; k < np; ++k) {
            rows_like.width[k] = job->src.width[k];
            rows_like.height[k] = pre_rows_count(job->src.height[k], k ? ssy : 0);
        }
        if (!alloc_picture(ctx, &rows_like, np, S_PRE0, &pre_rows, &e)) return cuda_fail(ctx, e, msg);
        for (int k = 0; k < np; ++k) pre_rows_dp[k] = mplane(pre_rows, k);
    }
    // Without superres, a plane whose restoration is off gets its output
    // from the fused deblock+CDEF kernel itself (copy_visible_plane,
    // decode.rs:673-681, with no copy afterwards), when the output is laid
    // out for 32-bit stores.
    DirectPlane direct[3] = {};
    for (int k = 0; k < np && !superres; ++k) {
        if (job->lr_type[k] != VACO_AV1_FRAME_LR_NONE) continue;
        const int sx = k ? ssx : 0, sy = k ? ssy : 0;
        const int w = info.upscaled_width >> sx, h = info.coded_height >> sy;
        const DevPlane out{job->dst.planes[k], w, h, job->dst.stride[k]};
        if (out.data && w > 0 && h > 0 && w <= job->dst.width[k] && h <= job->dst.height[k] &&
            (out.stride & 1) == 0 && (reinterpret_cast<uintptr_t>(out.data) & 3) == 0)
            direct[k] = DirectPlane{out};
    }
    ctx->mark(0, s);

    // ---- deblocking + CDEF (host checks in the order deblock_frame / apply_cdef run them)
    unsigned long long hk = kNoError;
    {
        const vaco_av1_deblock_params& db = job->deblock;
        bool params_ok = bd_valid(info.bit_depth) && db.sharpness <= 7;
        for (int k = 0; k < 4; ++k) params_ok = params_ok && db.levels[k] <= 63;
        if (!params_ok || !job->tx_luma || (np > 1 && !job->tx_chroma))
            hk = make_key(STAGE_DEBLOCK, 0, params_ok ? VACO_AV1_MSG_NULL_ARGUMENT : VACO_AV1_MSG_DB_PARAMS);
        const vaco_av1_cdef_params& cp = job->cdef;
        bool all_zero = true;
        for (int k = 0; k < 8; ++k)
            all_zero = all_zero && cp.y_primary[k] == 0 && cp.y_secondary[k] == 0 && cp.uv_primary[k] == 0 &&
                       cp.uv_secondary[k] == 0;
        const bool cdef_on = cp.enabled && !all_zero;
        if (hk == kNoError && cdef_on && (!job->skip || (!job->cdef_idx && job->cdef_count > 0)))
            hk = make_key(STAGE_CDEF, 0, VACO_AV1_MSG_NULL_ARGUMENT);
        if (hk == kNoError) {
            DbCdefLaunch L;
            L.src = job->src;
            L.dst = cdef;
            for (int k = 0; k < 3; ++k) L.pre_rows[k] = k < np && lr_active ? pre_rows_dp[k] : DevPlane{nullptr, 0, 0, 0};
            L.info = info;
            L.tx_luma = job->tx_luma;
            L.tx_chroma = job->tx_chroma;
            L.lvl_map = job->lvl_map;
            L.deblock = db;
            L.skip = cdef_on ? job->skip : nullptr;
            L.cdef_idx = job->cdef_idx;
            L.cdef_stride = job->cdef_stride;
            L.cdef_count = job->cdef_count;
            L.cdef = cp;
            L.status = ctx->status;
            L.threads = ctx->tuning.dbcdef_threads == 128 ? 128 : 256;
            for (int k = 0; k < 3; ++k) L.direct[k] = direct[k];
            e = launch_dbcdef(L, s);
            ctx->launches++;
            if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
        }
    }
    ctx->mark(1, s);
    ctx->mark(2, s);

    // ---- superres of the CDEF picture and of the boundary rows
    vaco_av1_picture after = cdef, before_rows = pre_rows;
    if (hk == kNoError && superres) {
        vaco_av1_picture out_like{}, rows_out_like{};
        for (int k = 0; k < np; ++k) {
            const int sx = k ? ssx : 0, sy = k ? ssy : 0;
            out_like.width[k] = (info.upscaled_width + sx) >> sx;
            out_like.height[k] = (info.coded_height + sy) >> sy;
            rows_out_like.width[k] = out_like.width[k];
            rows_out_like.height[k] = pre_rows.height[k];
        }
        vaco_av1_picture ucdef, urows;
        if (!alloc_picture(ctx, &out_like, np, S_UCDEF0, &ucdef, &e)) return cuda_fail(ctx, e, msg);
        // The picture's planes and, for restoration, the pre-CDEF boundary
        // rows go to one launch.
        SuperresPlane sp[2 * 3];
        int nsp = np;
        for (int k = 0; k < np; ++k) {
            const int sx = k ? ssx : 0, sy = k ? ssy : 0;
            sp[k].in = cplane(cdef, k);
            sp[k].out = mplane(ucdef, k);
            sp[k].visible_width = (info.coded_width + sx) >> sx;
            sp[k].output_width = (info.upscaled_width + sx) >> sx;
            sp[k].height = (info.coded_height + sy) >> sy;
        }
        after = ucdef;
        if (lr_active) {
            if (!alloc_picture(ctx, &rows_out_like, np, S_UPRE0, &urows, &e)) return cuda_fail(ctx, e, msg);
            // only the rows the fused kernel wrote (indices 4 .. 4+n)
            for (int k = 0; k < np; ++k) {
                const int n_rows = pre_rows_written(job->src.height[k], k ? ssy : 0);
                SuperresPlane& r = sp[np + k];
                r = sp[k];
                r.in = DevPlaneC{pre_rows.planes[k] + 4L * pre_rows.stride[k], pre_rows.width[k], n_rows,
                                 pre_rows.stride[k]};
                r.out = DevPlane{urows.planes[k] + 4L * urows.stride[k], urows.width[k], n_rows, urows.stride[k]};
                r.height = n_rows;
            }
            nsp = 2 * np;
            before_rows = urows;
        }
        e = launch_superres(sp, nsp, info.bit_depth, ctx->status, STAGE_SUPERRES, s);
        ctx->launches++;
        if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    }
    ctx->mark(3, s);

    // ---- restoration (or the visible copy) into the output
    if (hk == kNoError) {
        LrPlane lp[3];
        int nlr = 0;
        for (int k = 0; k < np && hk == kNoError; ++k) {
            const int sx = k ? ssx : 0, sy = k ? ssy : 0;
            const int w = info.upscaled_width >> sx, h = info.coded_height >> sy;
            if (job->lr_type[k] == VACO_AV1_FRAME_LR_NONE) {
                // copy_visible_plane (decode.rs:673-681), as copy-only tiles
                // of the same launch: SM copies run at HBM speed, a
                // device-to-device memcpy at copy-engine speed.  Nothing to
                // do when the fused kernel wrote the plane (direct).
                if (!direct[k].out.data)
                    lp[nlr++] = copy_only_plane(cplane(after, k), mplane(job->dst, k), w, h, (k && ssy) ? 1 : 0, k);
                continue;
            }
            if (job->lr_unit_size[k] == 0) {
                hk = make_key(STAGE_LR, lr_position(k, LR_NO_UNIT_SIZE, 0), VACO_AV1_MSG_LR_NO_UNIT_SIZE);
                break;
            }
            vaco_av1_lr_plane_config c{w, h, info.bit_depth, job->lr_unit_size[k], (k && ssy) ? 1 : 0};
            int cols = 0, rows = 0;
            hk = lr_host_checks(k, &c, after.width[k], after.height[k], after.width[k], after.height[k],
                                job->lr_unit_count[k], &cols, &rows);
            if (hk != kNoError) break;
            if (!job->lr_units[k]) {
                hk = make_key(STAGE_LR, lr_position(k, LR_COUNT, 0), VACO_AV1_MSG_NULL_ARGUMENT);
                break;
            }
            LrPlane& p = lp[nlr++];
            p.plane_index = k;
            p.unit_status = ctx->status;  // units are validated by the restoration tiles
            p.before = DevPlaneC{nullptr, 0, 0, 0};
            p.before_rows = cplane(before_rows, k);
            p.after = cplane(after, k);
            p.out = mplane(job->dst, k);
            p.width = w;
            p.height = h;
            p.unit_size = c.unit_size;
            p.sub_y = c.subsampling_y;
            p.units = job->lr_units[k];
            p.unit_cols = cols;
            p.unit_rows = rows;
            p.copy_only = 0;
        }
        // Samples reaching restoration inside the chain were produced by the
        // deblocking / CDEF / superres kernels from range-checked input, so
        // they are in range by construction: no second scan is needed.
        if (hk == kNoError && nlr > 0) {
            e = launch_restoration(lp, nlr, info.bit_depth, s);
            ctx->launches++;
            if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
        }
    }
    ctx->mark(4, s);
    if (defer) {
        // Host-side failures are known now; device-side ones wait for the flush.
        if (hk != kNoError) {
            set_msg(msg, (int)(hk & 0xFF));
            return VACO_AV1_INVALID_DATA;
        }
        set_msg(msg, VACO_AV1_MSG_NONE);
        return VACO_AV1_OK;
    }
    return finish(ctx, s, hk, msg);
}

int32_t vaco_av1_postfilter_frame_dev(vaco_av1_ctx* ctx, void* stream, const vaco_av1_frame_job* job, int32_t* msg) {
    if (!ctx || !job) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    if (!chain_geometry_ok(job)) return invalid(msg, VACO_AV1_MSG_FRAME_GEOMETRY);
    cudaSetDevice(ctx->device);
    return postfilter_dev_impl(ctx, (cudaStream_t)stream, job, msg, ctx->deferred);
}

// The chain on a job whose pictures and side information are in host memory:
// stages the inputs into context scratch, runs the chain into a device
// picture `*d_out` (context scratch), and leaves the stream synchronized.
// With sc != s the inputs are copied on stream sc, which `staged` then
// orders before the chain on s; `defer` is postfilter_dev_impl's.
static int32_t postfilter_from_host(vaco_av1_ctx* ctx, cudaStream_t s, const vaco_av1_frame_job* job,
                                    vaco_av1_picture* d_out, int32_t* msg, cudaStream_t sc = nullptr,
                                    cudaEvent_t staged = nullptr, bool defer = false) {
    if (!sc) sc = s;
    const vaco_av1_frame_info& info = job->info;
    const int np = info.monochrome ? 1 : 3;
    const int ssx = info.subsampling_x, ssy = info.subsampling_y;
    cudaError_t e = cudaSuccess;
    vaco_av1_frame_job d = *job;
    if (!stage_picture_in(ctx, &job->src, np, S_H_IN0, &d.src, sc, &e)) return cuda_fail(ctx, e, msg);
    if (!alloc_picture(ctx, &job->dst, np, S_H_OUT0, &d.dst, &e)) return cuda_fail(ctx, e, msg);
    size_t n_luma = (size_t)info.mi_rows * info.mi_cols;
    size_t n_chroma = (size_t)((info.mi_rows + ssy) >> ssy) * ((info.mi_cols + ssx) >> ssx);
    d.tx_luma = stage_array(ctx, S_H_SIDE0, job->tx_luma, n_luma, sc, &e);
    if (e == cudaSuccess) d.tx_chroma = np > 1 ? stage_array(ctx, S_H_SIDE1, job->tx_chroma, n_chroma, sc, &e) : nullptr;
    if (e == cudaSuccess) d.lvl_map = stage_array(ctx, S_H_SIDE2, job->lvl_map, n_luma * 4, sc, &e);
    if (e == cudaSuccess) d.skip = stage_array(ctx, S_H_SIDE3, job->skip, n_luma, sc, &e);
    if (e == cudaSuccess)
        d.cdef_idx = stage_array(ctx, S_H_SIDE4, job->cdef_idx, (size_t)(job->cdef_count > 0 ? job->cdef_count : 0),
                                 sc, &e);
    // All planes' units in one staging buffer.
    size_t total_units = 0;
    for (int k = 0; k < 3; ++k)
        if (job->lr_units[k] && job->lr_unit_count[k] > 0) total_units += (size_t)job->lr_unit_count[k];
    if (e == cudaSuccess && total_units > 0) {
        vaco_av1_lr_unit* du = (vaco_av1_lr_unit*)ctx->scratch(S_H_SIDE5, total_units * sizeof(vaco_av1_lr_unit));
        if (!du) return cuda_fail(ctx, cudaErrorMemoryAllocation, msg);
        size_t o = 0;
        for (int k = 0; k < 3; ++k) {
            if (job->lr_units[k] && job->lr_unit_count[k] > 0) {
                e = cudaMemcpyAsync(du + o, job->lr_units[k], sizeof(vaco_av1_lr_unit) * job->lr_unit_count[k],
                                    cudaMemcpyHostToDevice, sc);
                d.lr_units[k] = du + o;
                o += (size_t)job->lr_unit_count[k];
                if (e != cudaSuccess) break;
            }
        }
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    if (sc != s) {
        e = cudaEventRecord(staged, sc);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s, staged, 0);
        if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    }
    int32_t st = postfilter_dev_impl(ctx, s, &d, msg, defer);
    *d_out = d.dst;
    return st;
}

int32_t vaco_av1_postfilter_frame_host(vaco_av1_ctx* ctx, const vaco_av1_frame_job* job, int32_t* msg) {
    if (!ctx || !job) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    if (!chain_geometry_ok(job)) return invalid(msg, VACO_AV1_MSG_FRAME_GEOMETRY);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    vaco_av1_picture dst;
    const int32_t st = postfilter_from_host(ctx, s, job, &dst, msg);
    if (st != VACO_AV1_OK) return st;
    cudaError_t e = copy_picture_out(&dst, &job->dst, job->info.monochrome ? 1 : 3, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    return VACO_AV1_OK;
}
// ---------------------------------------------------------------- pipelined host entry points

int32_t vaco_av1_postfilter_frame_host_submit(vaco_av1_ctx* ctx, const vaco_av1_frame_job* job, uint64_t* ticket,
                                              int32_t* msg) {
    if (!ctx || !job || !ticket) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    if (!chain_geometry_ok(job)) return invalid(msg, VACO_AV1_MSG_FRAME_GEOMETRY);
    cudaSetDevice(ctx->device);
    const int k = (int)(ctx->next_ticket % vaco_av1_ctx::kPipeSlots);
    vaco_av1_ctx::PipeSlot& slot = ctx->pipe[k];
    if (slot.busy) {
        set_msg(msg, VACO_AV1_MSG_QUEUE_FULL);
        return VACO_AV1_LIMIT_EXCEEDED;
    }
    cudaError_t e = cudaSuccess;
    if (!ctx->copy_in) e = cudaStreamCreateWithFlags(&ctx->copy_in, cudaStreamNonBlocking);
    if (e == cudaSuccess && !ctx->copy_out) e = cudaStreamCreateWithFlags(&ctx->copy_out, cudaStreamNonBlocking);
    if (e == cudaSuccess && !slot.done) {
        e = cudaEventCreateWithFlags(&slot.staged, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&slot.filtered, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&slot.done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMalloc(&slot.status, sizeof(DeviceStatus));
        if (e == cudaSuccess) e = cudaMallocHost(&slot.status_host, sizeof(unsigned long long));
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    // The slot's own scratch and status word for this frame.
    vaco::DeviceStatus* const ctx_status = ctx->status;
    ctx->scratch_set = 1 + k;
    ctx->status = slot.status;
    cudaStream_t s = ctx->stream;
    e = cudaMemsetAsync(slot.status, 0xFF, sizeof(DeviceStatus), s);
    vaco_av1_picture dst{};
    int32_t st = e == cudaSuccess ? postfilter_from_host(ctx, s, job, &dst, msg, ctx->copy_in, slot.staged, true)
                                  : cuda_fail(ctx, e, msg);
    if (st == VACO_AV1_OK) {
        e = cudaEventRecord(slot.filtered, s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->copy_out, slot.filtered, 0);
        if (e == cudaSuccess) e = copy_picture_out(&dst, &job->dst, job->info.monochrome ? 1 : 3, ctx->copy_out);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(slot.status_host, slot.status, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                ctx->copy_out);
        if (e == cudaSuccess) e = cudaEventRecord(slot.done, ctx->copy_out);
        if (e != cudaSuccess) st = cuda_fail(ctx, e, msg);
    }
    ctx->scratch_set = 0;
    ctx->status = ctx_status;
    if (st != VACO_AV1_OK) return st;
    slot.busy = true;
    slot.ticket = ctx->next_ticket++;
    *ticket = slot.ticket;
    set_msg(msg, VACO_AV1_MSG_NONE);
    return VACO_AV1_OK;
}

int32_t vaco_av1_postfilter_frame_host_wait(vaco_av1_ctx* ctx, uint64_t ticket, int32_t* msg) {
    if (!ctx) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    vaco_av1_ctx::PipeSlot& slot = ctx->pipe[ticket % vaco_av1_ctx::kPipeSlots];
    if (!slot.busy || slot.ticket != ticket) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    cudaSetDevice(ctx->device);
    const cudaError_t e = cudaEventSynchronize(slot.done);
    slot.busy = false;
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    const unsigned long long key = *slot.status_host;
    if (key == kNoError) {
        set_msg(msg, VACO_AV1_MSG_NONE);
        return VACO_AV1_OK;
    }
    set_msg(msg, (int)(key & 0xFF));
    return VACO_AV1_INVALID_DATA;
}

// ---------------------------------------------------------------- frame emission

// The pixel formats pic_to_frame can name (src/decode.rs:3802-3819): every
// AV1 layout except 8-bit 4:4:0, for which vaco-pixfmt has no "yuv440p8le".
static bool emit_format_ok(const vaco_av1_frame_info& i) {
    if (i.bit_depth != 8 && i.bit_depth != 10 && i.bit_depth != 12) return false;
    if (i.subsampling_x < 0 || i.subsampling_x > 1 || i.subsampling_y < 0 || i.subsampling_y > 1) return false;
    return !(i.bit_depth == 8 && !i.monochrome && i.subsampling_x == 0 && i.subsampling_y == 1);
}

// Per plane: pic_to_frame's extents (upscaled_width x coded_height, chroma
// rounded up, src/decode.rs:3820-3828) cut to the source plane, as blit's
// w.min(pic.width()) does.  Returns 0 or a message id.
static int emit_plan(const vaco_av1_picture* pic, const vaco_av1_frame_info& i, const vaco_av1_frame_buffer* out,
                     EmitPlane* ep, int* np_out) {
    if (!emit_format_ok(i)) return VACO_AV1_MSG_PIXEL_FORMAT;
    if (i.upscaled_width <= 0 || i.coded_height <= 0) return VACO_AV1_MSG_FRAME_GEOMETRY;
    const int np = i.monochrome ? 1 : 3;
    const int bps = i.bit_depth > 8 ? 2 : 1;
    for (int k = 0; k < np; ++k) {
        const int sx = k ? i.subsampling_x : 0, sy = k ? i.subsampling_y : 0;
        const int fw = (i.upscaled_width + (1 << sx) - 1) >> sx, fh = (i.coded_height + (1 << sy) - 1) >> sy;
        if (!pic->planes[k] || !out->planes[k]) return VACO_AV1_MSG_NULL_ARGUMENT;
        if (pic->width[k] < 0 || pic->height[k] < 0 || pic->stride[k] < pic->width[k]) return VACO_AV1_MSG_FRAME_GEOMETRY;
        const int w = std::min(fw, pic->width[k]), h = std::min(fh, pic->height[k]);
        if (out->linesize[k] < (int64_t)w * bps) return VACO_AV1_MSG_FRAME_GEOMETRY;
        ep[k] = EmitPlane{pic->planes[k], pic->stride[k], (uint8_t*)out->planes[k], out->linesize[k], w, h};
    }
    *np_out = np;
    return 0;
}

int32_t vaco_av1_emit_frame_dev(vaco_av1_ctx* ctx, void* stream, const vaco_av1_picture* pic,
                                const vaco_av1_frame_info* info, const vaco_av1_frame_buffer* out, int32_t* msg) {
    if (!ctx || !pic || !info || !out) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    EmitPlane ep[3];
    int np = 0;
    if (int m = emit_plan(pic, *info, out, ep, &np)) return invalid(msg, m);
    cudaSetDevice(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    // No sample can fail emission, so nothing on the device needs reporting:
    // the call returns once the kernel is enqueued.
    cudaError_t e = launch_emit(ep, np, info->bit_depth > 8, ctx->sm_count, s);
    ctx->launches++;
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    set_msg(msg, VACO_AV1_MSG_NONE);
    return VACO_AV1_OK;
}

// Packs the device picture `dev` into context scratch and copies the packed
// rows to the host frame `out` (one 2-D copy per plane), synchronously.
static int32_t emit_to_host(vaco_av1_ctx* ctx, cudaStream_t s, const vaco_av1_picture* dev,
                            const vaco_av1_frame_info& info, const vaco_av1_frame_buffer* out, int32_t* msg) {
    EmitPlane ep[3];
    int np = 0;
    if (int m = emit_plan(dev, info, out, ep, &np)) return invalid(msg, m);
    const int bps = info.bit_depth > 8 ? 2 : 1;
    for (int k = 0; k < np; ++k) {
        const long long row = (long long)align_up((size_t)std::max(ep[k].width * bps, 1), 64);
        void* d = ctx->scratch(S_EMIT0 + k, (size_t)row * std::max(ep[k].height, 1));
        if (!d) return cuda_fail(ctx, cudaErrorMemoryAllocation, msg);
        ep[k].dst = (uint8_t*)d;
        ep[k].dst_stride = row;
    }
    cudaError_t e = launch_emit(ep, np, bps == 2, ctx->sm_count, s);
    ctx->launches++;
    for (int k = 0; k < np && e == cudaSuccess; ++k)
        if (ep[k].width > 0 && ep[k].height > 0)
            e = cudaMemcpy2DAsync(out->planes[k], (size_t)out->linesize[k], ep[k].dst, (size_t)ep[k].dst_stride,
                                  (size_t)ep[k].width * bps, (size_t)ep[k].height, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    set_msg(msg, VACO_AV1_MSG_NONE);
    return VACO_AV1_OK;
}

int32_t vaco_av1_emit_frame_host(vaco_av1_ctx* ctx, const vaco_av1_picture* pic, const vaco_av1_frame_info* info,
                                 const vaco_av1_frame_buffer* out, int32_t* msg) {
    if (!ctx || !pic || !info || !out) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    if (!emit_format_ok(*info)) return invalid(msg, VACO_AV1_MSG_PIXEL_FORMAT);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const int np = info->monochrome ? 1 : 3;
    for (int k = 0; k < np; ++k)
        if (!pic->planes[k]) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    vaco_av1_picture dev;
    cudaError_t e = cudaSuccess;
    if (!stage_picture_in(ctx, pic, np, S_H_IN0, &dev, s, &e)) return cuda_fail(ctx, e, msg);
    return emit_to_host(ctx, s, &dev, *info, out, msg);
}

int32_t vaco_av1_postfilter_frame_emit_host(vaco_av1_ctx* ctx, const vaco_av1_frame_job* job,
                                            const vaco_av1_frame_buffer* out, int32_t* msg) {
    if (!ctx || !job || !out) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    if (!chain_geometry_ok(job, false)) return invalid(msg, VACO_AV1_MSG_FRAME_GEOMETRY);
    if (!emit_format_ok(job->info)) return invalid(msg, VACO_AV1_MSG_PIXEL_FORMAT);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    // The chain's own output stays on the device, in scratch of the chain's
    // output extents.
    vaco_av1_frame_job j = *job;
    const vaco_av1_frame_info& i = job->info;
    for (int k = 0; k < 3; ++k) {
        const int sx = k ? i.subsampling_x : 0, sy = k ? i.subsampling_y : 0;
        j.dst.width[k] = i.upscaled_width >> sx;
        j.dst.height[k] = i.coded_height >> sy;
        j.dst.stride[k] = j.dst.width[k];
    }
    vaco_av1_picture dst;
    const int32_t st = postfilter_from_host(ctx, s, &j, &dst, msg);
    if (st != VACO_AV1_OK) return st;
    return emit_to_host(ctx, s, &dst, i, out, msg);
}

}  // extern "C"

// ---------------------------------------------------------------- film grain

// Ranges of film_grain_params() (AV1 5.9.30); point values must increase,
// which the scaling lookup's divisions rely on.
static bool grain_params_ok(const vaco_av1_film_grain_params& p) {
    auto increasing = [](const uint8_t* v, int n) {
        for (int i = 1; i < n; ++i)
            if (v[i] <= v[i - 1]) return false;
        return true;
    };
    return p.num_y_points <= 14 && p.num_cb_points <= 10 && p.num_cr_points <= 10 && p.ar_coeff_lag <= 3 &&
           p.grain_scaling_minus_8 <= 3 && p.ar_coeff_shift_minus_6 <= 3 && p.grain_scale_shift <= 3 &&
           p.cb_offset <= 511 && p.cr_offset <= 511 && increasing(p.point_y_value, p.num_y_points) &&
           increasing(p.point_cb_value, p.num_cb_points) && increasing(p.point_cr_value, p.num_cr_points);
}

// Checks shared by both film grain entry points; returns a message id.
static int grain_check(const vaco_av1_picture* in, const vaco_av1_picture* out, const vaco_av1_frame_info* info,
                       const vaco_av1_film_grain_params* params, const int16_t* gauss) {
    if (!in || !out || !info || !params || !gauss) return VACO_AV1_MSG_NULL_ARGUMENT;
    if (!bd_valid(info->bit_depth) || !grain_params_ok(*params)) return VACO_AV1_MSG_FG_PARAMS;
    if (!av1_subsampling_ok(info->subsampling_x, info->subsampling_y)) return VACO_AV1_MSG_FRAME_GEOMETRY;
    const int w = info->upscaled_width, h = info->coded_height;
    if (w <= 0 || h <= 0 || w > 65536 || h > 65536) return VACO_AV1_MSG_FRAME_GEOMETRY;
    const int np = info->monochrome ? 1 : 3;
    for (int k = 0; k < np; ++k) {
        const int pw = k ? (w + info->subsampling_x) >> info->subsampling_x : w;
        const int ph = k ? (h + info->subsampling_y) >> info->subsampling_y : h;
        if (!in->planes[k] || !out->planes[k]) return VACO_AV1_MSG_NULL_ARGUMENT;
        if (in->width[k] < pw || in->height[k] < ph || out->width[k] < pw || out->height[k] < ph ||
            in->stride[k] < in->width[k] || out->stride[k] < out->width[k])
            return VACO_AV1_MSG_FRAME_GEOMETRY;
    }
    return VACO_AV1_MSG_NONE;
}

// defer: as postfilter_dev_impl's (deferred status: no reset, no sync; the
// flush reports device-side errors).
static int32_t film_grain_impl(vaco_av1_ctx* ctx, cudaStream_t s, const vaco_av1_picture* in,
                               const vaco_av1_picture* out, const vaco_av1_frame_info* info,
                               const vaco_av1_film_grain_params* params, const int16_t* gauss, int32_t* msg,
                               bool defer) {
    const int np = info->monochrome ? 1 : 3;
    const int w = info->upscaled_width, h = info->coded_height;
    cudaError_t e = defer ? cudaSuccess : reset_status(ctx, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    // The frame's workspace set; its template kernel runs on the set's own
    // stream once the set's previous reader has run, and `s` waits for it.
    const int k_set = (int)(ctx->grain_next++ % vaco_av1_ctx::kGrainSets);
    vaco_av1_ctx::GrainSet& gs = ctx->grain[k_set];
    if (!gs.stream) e = cudaStreamCreateWithFlags(&gs.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess && !gs.ready) e = cudaEventCreateWithFlags(&gs.ready, cudaEventDisableTiming);
    if (e == cudaSuccess && !gs.free) e = cudaEventCreateWithFlags(&gs.free, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    void* ws = ctx->scratch(S_GRAIN0 + k_set, film_grain_workspace_bytes(np, w, h));
    if (!ws) return cuda_fail(ctx, cudaErrorMemoryAllocation, msg);
    DevPlaneC din[3];
    DevPlane dout[3];
    for (int k = 0; k < np; ++k) {
        din[k] = cplane(*in, k);
        dout[k] = mplane(*out, k);
    }
    const int bd = info->bit_depth, ssx = info->subsampling_x, ssy = info->subsampling_y;
    if (params->apply_grain) {
        if (gs.used) e = cudaStreamWaitEvent(gs.stream, gs.free, 0);
        if (e == cudaSuccess) e = launch_grain_template(*params, gauss, np, bd, ssx, ssy, w, h, ws, gs.stream);
        ctx->launches++;
        if (e == cudaSuccess) e = cudaEventRecord(gs.ready, gs.stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s, gs.ready, 0);
    }
    if (e == cudaSuccess) e = launch_grain_apply(*params, din, dout, np, bd, ssx, ssy, w, h, ws, ctx->status,
                                                 ctx->sm_count, s);
    ctx->launches++;
    if (e == cudaSuccess) e = cudaEventRecord(gs.free, s);
    gs.used = true;
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    if (defer) {
        set_msg(msg, VACO_AV1_MSG_NONE);
        return VACO_AV1_OK;
    }
    return finish(ctx, s, kNoError, msg);
}

int32_t vaco_av1_film_grain_dev(vaco_av1_ctx* ctx, void* stream, const vaco_av1_picture* in,
                                const vaco_av1_picture* out, const vaco_av1_frame_info* info,
                                const vaco_av1_film_grain_params* params, const int16_t* gaussian_sequence,
                                int32_t* msg) {
    if (!ctx) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    if (int m = grain_check(in, out, info, params, gaussian_sequence)) return invalid(msg, m);
    cudaSetDevice(ctx->device);
    return film_grain_impl(ctx, (cudaStream_t)stream, in, out, info, params, gaussian_sequence, msg, ctx->deferred);
}

int32_t vaco_av1_film_grain_host(vaco_av1_ctx* ctx, const vaco_av1_picture* in, const vaco_av1_picture* out,
                                 const vaco_av1_frame_info* info, const vaco_av1_film_grain_params* params,
                                 const int16_t* gaussian_sequence, int32_t* msg) {
    if (!ctx) return invalid(msg, VACO_AV1_MSG_NULL_ARGUMENT);
    if (int m = grain_check(in, out, info, params, gaussian_sequence)) return invalid(msg, m);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const int np = info->monochrome ? 1 : 3;
    vaco_av1_picture din, dout;
    cudaError_t e = cudaSuccess;
    if (!stage_picture_in(ctx, in, np, S_H_IN0, &din, s, &e)) return cuda_fail(ctx, e, msg);
    if (!alloc_picture(ctx, out, np, S_H_OUT0, &dout, &e)) return cuda_fail(ctx, e, msg);
    const int32_t st = film_grain_impl(ctx, s, &din, &dout, info, params, gaussian_sequence, msg, false);
    if (st != VACO_AV1_OK) return st;
    e = copy_picture_out(&dout, out, np, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, msg);
    return VACO_AV1_OK;
}
