// noalloc.cu -- the post-filter chain without any device allocation.
//
// vaco_av1_postfilter_frame_noalloc() runs the same chain as
// vaco_av1_postfilter_frame_dev(), with the same results, but it needs no
// context and it allocates nothing.  It runs the per-stage kernels
// (deblocking passes, CDEF, superres, restoration) rather than the fused
// deblock+CDEF kernel: they keep the whole deblocked picture, which is what
// the fixed array holds, instead of the context's separate stripe-row
// buffer.  It serves callers that cannot call cudaMalloc.  One example is a
// decoder plugin inside a host application that owns all device memory
// through its own pool and forbids plugins from allocating.  Another is a
// real-time path where an allocation's implicit device-wide synchronization
// would stall unrelated streams.  Such callers still pass device pointers
// for every input and output; the chain's intermediate pictures (the
// deblocked picture, the CDEF picture and, with superres, their upscaled
// copies) and its status word live in one file-scope device array instead.
//
// Limits and sharing rules:
//   - The array is kNoAllocScratchBytes (16 MiB) of sample storage plus
//     256 bytes for the status word.  Every GPU that loads this library holds
//     it until the process exits.  A frame whose intermediates do not fit is
//     rejected with VACO_AV1_LIMIT_EXCEEDED / VACO_AV1_MSG_SCRATCH_LIMIT.
//     A frame needs, per plane, two pictures at the Mi-padded size and,
//     with superres, one or (when restoration runs) two more at the
//     upscaled size, each row pitch rounded up to 64 samples.  So a
//     1920-wide 4:2:0 frame fits up to 1456 rows without superres (1920x1088
//     with room to spare, 1920x1464 does not), and with superres and
//     restoration 1024x720 -> 1280x720 fits while 1440x1080 -> 1920x1080
//     does not.
//   - All calls in the process share the array, which keeps the contents of
//     the last call.  Every call rewrites the intermediates in full and
//     resets the status word before its first kernel.  Calls whose GPU work
//     overlaps -- from two host threads, or on two streams without ordering
//     between them -- race on the array and produce undefined output.
//   - The first call on a device looks up the array's device address with
//     cudaGetSymbolAddress() while that device is current, and caches it.
//     Make that first call before any stream capture begins on the device.
//   - A call synchronizes `stream` once, to read the status word back into a
//     host variable.
#include <cstring>
#include <mutex>

#include "common.cuh"
#include "kernels.cuh"

namespace vaco {
namespace {

constexpr size_t kNoAllocStatusBytes = 256;
constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;

// Status word in the first 256 bytes, then the intermediate planes.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocStatusBytes + kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on `device` (current), looked up once.
cudaError_t scratch_address(int device, unsigned char** out) {
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[device] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_ptr[device];
    return cudaSuccess;
}

unsigned long long key_of(unsigned stage, unsigned long long position, unsigned msg) {
    return ((unsigned long long)stage << 60) | ((position & ((1ull << 52) - 1)) << 8) | msg;
}

bool depth_ok(int bd) { return bd == 8 || bd == 10 || bd == 12; }
size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Carves pictures out of the scratch array (pitch rounded to 64 samples,
// every plane 256-byte aligned).
struct Carver {
    unsigned char* base;
    size_t used = 0, cap;
    bool take(int w, int h, DevPlane* out) {
        const int pitch = (int)round_up((size_t)(w > 0 ? w : 1), 64);
        const size_t bytes = round_up((size_t)pitch * (size_t)(h > 0 ? h : 1) * 2, 256);
        if (used + bytes > cap) return false;
        *out = DevPlane{reinterpret_cast<uint16_t*>(base + used), w, h, pitch};
        used += bytes;
        return true;
    }
};

bool job_geometry_ok(const vaco_av1_frame_job& j) {
    const vaco_av1_frame_info& i = j.info;
    if (i.mi_rows <= 0 || i.mi_cols <= 0 || i.mi_rows > (1 << 15) || i.mi_cols > (1 << 15)) return false;
    // 4:4:0 is refused as the context entry points refuse it: AV1 cannot
    // signal it, and the chain's tile layout assumes it away.
    if (!av1_subsampling_ok(i.subsampling_x, i.subsampling_y)) return false;
    if (i.coded_width <= 0 || i.coded_height <= 0) return false;
    if (i.mi_cols != 2 * ((i.coded_width + 7) >> 3) || i.mi_rows != 2 * ((i.coded_height + 7) >> 3)) return false;
    if (i.upscaled_width < i.coded_width) return false;
    const int np = i.monochrome ? 1 : 3;
    if (np > 1 && ((i.subsampling_x && ((i.coded_width | i.upscaled_width) & 1)) ||
                   (i.subsampling_y && (i.coded_height & 1))))
        return false;
    for (int k = 0; k < np; ++k) {
        const int sx = k ? i.subsampling_x : 0, sy = k ? i.subsampling_y : 0;
        if (!j.src.planes[k] || j.src.width[k] != (i.mi_cols * 4) >> sx || j.src.height[k] != (i.mi_rows * 4) >> sy ||
            j.src.stride[k] < j.src.width[k])
            return false;
        if (!j.dst.planes[k] || j.dst.width[k] != (i.upscaled_width >> sx) || j.dst.height[k] != (i.coded_height >> sy) ||
            j.dst.stride[k] < j.dst.width[k])
            return false;
    }
    return true;
}

int32_t fail(int32_t* msg, int32_t status, int m) {
    if (msg) *msg = m;
    return status;
}

}  // namespace
}  // namespace vaco

using namespace vaco;

extern "C" int32_t vaco_av1_postfilter_frame_noalloc(void* stream, const vaco_av1_frame_job* job, int32_t* msg) {
    if (!job) return fail(msg, VACO_AV1_INVALID_DATA, VACO_AV1_MSG_NULL_ARGUMENT);
    const vaco_av1_frame_job& J = *job;
    if (!job_geometry_ok(J)) return fail(msg, VACO_AV1_INVALID_DATA, VACO_AV1_MSG_FRAME_GEOMETRY);
    const vaco_av1_frame_info& info = J.info;
    const int np = info.monochrome ? 1 : 3;
    const int ssx = info.subsampling_x, ssy = info.subsampling_y;
    const bool superres = info.upscaled_width != info.coded_width;
    bool lr_active = false;
    for (int k = 0; k < np; ++k) lr_active = lr_active || J.lr_type[k] != VACO_AV1_FRAME_LR_NONE;

    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    unsigned char* base = nullptr;
    if (e == cudaSuccess) e = scratch_address(device, &base);
    if (e != cudaSuccess) return fail(msg, VACO_AV1_DEVICE_ERROR, VACO_AV1_MSG_CUDA);
    cudaStream_t s = (cudaStream_t)stream;
    DeviceStatus* status = reinterpret_cast<DeviceStatus*>(base);

    // Intermediate pictures inside the fixed scratch (rejects frames that do not fit).
    Carver cv{base + kNoAllocStatusBytes, 0, kNoAllocScratchBytes};
    DevPlane pre[3], cdef[3], upre[3], ucdef[3];
    bool fits = true;
    for (int k = 0; k < np; ++k) {
        fits = fits && cv.take(J.src.width[k], J.src.height[k], &pre[k]) &&
               cv.take(J.src.width[k], J.src.height[k], &cdef[k]);
        if (superres) {
            const int sx = k ? ssx : 0, sy = k ? ssy : 0;
            const int w = (info.upscaled_width + sx) >> sx, h = (info.coded_height + sy) >> sy;
            fits = fits && cv.take(w, h, &ucdef[k]);
            if (lr_active) fits = fits && cv.take(w, h, &upre[k]);
        }
    }
    if (!fits) return fail(msg, VACO_AV1_LIMIT_EXCEEDED, VACO_AV1_MSG_SCRATCH_LIMIT);

    // Clear the status word before any kernel of this call.
    e = cudaMemsetAsync(status, 0xFF, sizeof(DeviceStatus), s);
    if (e != cudaSuccess) return fail(msg, VACO_AV1_DEVICE_ERROR, VACO_AV1_MSG_CUDA);
    unsigned long long host_key = kNoError;

    // ---- deblocking: src -> pre
    const vaco_av1_deblock_params& db = J.deblock;
    bool db_ok = depth_ok(info.bit_depth) && db.sharpness <= 7;
    for (int k = 0; k < 4; ++k) db_ok = db_ok && db.levels[k] <= 63;
    if (!db_ok || !J.tx_luma || (np > 1 && !J.tx_chroma)) {
        host_key = key_of(STAGE_DEBLOCK, 0, db_ok ? VACO_AV1_MSG_NULL_ARGUMENT : VACO_AV1_MSG_DB_PARAMS);
    } else {
        DevPlaneC sp[3];
        for (int k = 0; k < np; ++k) sp[k] = DevPlaneC{J.src.planes[k], J.src.width[k], J.src.height[k], J.src.stride[k]};
        const long n_luma = (long)info.mi_rows * info.mi_cols;
        const long n_chroma = np > 1 ? (long)((info.mi_rows + ssy) >> ssy) * ((info.mi_cols + ssx) >> ssx) : 0;
        e = launch_deblock_prepare(sp, pre, np, info.bit_depth, J.tx_luma, n_luma, J.tx_chroma, n_chroma, J.lvl_map,
                                   status, s);
        if (e == cudaSuccess) {
            DeblockLaunch L;
            for (int k = 0; k < 3; ++k) L.pic[k] = k < np ? pre[k] : DevPlane{nullptr, 0, 0, 0};
            L.num_planes = np;
            L.ssx = ssx;
            L.ssy = ssy;
            L.bit_depth = info.bit_depth;
            L.mi_rows = info.mi_rows;
            L.mi_cols = info.mi_cols;
            L.coded_width = info.coded_width;
            L.coded_height = info.coded_height;
            L.tx_luma = J.tx_luma;
            L.tx_chroma = J.tx_chroma;
            L.lvl_map = J.lvl_map;
            for (int k = 0; k < 4; ++k) L.levels[k] = db.levels[k];
            L.sharpness = db.sharpness;
            e = launch_deblock_passes(L, s);
        }
    }
    if (e != cudaSuccess) return fail(msg, VACO_AV1_DEVICE_ERROR, VACO_AV1_MSG_CUDA);

    // ---- CDEF: pre -> cdef
    vaco_av1_picture pre_pic{}, cdef_pic{};
    for (int k = 0; k < np; ++k) {
        pre_pic.planes[k] = pre[k].data;
        pre_pic.width[k] = pre[k].width;
        pre_pic.height[k] = pre[k].height;
        pre_pic.stride[k] = pre[k].stride;
        cdef_pic.planes[k] = cdef[k].data;
        cdef_pic.width[k] = cdef[k].width;
        cdef_pic.height[k] = cdef[k].height;
        cdef_pic.stride[k] = cdef[k].stride;
    }
    if (host_key == kNoError) {
        const vaco_av1_cdef_params& cp = J.cdef;
        bool all_zero = true;
        for (int k = 0; k < 8; ++k)
            all_zero = all_zero && cp.y_primary[k] == 0 && cp.y_secondary[k] == 0 && cp.uv_primary[k] == 0 &&
                       cp.uv_secondary[k] == 0;
        if (!cp.enabled || all_zero) {
            for (int k = 0; k < np && e == cudaSuccess; ++k)
                e = cudaMemcpy2DAsync(cdef[k].data, (size_t)cdef[k].stride * 2, pre[k].data, (size_t)pre[k].stride * 2,
                                      (size_t)pre[k].width * 2, pre[k].height, cudaMemcpyDeviceToDevice, s);
        } else if (!J.skip || (!J.cdef_idx && J.cdef_count > 0)) {
            host_key = key_of(STAGE_CDEF, 0, VACO_AV1_MSG_NULL_ARGUMENT);
        } else {
            CdefLaunch L;
            L.src = pre_pic;
            L.dst = cdef_pic;
            L.info = info;
            L.skip = J.skip;
            L.cdef_idx = J.cdef_idx;
            L.cdef_stride = J.cdef_stride;
            L.cdef_count = J.cdef_idx ? J.cdef_count : 0;
            L.params = cp;
            L.status = status;
            e = launch_cdef_frame(L, s);
        }
    }
    if (e != cudaSuccess) return fail(msg, VACO_AV1_DEVICE_ERROR, VACO_AV1_MSG_CUDA);

    // ---- superres of the CDEF picture (and of the pre-CDEF picture for restoration)
    DevPlane* before = pre;
    DevPlane* after = cdef;
    if (host_key == kNoError && superres) {
        SuperresPlane sp[2 * 3];
        int nsp = np;
        for (int k = 0; k < np; ++k) {
            const int sx = k ? ssx : 0, sy = k ? ssy : 0;
            sp[k].in = DevPlaneC{cdef[k].data, cdef[k].width, cdef[k].height, cdef[k].stride};
            sp[k].out = ucdef[k];
            sp[k].visible_width = (info.coded_width + sx) >> sx;
            sp[k].output_width = (info.upscaled_width + sx) >> sx;
            sp[k].height = (info.coded_height + sy) >> sy;
        }
        after = ucdef;
        if (lr_active) {  // the pre-CDEF picture too, in the same launch
            for (int k = 0; k < np; ++k) {
                sp[np + k] = sp[k];
                sp[np + k].in = DevPlaneC{pre[k].data, pre[k].width, pre[k].height, pre[k].stride};
                sp[np + k].out = upre[k];
            }
            nsp = 2 * np;
            before = upre;
        }
        e = launch_superres(sp, nsp, info.bit_depth, status, STAGE_SUPERRES, s);
        if (e != cudaSuccess) return fail(msg, VACO_AV1_DEVICE_ERROR, VACO_AV1_MSG_CUDA);
    }

    // ---- restoration (or the visible copy) into the caller's output
    if (host_key == kNoError) {
        LrPlane lp[3];
        int nlr = 0;
        for (int k = 0; k < np && host_key == kNoError; ++k) {
            const int sx = k ? ssx : 0, sy = k ? ssy : 0;
            const int w = info.upscaled_width >> sx, h = info.coded_height >> sy;
            const unsigned long long plane_pos = (unsigned long long)k << 44;
            if (J.lr_type[k] == VACO_AV1_FRAME_LR_NONE) {  // copy_visible_plane, as copy-only tiles
                lp[nlr++] = copy_only_plane(DevPlaneC{after[k].data, after[k].width, after[k].height, after[k].stride},
                                            DevPlane{J.dst.planes[k], w, h, J.dst.stride[k]}, w, h, (k && ssy) ? 1 : 0,
                                            k);
                continue;
            }
            const int unit = J.lr_unit_size[k];
            if (unit == 0) {
                host_key = key_of(STAGE_LR, plane_pos, VACO_AV1_MSG_LR_NO_UNIT_SIZE);
                break;
            }
            if (!(unit == 32 || unit == 64 || unit == 128 || unit == 256)) {
                host_key = key_of(STAGE_LR, plane_pos | (1ull << 40), VACO_AV1_MSG_LR_GEOMETRY);
                break;
            }
            const int cols = (w + unit / 2) / unit < 1 ? 1 : (w + unit / 2) / unit;
            const int rows = (h + unit / 2) / unit < 1 ? 1 : (h + unit / 2) / unit;
            if ((long)cols * rows != J.lr_unit_count[k] || !J.lr_units[k]) {
                host_key = key_of(STAGE_LR, plane_pos | (2ull << 40),
                                  J.lr_units[k] ? VACO_AV1_MSG_LR_UNIT_COUNT : VACO_AV1_MSG_NULL_ARGUMENT);
                break;
            }
            e = launch_lr_unit_check(J.lr_units[k], J.lr_unit_count[k], k, status, s);
            if (e != cudaSuccess) return fail(msg, VACO_AV1_DEVICE_ERROR, VACO_AV1_MSG_CUDA);
            LrPlane& p = lp[nlr++];
            p.before = DevPlaneC{before[k].data, before[k].width, before[k].height, before[k].stride};
            p.before_rows = DevPlaneC{nullptr, 0, 0, 0};
            p.plane_index = k;
            p.unit_status = nullptr;  // validated by the unit check above
            p.after = DevPlaneC{after[k].data, after[k].width, after[k].height, after[k].stride};
            p.out = DevPlane{J.dst.planes[k], w, h, J.dst.stride[k]};
            p.width = w;
            p.height = h;
            p.unit_size = unit;
            p.sub_y = (k && ssy) ? 1 : 0;
            p.units = J.lr_units[k];
            p.unit_cols = cols;
            p.unit_rows = rows;
            p.copy_only = 0;
        }
        if (host_key == kNoError && nlr > 0) {
            e = launch_restoration(lp, nlr, info.bit_depth, s);
            if (e != cudaSuccess) return fail(msg, VACO_AV1_DEVICE_ERROR, VACO_AV1_MSG_CUDA);
        }
    }

    // ---- read the status word into a host variable (no pinned allocation)
    unsigned long long key = kNoError;
    e = cudaMemcpyAsync(&key, status, sizeof(key), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(msg, VACO_AV1_DEVICE_ERROR, VACO_AV1_MSG_CUDA);
    if (host_key < key) key = host_key;
    if (key == kNoError) return fail(msg, VACO_AV1_OK, VACO_AV1_MSG_NONE);
    return fail(msg, VACO_AV1_INVALID_DATA, (int)(key & 0xFF));
}
