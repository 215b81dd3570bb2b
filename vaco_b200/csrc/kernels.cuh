// kernels.cuh -- launchers of the post-filter kernels (host side, internal).
#pragma once

#include "common.cuh"

namespace vaco {

// ---------------------------------------------------------------- CDEF
struct CdefLaunch {
    vaco_av1_picture src;  // device planes
    vaco_av1_picture dst;
    vaco_av1_frame_info info;
    const uint8_t* skip;
    const int32_t* cdef_idx;
    int cdef_stride, cdef_count;
    vaco_av1_cdef_params params;
    DeviceStatus* status;
};
cudaError_t launch_cdef_frame(const CdefLaunch& L, cudaStream_t stream);
cudaError_t launch_find_direction(const uint16_t* blocks, int n, int bit_depth, uint8_t* dirs, uint32_t* vars,
                                  DeviceStatus* status, cudaStream_t stream);
cudaError_t launch_filter_block(const uint16_t* inputs, const vaco_av1_cdef_filter_params* params, int n,
                                uint16_t* outputs, DeviceStatus* status, cudaStream_t stream);

// ---------------------------------------------------------------- superres
struct SuperresPlane {
    DevPlaneC in;        // Mi-padded input
    DevPlane out;        // output_width x height
    int visible_width;
    int output_width;
    int height;
};
// Upscales up to kSuperresMaxPlanes planes in one launch (a picture's planes
// and, for restoration, its pre-CDEF boundary rows).
constexpr int kSuperresMaxPlanes = 6;
cudaError_t launch_superres(const SuperresPlane* planes, int count, int bit_depth, DeviceStatus* status,
                            unsigned stage, cudaStream_t stream);

// ---------------------------------------------------------------- film grain
// Film grain synthesis (AV1 7.18.3) of an np-plane frame of w x h luma
// samples from `in` into `out`; `gauss` is the 2048-entry Gaussian table in
// host memory (copied into the launch).  `workspace` holds
// film_grain_workspace_bytes(np, w, h) bytes.
// launch_grain_template fills the workspace from the parameters alone;
// launch_grain_apply reads it.
size_t film_grain_workspace_bytes(int np, int w, int h);
cudaError_t launch_grain_template(const vaco_av1_film_grain_params& p, const int16_t* gauss, int np, int bd,
                                  int sub_x, int sub_y, int w, int h, void* workspace, cudaStream_t stream);
cudaError_t launch_grain_apply(const vaco_av1_film_grain_params& p, const DevPlaneC* in, const DevPlane* out,
                               int np, int bd, int sub_x, int sub_y, int w, int h, const void* workspace,
                               DeviceStatus* status, int sm_count, cudaStream_t stream);

// ---------------------------------------------------------------- frame emission
// One plane of pic_to_frame / blit (src/decode.rs:3795-3891): `width` x
// `height` samples of `src` (stride in samples) packed into `dst` (stride in
// bytes), one byte per sample or, with two_bytes, a little-endian u16.
struct EmitPlane {
    const uint16_t* src;
    int src_stride;
    uint8_t* dst;
    long long dst_stride;
    int width, height;
};
cudaError_t launch_emit(const EmitPlane* planes, int count, int two_bytes, int sm_count, cudaStream_t stream);

// ---------------------------------------------------------------- restoration
struct LrPlane {
    DevPlaneC before;
    // When before_rows.data is set, the pre-CDEF picture is read from this
    // compact buffer instead of `before`: 4 rows per stripe boundary k, rows
    // (k*stripe - offset) - 2 .. +1 at indices 4k .. 4k+3 (as written by the
    // fused deblock+CDEF kernel).
    DevPlaneC before_rows;
    DevPlaneC after;
    DevPlane out;
    int width, height, unit_size, sub_y;
    const vaco_av1_lr_unit* units;  // device
    int unit_cols, unit_rows;
    int copy_only;                  // 1: output = `after` (frame-level restoration off for the plane)
    int plane_index;                // 0 = Y, 1 = U, 2 = V (status-word key of unit checks)
    DeviceStatus* unit_status;      // non-null: validate each tile's unit here (restoration.rs:67-91)
};
// A plane whose restoration is off: its tiles only copy `after` into `out`.
LrPlane copy_only_plane(const DevPlaneC& after, const DevPlane& out, int w, int h, int sub_y, int plane_index);
// Restores up to 3 planes in one launch.  Units must have been validated.
cudaError_t launch_restoration(const LrPlane* planes, int count, int bit_depth, cudaStream_t stream);
// Batched form (see launch_dbcdef_batch): per-frame records of lr_args_size()
// bytes built by build_lr_args (which returns the frame's tile count).
size_t lr_args_size();
int build_lr_args(const LrPlane* planes, int count, int bit_depth, void* out);
cudaError_t launch_restoration_batch(const void* dev_args, const int* dev_prefix, int n, int tiles, int ctas_per_sm,
                                     cudaStream_t stream);
// Shared-memory opt-ins of every kernel on the current device (idempotent);
// call before stream capture.
cudaError_t dbcdef_kernel_attributes();
cudaError_t lr_kernel_attributes();
inline cudaError_t kernel_attributes() {
    cudaError_t e = dbcdef_kernel_attributes();
    return e == cudaSuccess ? lr_kernel_attributes() : e;
}

// Reports VACO_AV1_MSG_LR_COEFFICIENT for the first invalid unit of `plane`,
// keyed after that plane's geometry/count checks and before its sample checks.
cudaError_t launch_lr_unit_check(const vaco_av1_lr_unit* units, int n, int plane, DeviceStatus* status,
                                 cudaStream_t stream);
// LR status-key positions: plane, then the check restore_plane runs first.
__host__ __device__ inline unsigned long long lr_key_position(int plane, unsigned check, unsigned long long index) {
    return ((unsigned long long)plane << 44) | ((unsigned long long)check << 40) | index;
}
enum LrCheckOrder : unsigned { LRC_NO_UNIT_SIZE = 0, LRC_GEOMETRY = 1, LRC_COUNT = 2, LRC_COEFFICIENT = 3, LRC_SAMPLE = 4 };

// ---------------------------------------------------------------- range checks / copies
// Reports `msg` at (stage, `position`) if any sample of the w x h region exceeds max.
cudaError_t launch_range_check(const DevPlaneC& p, int w, int h, int max_value, DeviceStatus* status,
                               unsigned stage, unsigned long long position, unsigned msg, cudaStream_t stream);

// ---------------------------------------------------------------- deblocking
struct DeblockLaunch {
    DevPlane pic[3];          // filtered in place (caller copied the source in)
    int num_planes, ssx, ssy, bit_depth;
    int mi_rows, mi_cols, coded_width, coded_height;
    const uint8_t* tx_luma;   // device
    const uint8_t* tx_chroma; // device
    const uint8_t* lvl_map;   // device or null
    uint8_t levels[4];
    int sharpness;
};
// Copies src to dst and checks samples (DB_SAMPLE) and side info (DB_PARAMS).
cudaError_t launch_deblock_prepare(const DevPlaneC* src, const DevPlane* dst, int num_planes, int bit_depth,
                                   const uint8_t* tx_luma, long n_luma, const uint8_t* tx_chroma, long n_chroma,
                                   const uint8_t* lvl_map, DeviceStatus* status, cudaStream_t stream);
cudaError_t launch_deblock_passes(const DeblockLaunch& L, cudaStream_t stream);

// ---------------------------------------------------------------- fused deblock + CDEF
// The final output of a plane without restoration in a frame without
// superres, written by the fused deblock+CDEF kernel itself instead of
// copied from the CDEF picture afterwards.
struct DirectPlane {
    DevPlane out;                    // visible output extent; data null: off
};

struct DbCdefLaunch {
    vaco_av1_picture src;       // reconstruction (device)
    vaco_av1_picture dst;       // CDEF output (device, same extents)
    DevPlane pre_rows[3];       // compact stripe-boundary rows (data may be null)
    vaco_av1_frame_info info;
    const uint8_t* tx_luma;
    const uint8_t* tx_chroma;
    const uint8_t* lvl_map;
    vaco_av1_deblock_params deblock;
    const uint8_t* skip;
    const int32_t* cdef_idx;
    int cdef_stride, cdef_count;
    vaco_av1_cdef_params cdef;
    DeviceStatus* status;
    int threads = 256;          // threads per tile: 256 or 128
    DirectPlane direct[3] = {};  // per plane; all off unless set
};
cudaError_t launch_dbcdef(const DbCdefLaunch& L, cudaStream_t stream);
// Batched form: `dev_args` holds n per-frame argument records (dbcdef_args_size()
// bytes each, built by build_dbcdef_args), `dev_prefix` n+1 running tile
// counts; one CTA per tile of all n frames (`tiles` = dev_prefix[n]).
// `ctas_per_sm` (resident CTAs per SM the body is compiled for, i.e. its
// register budget), `threads` (per tile, 256 or 128) and `layout` (the
// frames' common chroma layout, ssx | ssy << 1 with monochrome as 0, or -1
// when they differ) pick the kernel body.
size_t dbcdef_args_size();
size_t build_dbcdef_args(const DbCdefLaunch& L, void* out);  // returns dynamic smem bytes
inline int dbcdef_tiles(const vaco_av1_frame_info& i) { return ((i.mi_cols + 15) / 16) * ((i.mi_rows + 15) / 16); }
cudaError_t launch_dbcdef_batch(const void* dev_args, const int* dev_prefix, int n, int tiles, size_t smem,
                                int ctas_per_sm, int threads, int layout, cudaStream_t stream);
// Rows in the compact boundary buffer of a plane of `height` rows.
inline int pre_rows_count(int height, int sub_y) {
    const int sh = 64 >> sub_y, off = 8 >> sub_y;
    return 4 * ((height + off + 2) / sh + 1);
}
// Rows of that buffer the fused kernel writes: indices [4, 4 + n) hold the
// plane rows k*stripe - offset - 2 + sub (k >= 1, sub < 4) that lie inside
// the plane; restoration reads no other index.
inline int pre_rows_written(int height, int sub_y) {
    const int sh = 64 >> sub_y, off = 8 >> sub_y;
    int n = 0;
    for (int i = 4; i < pre_rows_count(height, sub_y); ++i)
        if ((i >> 2) * sh - off - 2 + (i & 3) < height) ++n;
    return n;
}

}  // namespace vaco
