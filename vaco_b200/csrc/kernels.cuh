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
// Upscales up to 3 planes in one launch (grid.z = plane).
cudaError_t launch_superres(const SuperresPlane* planes, int count, int bit_depth, DeviceStatus* status,
                            unsigned stage, cudaStream_t stream);

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
};
// Restores up to 3 planes in one launch.  Units must have been validated.
cudaError_t launch_restoration(const LrPlane* planes, int count, int bit_depth, cudaStream_t stream);
// Reports VACO_AV1_MSG_LR_COEFFICIENT for the first invalid unit (key order:
// before any sample error).
cudaError_t launch_lr_unit_check(const vaco_av1_lr_unit* units, int n, DeviceStatus* status, cudaStream_t stream);

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
};
cudaError_t launch_dbcdef(const DbCdefLaunch& L, cudaStream_t stream);
// Rows in the compact boundary buffer of a plane of `height` rows.
inline int pre_rows_count(int height, int sub_y) {
    const int sh = 64 >> sub_y, off = 8 >> sub_y;
    return 4 * ((height + off + 2) / sh + 1);
}

}  // namespace vaco
