// common.cuh -- shared device helpers for the sm_100a AV1 post-filter kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/vaco_av1_gpu.h"

namespace vaco {

// ---------------------------------------------------------------- status word
//
// Data checks that vaco performs while it filters (sample ranges, strength
// indices, ...) are reported through one 64-bit status word per context:
//   bits 63..8  ordering key (stage, then the raster position vaco would have
//               reached the failing check at), bits 7..0  vaco_av1_msg
// Kernels atomicMin it, so the host reads the error vaco itself would have
// returned first.  ~0 means "no error".
struct DeviceStatus {
    unsigned long long first_error;
};

constexpr unsigned long long kNoError = ~0ull;

// Stage numbers order errors across the chain (deblock -> CDEF -> superres -> LR).
enum Stage : unsigned { STAGE_DEBLOCK = 0, STAGE_CDEF = 1, STAGE_SUPERRES = 2, STAGE_LR = 3 };

__device__ __forceinline__ void report_error(DeviceStatus* st, unsigned stage,
                                             unsigned long long position, unsigned msg) {
    unsigned long long key = ((unsigned long long)stage << 60) | ((position & ((1ull << 52) - 1)) << 8) | msg;
    atomicMin(&st->first_error, key);
}

// ---------------------------------------------------------------- planes

struct DevPlane {
    uint16_t* data;
    int width, height, stride;
};

struct DevPlaneC {
    const uint16_t* data;
    int width, height, stride;
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return min(max(v, lo), hi); }

// framebuf::Plane::get_clamped (vaco src/framebuf.rs:50-59)
__device__ __forceinline__ int get_clamped(const DevPlaneC& p, int x, int y) {
    x = clampi(x, 0, p.width - 1);
    y = clampi(y, 0, p.height - 1);
    return __ldg(p.data + (long)y * p.stride + x);
}

__device__ __forceinline__ int round2(int v, int shift) { return shift == 0 ? v : (v + (1 << (shift - 1))) >> shift; }

// AV1 TX_SIZE enum -> log2 width / height
__host__ __device__ constexpr int tx_w_log2(int t) {
    return t == 0 ? 2 : t == 1 ? 3 : t == 2 ? 4 : t == 3 ? 5 : t == 4 ? 6 : t == 5 ? 2 : t == 6 ? 3
         : t == 7 ? 3 : t == 8 ? 4 : t == 9 ? 4 : t == 10 ? 5 : t == 11 ? 5 : t == 12 ? 6 : t == 13 ? 2
         : t == 14 ? 4 : t == 15 ? 3 : t == 16 ? 5 : t == 17 ? 4 : 6;
}
__host__ __device__ constexpr int tx_h_log2(int t) {
    return t == 0 ? 2 : t == 1 ? 3 : t == 2 ? 4 : t == 3 ? 5 : t == 4 ? 6 : t == 5 ? 3 : t == 6 ? 2
         : t == 7 ? 4 : t == 8 ? 3 : t == 9 ? 5 : t == 10 ? 4 : t == 11 ? 6 : t == 12 ? 5 : t == 13 ? 4
         : t == 14 ? 2 : t == 15 ? 5 : t == 16 ? 3 : t == 17 ? 6 : 4;
}

inline int div_up(int a, int b) { return (a + b - 1) / b; }

// Chroma layouts AV1 can signal (color_config, spec 5.5.2): 4:2:0, 4:2:2 and
// 4:4:4.  subsampling_y is only coded when subsampling_x is 1, so 4:4:0 does
// not exist; the fused deblock+CDEF tile layout relies on that.
inline bool av1_subsampling_ok(int ssx, int ssy) {
    return (ssx == 0 || ssx == 1) && (ssy == 0 || ssy == 1) && !(ssx == 0 && ssy == 1);
}

}  // namespace vaco
