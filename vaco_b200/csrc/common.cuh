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

// Stage numbers order errors across the chain (deblock -> CDEF -> superres ->
// LR), then film grain, which runs on the chain's output.
enum Stage : unsigned { STAGE_DEBLOCK = 0, STAGE_CDEF = 1, STAGE_SUPERRES = 2, STAGE_LR = 3, STAGE_GRAIN = 4 };

__device__ __forceinline__ void report_error(DeviceStatus* st, unsigned stage,
                                             unsigned long long position, unsigned msg) {
    unsigned long long key = ((unsigned long long)stage << 60) | ((position & ((1ull << 52) - 1)) << 8) | msg;
    atomicMin(&st->first_error, key);
}

// ---------------------------------------------------------------- overlapped launches
//
// The chain's kernels (fused deblock+CDEF, superres, restoration) are
// launched with programmatic stream serialization: a kernel may be scheduled
// while the kernel before it on the stream runs its last CTAs.  Each of them
// calls overlap_prologue() before anything else.  It first lets the next
// kernel on the stream be scheduled the same way, then waits until the
// previous kernel has completed and its writes are visible, so every read and
// write after it is ordered exactly as with a plain launch.  Only the launch
// latency and the CTA start-up overlap the previous kernel's tail.  Without
// the launch attribute both instructions are no-ops.  While the stream is
// being captured into a CUDA graph the launch is a plain one, so captured
// graphs hold only ordinary dependencies.
__device__ __forceinline__ void overlap_prologue() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

template <typename... Params, typename... Args>
inline cudaError_t launch_overlapped(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem,
                                     cudaStream_t stream, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    const bool plain = cudaStreamIsCapturing(stream, &capture) != cudaSuccess || capture != cudaStreamCaptureStatusNone;
    cfg.attrs = attr;
    cfg.numAttrs = plain ? 0 : 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
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
// log2 of Tx_Width / Tx_Height per TX_SIZE (AV1 §6.10.19 ordering), packed
// 3 bits per size (log2 - 2) into one 64-bit immediate, so a lookup with a
// per-lane size is a shift and a mask.  Sizes past the table (invalid input,
// which the callers report) read as the last entry.
struct TxLog2Table {
    int w[19], h[19];
};
constexpr TxLog2Table kTxLog2 = {{2, 3, 4, 5, 6, 2, 3, 3, 4, 4, 5, 5, 6, 2, 4, 3, 5, 4, 6},
                                 {2, 3, 4, 5, 6, 3, 2, 4, 3, 5, 4, 6, 5, 4, 2, 5, 3, 6, 4}};
__host__ __device__ constexpr unsigned long long tx_log2_packed(bool height) {
    unsigned long long m = 0;
    for (int t = 0; t < 19; ++t) m |= (unsigned long long)((height ? kTxLog2.h[t] : kTxLog2.w[t]) - 2) << (3 * t);
    return m;
}
__host__ __device__ inline int tx_w_log2(int t) {
    constexpr unsigned long long m = tx_log2_packed(false);
    return (int)((m >> (3 * (t < 18 ? t : 18))) & 7u) + 2;
}
__host__ __device__ inline int tx_h_log2(int t) {
    constexpr unsigned long long m = tx_log2_packed(true);
    return (int)((m >> (3 * (t < 18 ? t : 18))) & 7u) + 2;
}

inline int div_up(int a, int b) { return (a + b - 1) / b; }

// n / d for 0 <= n < 2^31 and d >= 1 without a division instruction sequence:
// recip = floor((2^32 - 1) / d) makes umulhi(n, recip) either n / d or one
// less (the error n / 2^32 stays below one half), and one compare fixes it.
inline unsigned fast_div_recip(unsigned d) { return 0xFFFFFFFFu / (d ? d : 1u); }
__device__ __forceinline__ unsigned fast_div(unsigned n, unsigned d, unsigned recip) {
    unsigned q = __umulhi(n, recip);
    if ((q + 1) * d <= n) ++q;
    return q;
}

// The frame of tile t in a batch whose frames' tiles are laid end to end:
// the last f in [0, n) with prefix[f] <= t (prefix holds n + 1 running tile
// counts, prefix[0] = 0; a frame without tiles is never picked, since the
// next frame starts at the same count).  Every thread of a CTA searches the
// same entries, so the loads are broadcasts.
__device__ __forceinline__ int frame_of_tile(const int* __restrict__ prefix, int n, int t) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Chroma layouts AV1 can signal (color_config, spec 5.5.2): 4:2:0, 4:2:2 and
// 4:4:4.  subsampling_y is only coded when subsampling_x is 1, so 4:4:0 does
// not exist; the fused deblock+CDEF tile layout relies on that.
inline bool av1_subsampling_ok(int ssx, int ssy) {
    return (ssx == 0 || ssx == 1) && (ssy == 0 || ssy == 1) && !(ssx == 0 && ssy == 1);
}

}  // namespace vaco
