// superres.cu -- AV1 horizontal super-resolution (spec 7.16) on sm_100a.
//
// Mirrors vaco crates/codec/vaco-codec-av1/src/superres.rs:145-216
// (subpel_start, upscale_plane).  One CTA upscales a 256-sample stretch of
// one output row: it stages the source span its taps can reach in shared
// memory (edge-clamped to the Mi-padded width, as vaco clamps each tap),
// then every thread evaluates one output sample's eight taps from there.
#include "common.cuh"
#include "kernels.cuh"

namespace vaco {

namespace {

// Upscale_Filter (AV1 7.16) phases 0..32; phase 64-p is phase p reversed.
__constant__ int16_t c_upscale_half[33][8] = {
    {0, 0, 0, 128, 0, 0, 0, 0},        {0, 0, -1, 128, 2, -1, 0, 0},
    {0, 1, -3, 127, 4, -2, 1, 0},      {0, 1, -4, 127, 6, -3, 1, 0},
    {0, 2, -6, 126, 8, -3, 1, 0},      {0, 2, -7, 125, 11, -4, 1, 0},
    {-1, 2, -8, 125, 13, -5, 2, 0},    {-1, 3, -9, 124, 15, -6, 2, 0},
    {-1, 3, -10, 123, 18, -6, 2, -1},  {-1, 3, -11, 122, 20, -7, 3, -1},
    {-1, 4, -12, 121, 22, -8, 3, -1},  {-1, 4, -13, 120, 25, -9, 3, -1},
    {-1, 4, -14, 118, 28, -9, 3, -1},  {-1, 4, -15, 117, 30, -10, 4, -1},
    {-1, 5, -16, 116, 32, -11, 4, -1}, {-1, 5, -16, 114, 35, -12, 4, -1},
    {-1, 5, -17, 112, 38, -12, 4, -1}, {-1, 5, -18, 111, 40, -13, 5, -1},
    {-1, 5, -18, 109, 43, -14, 5, -1}, {-1, 6, -19, 107, 45, -14, 5, -1},
    {-1, 6, -19, 105, 48, -15, 5, -1}, {-1, 6, -19, 103, 51, -16, 5, -1},
    {-1, 6, -20, 101, 53, -16, 6, -1}, {-1, 6, -20, 99, 56, -17, 6, -1},
    {-1, 6, -20, 97, 58, -17, 6, -1},  {-1, 6, -20, 95, 61, -18, 6, -1},
    {-2, 7, -20, 93, 64, -18, 6, -2},  {-2, 7, -20, 91, 66, -19, 6, -1},
    {-2, 7, -20, 88, 69, -19, 6, -1},  {-2, 7, -20, 86, 71, -19, 6, -1},
    {-2, 7, -20, 84, 74, -20, 7, -2},  {-2, 7, -20, 81, 76, -20, 7, -1},
    {-2, 7, -20, 79, 79, -20, 7, -2},
};

constexpr int kSrThreads = 256;
constexpr int kSrMaxSpan = 2 * kSrThreads + 16;  // source span for ratios down to 1/2

struct SrArgs {
    SuperresPlane p[3];
    int bit_depth;
    DeviceStatus* status;
    unsigned stage;
};

__global__ void __launch_bounds__(kSrThreads) superres_kernel(SrArgs a) {
    __shared__ int16_t s_coef[64][8];
    __shared__ uint16_t s_src[kSrMaxSpan];
    const SuperresPlane& P = a.p[blockIdx.z];
    const int y = blockIdx.y;
    if (y >= P.height) return;
    const int tid = threadIdx.x;
    for (int i = tid; i < 64 * 8; i += kSrThreads) {
        int ph = i >> 3, t = i & 7;
        s_coef[ph][t] = ph <= 32 ? c_upscale_half[ph][t] : c_upscale_half[64 - ph][7 - t];
    }
    // step and initial phase (superres.rs:168-169, :145-152)
    const long long vis = P.visible_width, outw = P.output_width;
    const int step = (int)(((vis << 14) + outw / 2) / outw);
    const long long err = outw * step - (vis << 14);
    const int init =
        (int)(((-((outw - vis) << 13) + outw / 2) / outw + (1 << 7) - err / 2) & ((1 << 14) - 1));
    const int x_first = blockIdx.x * kSrThreads;
    if (x_first >= P.output_width) return;
    const int x_last = min(x_first + kSrThreads, P.output_width) - 1;
    const int first_src = ((-(1 << 14) + init + x_first * step) >> 14) - 3;
    const int last_src = ((-(1 << 14) + init + x_last * step) >> 14) + 4;
    const int span = last_src - first_src + 1;  // <= kSrMaxSpan while output >= input
    const uint16_t* row = P.in.data + (long)y * P.in.stride;
    const int maxv = (1 << a.bit_depth) - 1;
    for (int i = tid; i < span; i += kSrThreads) s_src[i] = __ldg(row + clampi(first_src + i, 0, P.in.width - 1));
    __syncthreads();
    const int x = x_first + tid;
    if (x > x_last) return;
    const int src_x = -(1 << 14) + init + x * step;
    const int base = (src_x >> 14) - 3 - first_src;
    const int phase = (src_x & 0x3FFF) >> 8;
    int sum = 0;
    bool bad = false;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        int s = s_src[base + t];
        bad |= s > maxv;
        sum += s * s_coef[phase][t];
    }
    if (bad) report_error(a.status, a.stage, (unsigned long long)y * P.output_width + x, VACO_AV1_MSG_SR_SAMPLE);
    int v = (sum + 64) >> 7;
    P.out.data[(long)y * P.out.stride + x] = (uint16_t)clampi(v, 0, maxv);
}

}  // namespace

cudaError_t launch_superres(const SuperresPlane* planes, int count, int bit_depth, DeviceStatus* status,
                            unsigned stage, cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    SrArgs a;
    int max_w = 0, max_h = 0;
    for (int k = 0; k < count; ++k) {
        a.p[k] = planes[k];
        max_w = max(max_w, planes[k].output_width);
        max_h = max(max_h, planes[k].height);
    }
    a.bit_depth = bit_depth;
    a.status = status;
    a.stage = stage;
    if (max_w <= 0 || max_h <= 0) return cudaSuccess;  // nothing to upscale
    dim3 grid(div_up(max_w, kSrThreads), max_h, count);
    superres_kernel<<<grid, kSrThreads, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace vaco
