// superres.cu -- AV1 horizontal super-resolution (spec 7.16) on sm_100a.
//
// Mirrors vaco crates/codec/vaco-codec-av1/src/superres.rs:145-216
// (subpel_start, upscale_plane).
#include "common.cuh"
#include "kernels.cuh"

namespace vaco {

namespace {

// Upscale_Filter (AV1 7.16) phases 0..32; phase 64-p is phase p reversed.
constexpr int16_t kUpscaleHalf[33][8] = {
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

constexpr int kSrThreads = 256;  // output columns per CTA
constexpr int kSrRows = 8;       // output rows per CTA, a multiple of 8
constexpr int kSrGroups = kSrRows / 8;  // 16-byte words per staged column
static_assert(kSrRows % 8 == 0, "a staged column is whole 16-byte words of 8 rows");
// The source span 256 output columns reach: step <= 1 << 14 (the output is
// never narrower than the input), so at most 255 steps plus the 8 taps, and
// one more column when the span is widened to start on an even column.
constexpr int kSrMaxSpan = kSrThreads + 16;

// The 64 filter phases, phase 64-p being phase p reversed, one 32-bit word
// per tap holding the coefficient as a byte at bits 0-7 and again at bits
// 24-31: dp2a.lo of a word of two samples (rows 2k, 2k+1) with it gives
// row 2k's product, dp2a.hi row 2k+1's.  Taps 3 and 4 lie in [0, 128] and
// are read unsigned; the other taps lie in [-20, 7] and are read signed.
struct alignas(16) SrCoefTable {
    uint32_t w[64][8];
};
constexpr int sr_coef(int ph, int t) { return ph <= 32 ? kUpscaleHalf[ph][t] : kUpscaleHalf[64 - ph][7 - t]; }
constexpr bool sr_coefs_fit_bytes() {
    for (int ph = 0; ph < 64; ++ph)
        for (int t = 0; t < 8; ++t) {
            const int c = sr_coef(ph, t);
            if ((t == 3 || t == 4) ? (c < 0 || c > 255) : (c < -128 || c > 127)) return false;
        }
    return true;
}
static_assert(sr_coefs_fit_bytes(), "upscale taps must fit the byte operands of dp2a");
constexpr SrCoefTable make_sr_coefs() {
    SrCoefTable tab{};
    for (int ph = 0; ph < 64; ++ph)
        for (int t = 0; t < 8; ++t) {
            const uint32_t b = (uint32_t)sr_coef(ph, t) & 0xFFu;
            tab.w[ph][t] = b | (b << 24);
        }
    return tab;
}
__device__ const SrCoefTable g_sr_coef = make_sr_coefs();

__device__ __forceinline__ int sr_tap(uint32_t w, int t) {  // the coefficient back from its word
    return (t == 3 || t == 4) ? (int)(w & 0xFFu) : (int)(int8_t)(w & 0xFFu);
}

// One plane, with the step and initial subpixel position computed once on
// the host (superres.rs:168-169, :145-152), and its CTAs in the flattened
// grid: first_block, col_blocks and a reciprocal of col_blocks.
struct SrPlane {
    SuperresPlane p;
    int step, init;
    int col_blocks;
    unsigned col_recip;  // fast_div_recip(col_blocks)
    int first_block;
    int pairs;           // rows can be read as aligned 32-bit pairs of samples
};

struct SrArgs {
    SrPlane p[kSuperresMaxPlanes];
    int count;
    int bit_depth;
    DeviceStatus* status;
    unsigned stage;
};

// A CTA computes 256 output columns of kSrRows rows of one plane.
//
// Staging: the source span those columns reach, widened to start on an even
// column, is read as 32-bit pairs of samples (edge-clamped per sample, as
// vaco clamps each tap, where the span crosses the Mi-padded width), every
// row's load issued before the first is used, and stored column-major: a
// 16-byte word holds 8 rows of one source column.  A tap is then one
// shared-memory load per 8 rows and one dp2a per row; each thread takes its
// output column's phase and eight coefficients once.
//
// vaco's per-tap range check (a sample above the bit depth is an error at
// the first output that reads it) runs, with plain multiply-adds, only in
// CTAs whose staged span holds such a sample.
__global__ void __launch_bounds__(kSrThreads) superres_kernel(SrArgs a) {
    __shared__ uint4 s_col[kSrMaxSpan][kSrGroups];
    overlap_prologue();
    const int blk_all = blockIdx.x;
    int k = 0;
    while (k + 1 < a.count && blk_all >= a.p[k + 1].first_block) ++k;
    const SrPlane& S = a.p[k];
    const SuperresPlane& P = S.p;
    const unsigned blk = blk_all - S.first_block;
    const unsigned row_block = fast_div(blk, S.col_blocks, S.col_recip);
    const int y0 = row_block * kSrRows;
    const int x_first = (blk - row_block * S.col_blocks) * kSrThreads;
    const int tid = threadIdx.x;
    const int rows = min(kSrRows, P.height - y0);
    const int x_last = min(x_first + kSrThreads, P.output_width) - 1;
    const int first_src = (((-(1 << 14) + S.init + x_first * S.step) >> 14) - 3) & ~1;
    const int last_src = ((-(1 << 14) + S.init + x_last * S.step) >> 14) + 4;
    const int npairs = (last_src - first_src + 2) >> 1;  // <= kSrMaxSpan / 2 <= kSrThreads
    const int maxv = (1 << a.bit_depth) - 1;
    uint32_t any = 0;
    if (tid < npairs) {
        const int c = first_src + 2 * tid;
        const uint16_t* row0 = P.in.data + (long)y0 * P.in.stride;
        uint32_t w[kSrRows];
        if (S.pairs && c >= 0 && c + 1 < P.in.width) {
            const uint32_t* q = reinterpret_cast<const uint32_t*>(row0 + c);
            const int st = P.in.stride >> 1;
#pragma unroll
            for (int r = 0; r < kSrRows; ++r) w[r] = r < rows ? __ldg(q + (long)r * st) : 0u;
        } else {
            const int c0 = clampi(c, 0, P.in.width - 1), c1 = clampi(c + 1, 0, P.in.width - 1);
#pragma unroll
            for (int r = 0; r < kSrRows; ++r)
                w[r] = r < rows ? __ldg(row0 + (long)r * P.in.stride + c0) |
                                      (uint32_t)__ldg(row0 + (long)r * P.in.stride + c1) << 16
                                : 0u;
        }
#pragma unroll
        for (int g = 0; g < kSrGroups; ++g) {
            const uint32_t* v = w + 8 * g;
            s_col[2 * tid][g] = make_uint4(__byte_perm(v[0], v[1], 0x5410), __byte_perm(v[2], v[3], 0x5410),
                                           __byte_perm(v[4], v[5], 0x5410), __byte_perm(v[6], v[7], 0x5410));
            s_col[2 * tid + 1][g] = make_uint4(__byte_perm(v[0], v[1], 0x7632), __byte_perm(v[2], v[3], 0x7632),
                                               __byte_perm(v[4], v[5], 0x7632), __byte_perm(v[6], v[7], 0x7632));
        }
#pragma unroll
        for (int r = 0; r < kSrRows; ++r) any |= w[r];
    }
    const int x = x_first + tid;
    int base = 0;
    uint32_t cw[8];
    if (x <= x_last) {
        const int src_x = -(1 << 14) + S.init + x * S.step;
        base = (src_x >> 14) - 3 - first_src;
        const uint4* c = reinterpret_cast<const uint4*>(g_sr_coef.w[(src_x & 0x3FFF) >> 8]);
        const uint4 lo = __ldg(c), hi = __ldg(c + 1);
        cw[0] = lo.x, cw[1] = lo.y, cw[2] = lo.z, cw[3] = lo.w;
        cw[4] = hi.x, cw[5] = hi.y, cw[6] = hi.z, cw[7] = hi.w;
    }
    const uint32_t in_range = (uint32_t)maxv | (uint32_t)maxv << 16;
    const bool check = __syncthreads_or((any & ~in_range) != 0);
    if (x > x_last) return;
    uint16_t* out = P.out.data + (long)y0 * P.out.stride + x;
    if (!check) {
        // Every sample is within the bit depth (< 2^12): the signed 16-bit
        // reading of dp2a sees it exactly.
#pragma unroll
        for (int g = 0; g < kSrGroups; ++g) {
            int sum[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) sum[r] = 64;
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                const uint4 q = s_col[base + t][g];
                const uint32_t wq[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    if (t == 3 || t == 4) {
                        sum[2 * h] = (int)__dp2a_lo(wq[h], cw[t], (unsigned)sum[2 * h]);
                        sum[2 * h + 1] = (int)__dp2a_hi(wq[h], cw[t], (unsigned)sum[2 * h + 1]);
                    } else {
                        sum[2 * h] = __dp2a_lo((int)wq[h], (int)cw[t], sum[2 * h]);
                        sum[2 * h + 1] = __dp2a_hi((int)wq[h], (int)cw[t], sum[2 * h + 1]);
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < 8; ++r)
                if (8 * g + r < rows) out[(long)(8 * g + r) * P.out.stride] = (uint16_t)clampi(sum[r] >> 7, 0, maxv);
        }
        return;
    }
    for (int r = 0; r < rows; ++r) {
        int sum = 0;
        bool bad = false;
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const int v = reinterpret_cast<const uint16_t*>(&s_col[base + t][r >> 3])[r & 7];
            bad |= v > maxv;
            sum += v * sr_tap(cw[t], t);
        }
        const int y = y0 + r;
        if (bad) report_error(a.status, a.stage, (unsigned long long)y * P.output_width + x, VACO_AV1_MSG_SR_SAMPLE);
        out[(long)r * P.out.stride] = (uint16_t)clampi((sum + 64) >> 7, 0, maxv);
    }
}

}  // namespace

cudaError_t launch_superres(const SuperresPlane* planes, int count, int bit_depth, DeviceStatus* status,
                            unsigned stage, cudaStream_t stream) {
    if (count <= 0 || count > kSuperresMaxPlanes) return count == 0 ? cudaSuccess : cudaErrorInvalidValue;
    SrArgs a;
    long long blocks = 0;
    for (int k = 0; k < count; ++k) {
        const SuperresPlane& P = planes[k];
        a.p[k].p = P;
        // step and initial phase (superres.rs:168-169, :145-152)
        const long long vis = P.visible_width, outw = P.output_width;
        const long long step = outw > 0 ? ((vis << 14) + outw / 2) / outw : 0;
        const long long err = outw * step - (vis << 14);
        if (step > (1 << 14)) return cudaErrorInvalidValue;  // narrower output: outside the staged span
        a.p[k].step = (int)step;
        a.p[k].init = outw > 0 ? (int)(((-((outw - vis) << 13) + outw / 2) / outw + (1 << 7) - err / 2) & ((1 << 14) - 1))
                               : 0;
        const int cols = P.output_width > 0 && P.height > 0 ? div_up(P.output_width, kSrThreads) : 0;
        a.p[k].col_blocks = cols > 0 ? cols : 1;
        a.p[k].col_recip = fast_div_recip((unsigned)a.p[k].col_blocks);
        a.p[k].first_block = (int)blocks;
        a.p[k].pairs = reinterpret_cast<uintptr_t>(P.in.data) % 4 == 0 && P.in.stride % 2 == 0;
        blocks += (long long)cols * (cols > 0 ? div_up(P.height, kSrRows) : 0);
    }
    if (blocks >= (1LL << 31)) return cudaErrorInvalidValue;  // fast_div needs n < 2^31
    a.count = count;
    a.bit_depth = bit_depth;
    a.status = status;
    a.stage = stage;
    if (blocks == 0) return cudaSuccess;  // nothing to upscale
    return launch_overlapped(superres_kernel, dim3((unsigned)blocks), dim3(kSrThreads), 0, stream, a);
}

}  // namespace vaco
