// vaco_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of vaco's scalar AV1 post-filter path, used as the checker
// for the CUDA library and as the timed CPU baseline.  Nothing in the product
// (vaco_b200/) links or calls this file.  Paths are relative to the vaco
// repository (crates/codec/vaco-codec-av1/ unless stated otherwise).
//
//   CDEF          src/cdef.rs:68-230 and the frame pass src/decode.rs:739-896
//   superres      src/superres.rs:124-216
//   restoration   src/restoration.rs:67-384
//   planes        src/framebuf.rs:50-69 (get_clamped / set)
//   deblocking    AV1 spec section 7.14 (vaco has no deblocking filter:
//                 src/lib.rs:16-18).  Parity of this part is unpinned: no
//                 vaco code or golden vector exists for it.
//   film grain    AV1 spec section 7.18.3 (vaco parses the parameters,
//                 src/frame_header.rs:1125-1210, but has no synthesis).
//                 Parity unpinned for the same reason.
//
// The restated parts are pinned by the dav1d golden vectors vaco checks in
// (tests/golden/ holds copies; tests/test_oracle_golden.py replays them).
//
// Every entry point returns a message id (0 = success) from
// include/vaco_av1_gpu.h's vaco_av1_msg, so results compare one-to-one with
// the CUDA library's statuses.

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "../include/vaco_av1_gpu.h"

namespace {

// ------------------------------------------------------------------ planes

// framebuf::Plane (src/framebuf.rs:16-74) over caller memory with a pitch.
struct PlaneRef {
    const uint16_t* data;
    int width, height, stride;
    // get_clamped (src/framebuf.rs:50-59): clamp both coordinates.
    uint16_t get_clamped(long x, long y) const {
        long max_x = width > 0 ? width - 1 : 0;
        long max_y = height > 0 ? height - 1 : 0;
        long cx = std::min(std::max(x, 0L), max_x);
        long cy = std::min(std::max(y, 0L), max_y);
        if (width <= 0 || height <= 0) return 0;
        return data[cy * (long)stride + cx];
    }
};

struct PlaneMut {
    uint16_t* data;
    int width, height, stride;
    // set (src/framebuf.rs:61-69): writes outside the plane are ignored.
    void set(long x, long y, uint16_t v) {
        if (x >= 0 && y >= 0 && x < width && y < height) data[y * (long)stride + x] = v;
    }
    PlaneRef ref() const { return PlaneRef{data, width, height, stride}; }
};

int ilog2_u32(uint32_t v) { return 31 - __builtin_clz(v); }

// Run fn(lo, hi, slot) over [0, n) split into `threads` contiguous ranges
// (slot = the range's index).  Callers flatten 2-D work (rows x column
// blocks) in raster order, so a thin band still spreads over every thread
// and each range's first error is its earliest in raster order.
template <class F>
void parallel_for(long n, int threads, F fn) {
    if (threads <= 1 || n < 2L * threads) {
        fn(0L, n, 0);
        return;
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) {
        long lo = n * t / threads, hi = n * (t + 1) / threads;
        pool.emplace_back([=] { fn(lo, hi, t); });
    }
    for (auto& th : pool) th.join();
}

// ------------------------------------------------------------------ CDEF

// (row, column) offsets per direction and distance, AV1 7.15.3 (src/cdef.rs:57-66).
const int kCdefDir[8][2][2] = {
    {{-1, 1}, {-2, 2}}, {{0, 1}, {-1, 2}}, {{0, 1}, {0, 2}},  {{0, 1}, {1, 2}},
    {{1, 1}, {2, 2}},   {{1, 0}, {2, 1}},  {{1, 0}, {2, 0}},  {{1, 0}, {2, -1}},
};

// coefficient_shift (src/cdef.rs:68-73).
int cdef_shift(int bit_depth, int* shift) {
    if (bit_depth == 8 || bit_depth == 10 || bit_depth == 12) {
        *shift = bit_depth - 8;
        return 0;
    }
    return VACO_AV1_MSG_CDEF_BIT_DEPTH;
}

// find_direction (src/cdef.rs:79-124).
int find_direction(const uint16_t* block, int bit_depth, uint8_t* dir_out, uint32_t* var_out) {
    int shift;
    if (int m = cdef_shift(bit_depth, &shift)) return m;
    int32_t partial[8][15];
    uint32_t counts[8][15];
    std::memset(partial, 0, sizeof partial);
    std::memset(counts, 0, sizeof counts);
    for (int index = 0; index < 64; ++index) {
        uint32_t sample = block[index];
        if (sample >= (1u << bit_depth)) return VACO_AV1_MSG_CDEF_SAMPLE;
        int i = index / 8, j = index % 8;
        int bins[8] = {i + j, i + j / 2, i, 3 + i - j / 2, 7 + i - j, 3 + j - i / 2, j, i / 2 + j};
        int value = (int)(sample >> shift) - 128;
        for (int d = 0; d < 8; ++d) {
            partial[d][bins[d]] += value;
            counts[d][bins[d]] += 1;
        }
    }
    int64_t costs[8] = {0};
    for (int d = 0; d < 8; ++d)
        for (int b = 0; b < 15; ++b) {
            uint32_t count = counts[d][b];
            if (count != 0) {
                int64_t sum = partial[d][b];
                costs[d] += sum * sum * (int64_t)(840u / count);
            }
        }
    int best = 0;
    for (int d = 1; d < 8; ++d)
        if (costs[d] > costs[best]) best = d;
    *dir_out = (uint8_t)best;
    int64_t v = (costs[best] - costs[(best + 4) & 7]) >> 10;
    *var_out = (v < 0 || v > 0xffffffffLL) ? 0u : (uint32_t)v;
    return 0;
}

// constrain (src/cdef.rs:126-133).
int constrain(int difference, int threshold, int damping) {
    if (threshold == 0) return 0;
    int shift = std::max(0, damping - ilog2_u32((uint32_t)threshold));
    int magnitude = std::abs(difference);
    int sign = (difference > 0) - (difference < 0);
    return sign * std::min(magnitude, std::max(0, threshold - (magnitude >> shift)));
}

// filter_block (src/cdef.rs:142-205).
int filter_block(const uint16_t* input, const vaco_av1_cdef_filter_params& p, uint16_t* output) {
    int shift;
    if (int m = cdef_shift(p.bit_depth, &shift)) return m;
    bool bad = !(p.width == 4 || p.width == 8) || !(p.height == 4 || p.height == 8) ||
               p.direction > 7 || p.edges > 15 || p.damping > 12 || p.primary > (15 << shift) ||
               p.secondary > (4 << shift);
    for (int k = 0; k < 144 && !bad; ++k)
        if (input[k] >= (1u << p.bit_depth)) bad = true;
    if (bad) return VACO_AV1_MSG_CDEF_BLOCK_PARAMS;
    std::memset(output, 0, 64 * sizeof(uint16_t));
    int primary_taps[2];
    if (((p.primary >> shift) & 1) == 0) {
        primary_taps[0] = 4;
        primary_taps[1] = 2;
    } else {
        primary_taps[0] = 3;
        primary_taps[1] = 3;
    }
    int x_min = (p.edges & 1) ? -2 : 0;
    int x_max = p.width + ((p.edges & 2) ? 2 : 0);
    int y_min = (p.edges & 4) ? -2 : 0;
    int y_max = p.height + ((p.edges & 8) ? 2 : 0);
    for (int y = 0; y < p.height; ++y)
        for (int x = 0; x < p.width; ++x) {
            int current = input[(y + 2) * 12 + x + 2];
            int minimum = current, maximum = current, sum = 0;
            for (int distance = 0; distance < 2; ++distance)
                for (int sign = -1; sign <= 1; sign += 2) {
                    int dirs[3] = {p.direction, (p.direction + 6) & 7, (p.direction + 2) & 7};
                    int strengths[3] = {p.primary, p.secondary, p.secondary};
                    int taps[3] = {primary_taps[distance], 2 - distance, 2 - distance};
                    for (int k = 0; k < 3; ++k) {
                        int dy = kCdefDir[dirs[k]][distance][0];
                        int dx = kCdefDir[dirs[k]][distance][1];
                        int nx = x + sign * dx, ny = y + sign * dy;
                        if (nx < x_min || nx >= x_max || ny < y_min || ny >= y_max) continue;
                        int neighbor = input[(ny + 2) * 12 + nx + 2];
                        minimum = std::min(minimum, neighbor);
                        maximum = std::max(maximum, neighbor);
                        sum += taps[k] * constrain(neighbor - current, strengths[k], p.damping);
                    }
                }
            int filtered = current + ((8 + sum - (sum < 0 ? 1 : 0)) >> 4);
            filtered = std::min(std::max(filtered, minimum), maximum);
            output[y * 8 + x] = (uint16_t)filtered;
        }
    return 0;
}

// adjust_strength (src/cdef.rs:209-220).
int adjust_strength(int primary, uint32_t variance) {
    if (variance == 0) return 0;
    uint32_t scaled = variance >> 6;
    uint32_t log = scaled == 0 ? 0 : std::min<uint32_t>(ilog2_u32(scaled), 12);
    return (int)(((uint32_t)primary * (4 + log) + 8) >> 4);
}

// chroma_direction (src/cdef.rs:224-230).
int chroma_direction(int direction, bool sub_x, bool sub_y) {
    static const int k10[8] = {7, 0, 2, 4, 5, 6, 6, 6};
    static const int k01[8] = {1, 2, 2, 2, 3, 4, 6, 0};
    if (sub_x && !sub_y) return k10[direction & 7];
    if (!sub_x && sub_y) return k01[direction & 7];
    return direction & 7;
}

// apply_cdef (src/decode.rs:739-862) with cdef_block_skipped (:892-896).
// `dst` must already hold a copy of `src` (apply_cdef copies first, :749-767).
int cdef_frame(const PlaneRef src[3], PlaneMut dst[3], int num_planes,
               const vaco_av1_frame_info& info, const uint8_t* skip, const int32_t* cdef_idx,
               int cdef_stride, int cdef_count, const vaco_av1_cdef_params& params, int threads) {
    bool all_zero = true;
    for (int k = 0; k < 8; ++k)
        all_zero = all_zero && params.y_primary[k] == 0 && params.y_secondary[k] == 0 &&
                   params.uv_primary[k] == 0 && params.uv_secondary[k] == 0;
    if (!params.enabled || all_zero) return 0;
    const int shift = info.bit_depth - 8;
    const int mi_rows = info.mi_rows, mi_cols = info.mi_cols;
    const int block_rows = (mi_rows + 1) / 2;
    // The reference stops at the first error in raster order; each worker
    // records its first error and the earliest one wins.
    std::vector<long> first_key(threads > 0 ? threads : 1, -1);
    std::vector<int> first_msg(first_key.size(), 0);
    const int block_cols = (mi_cols + 1) / 2;
    auto work = [&](long lo, long hi, int slot) {
        for (long i = lo; i < hi; ++i) {
            const int r = (int)(i / block_cols) * 2, c = (int)(i % block_cols) * 2;
            {
                long sidx = (long)(r >> 4) * cdef_stride + (c >> 4);
                int index = (sidx >= 0 && sidx < cdef_count) ? cdef_idx[sidx] : -1;
                auto skipped = [&](int row, int col) {
                    return row < mi_rows && col < mi_cols && skip[(long)row * mi_cols + col] != 0;
                };
                bool block_skipped =
                    skipped(r, c) && skipped(r + 1, c) && skipped(r, c + 1) && skipped(r + 1, c + 1);
                if (index < 0 || block_skipped) continue;
                auto fail = [&](int m, int stage) {
                    first_key[slot] = ((long)r * mi_cols + c) * 4 + stage;
                    first_msg[slot] = m;
                };
                uint16_t luma[64];
                for (int i = 0; i < 64; ++i) luma[i] = src[0].get_clamped(c * 4 + i % 8, r * 4 + (i >> 3));
                uint8_t direction;
                uint32_t variance;
                if (int m = find_direction(luma, info.bit_depth, &direction, &variance)) {
                    fail(m, 0);
                    return;
                }
                for (int pl = 0; pl < num_planes; ++pl) {
                    bool chroma = pl != 0;
                    int sx = chroma && info.subsampling_x, sy = chroma && info.subsampling_y;
                    int x = (c * 4) >> sx, y = (r * 4) >> sy, width = 8 >> sx, height = 8 >> sy;
                    if (index >= 8) {
                        fail(VACO_AV1_MSG_CDEF_STRENGTH_INDEX, 1 + pl);
                        return;
                    }
                    int sp = chroma ? params.uv_primary[index] : params.y_primary[index];
                    int ss = chroma ? params.uv_secondary[index] : params.y_secondary[index];
                    int primary = (uint16_t)(sp << shift);
                    int secondary = (uint16_t)(ss << shift);
                    int chosen = primary == 0 ? 0
                                 : chroma     ? chroma_direction(direction, info.subsampling_x,
                                                                 info.subsampling_y)
                                              : direction;
                    if (!chroma) primary = adjust_strength(primary, variance);
                    uint16_t hood[144];
                    std::memset(hood, 0, sizeof hood);
                    for (int ny = 0; ny < height + 4; ++ny)
                        for (int nx = 0; nx < width + 4; ++nx)
                            hood[ny * 12 + nx] = src[pl].get_clamped(x + nx - 2, y + ny - 2);
                    vaco_av1_cdef_filter_params fp;
                    fp.width = (uint8_t)width;
                    fp.height = (uint8_t)height;
                    fp.edges = (uint8_t)((x > 0) | ((x + width < src[pl].width) << 1) | ((y > 0) << 2) |
                                         ((y + height < src[pl].height) << 3));
                    fp.bit_depth = (uint8_t)info.bit_depth;
                    fp.direction = (uint8_t)chosen;
                    fp.primary = (uint16_t)primary;
                    fp.secondary = (uint16_t)secondary;
                    fp.damping = (uint8_t)(params.damping + shift - (chroma ? 1 : 0));
                    uint16_t out[64];
                    if (int m = filter_block(hood, fp, out)) {
                        fail(m, 1 + pl);
                        return;
                    }
                    for (int oy = 0; oy < height; ++oy)
                        for (int ox = 0; ox < width; ++ox) dst[pl].set(x + ox, y + oy, out[oy * 8 + ox]);
                }
            }
        }
    };
    parallel_for((long)block_rows * block_cols, (int)first_key.size(), work);
    long best = -1;
    int msg = 0;
    for (size_t t = 0; t < first_key.size(); ++t)
        if (first_key[t] >= 0 && (best < 0 || first_key[t] < best)) {
            best = first_key[t];
            msg = first_msg[t];
        }
    return msg;
}

// ------------------------------------------------------------------ superres

// AV1 7.16 Upscale_Filter, phases 0..32.  Phase 64-p is phase p reversed
// (the spec table is mirror-symmetric), so phases 33..63 are derived.
const int16_t kUpscaleHalf[33][8] = {
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

int upscale_tap(int phase, int tap) {
    return phase <= 32 ? kUpscaleHalf[phase][tap] : kUpscaleHalf[64 - phase][7 - tap];
}

// subpel_start (src/superres.rs:145-152).
int64_t subpel_start(int64_t vis, int64_t out, int64_t step) {
    int64_t error = out * step - (vis << 14);
    int64_t start = (-((out - vis) << 13) + out / 2) / out + (1 << 7) - error / 2;
    return start & ((1 << 14) - 1);
}

// upscale_plane (src/superres.rs:163-216), validate (:128-143).
int upscale_plane(const PlaneRef& in, int visible_width, int output_width, int height,
                  int bit_depth, PlaneMut out, int threads) {
    if (!(bit_depth == 8 || bit_depth == 10 || bit_depth == 12)) return VACO_AV1_MSG_SR_BIT_DEPTH;
    if (visible_width == 0 || output_width <= visible_width || height == 0 ||
        visible_width > in.width || height > in.height || visible_width < 0 || height < 0)
        return VACO_AV1_MSG_SR_GEOMETRY;
    const int64_t vis = visible_width, outw = output_width, padded = in.width;
    const int64_t step = ((vis << 14) + outw / 2) / outw;
    const int64_t init = subpel_start(vis, outw, step);
    const int64_t max_sample = (1LL << bit_depth) - 1;
    std::vector<long> first_row(threads > 1 ? threads : 1, -1);
    const long segs = (long)((outw + 255) / 256);  // 256-sample row segments
    auto work = [&](long lo, long hi, int slot) {
        for (long i = lo; i < hi; ++i) {
            const int y = (int)(i / segs);
            const int64_t x0 = (i % segs) * 256;
            for (int64_t x = x0; x < std::min(x0 + 256, outw); ++x) {
                int64_t src_x = -(1 << 14) + init + x * step;
                int64_t src_px = src_x >> 14;
                int phase = (int)((src_x & ((1 << 14) - 1)) >> 8);
                int64_t sum = 0;
                for (int t = 0; t < 8; ++t) {
                    int64_t sx = std::min(std::max(src_px + t - 3, (int64_t)0), padded - 1);
                    int64_t sample = in.data[(long)y * in.stride + sx];
                    if (sample > max_sample) {
                        first_row[slot] = y;
                        return;
                    }
                    sum += sample * upscale_tap(phase, t);
                }
                int64_t rounded = (sum + 64) >> 7;
                out.set(x, y, (uint16_t)std::min(std::max(rounded, (int64_t)0), max_sample));
            }
        }
    };
    parallel_for((long)height * segs, (int)first_row.size(), work);
    for (long r : first_row)
        if (r >= 0) return VACO_AV1_MSG_SR_SAMPLE;
    return 0;
}

// ------------------------------------------------------------------ restoration

// Sgr_Params as (radius, epsilon) per pass (src/restoration.rs:286-303).
const int kSgr[16][2][2] = {
    {{2, 12}, {1, 4}},  {{2, 15}, {1, 6}},  {{2, 18}, {1, 8}},  {{2, 21}, {1, 9}},
    {{2, 24}, {1, 10}}, {{2, 29}, {1, 11}}, {{2, 36}, {1, 12}}, {{2, 45}, {1, 13}},
    {{2, 56}, {1, 14}}, {{2, 68}, {1, 15}}, {{0, 0}, {1, 5}},   {{0, 0}, {1, 8}},
    {{0, 0}, {1, 11}},  {{0, 0}, {1, 14}},  {{2, 30}, {0, 0}},  {{2, 75}, {0, 0}},
};

int64_t round2(int64_t v, int shift) { return shift == 0 ? v : (v + (1LL << (shift - 1))) >> shift; }

// RestorationUnit::validate (src/restoration.rs:67-91).
bool unit_valid(const vaco_av1_lr_unit& u) {
    if (u.type == VACO_AV1_LR_NONE) return true;
    if (u.type == VACO_AV1_LR_WIENER) {
        const int lo[3] = {-5, -23, -17}, hi[3] = {10, 8, 46};
        for (int k = 0; k < 3; ++k) {
            if (u.vertical[k] < lo[k] || u.vertical[k] > hi[k]) return false;
            if (u.horizontal[k] < lo[k] || u.horizontal[k] > hi[k]) return false;
        }
        return true;
    }
    if (u.type == VACO_AV1_LR_SGRPROJ)
        return u.set >= 0 && u.set < 16 && u.xqd[0] >= -96 && u.xqd[0] <= 31 && u.xqd[1] >= -32 &&
               u.xqd[1] <= 95;
    return false;
}

struct LrConfig {
    int width, height, bit_depth, unit_size, sub_y;
    // unit_counts (src/restoration.rs:111-120).
    void counts(int* cols, int* rows) const {
        auto count = [&](long extent) {
            long c = unit_size ? (extent + unit_size / 2) / unit_size : 0;
            return (int)std::max(c, 1L);
        };
        *cols = count(width);
        *rows = count(height);
    }
    // unit_index (src/restoration.rs:124-133).
    int unit_index(int x, int y, int cols, int rows) const {
        int row = std::min((y + (8 >> sub_y)) / unit_size, rows - 1);
        int col = std::min(x / unit_size, cols - 1);
        return row * cols + col;
    }
};

// Source (src/restoration.rs:209-245).
struct Source {
    PlaneRef before, after;
    int width, height, stripe_start, stripe_end;
    Source(PlaneRef b, PlaneRef a, const LrConfig& cfg, int y) : before(b), after(a) {
        width = cfg.width;
        height = cfg.height;
        int stripe_height = 64 >> cfg.sub_y, offset = 8 >> cfg.sub_y;
        int stripe = (y + offset) / stripe_height;
        stripe_start = stripe * stripe_height - offset;
        stripe_end = stripe_start + stripe_height - 1;
    }
    int64_t get(int x, int y) const {
        x = std::min(std::max(x, 0), width - 1);
        y = std::min(std::max(y, 0), height - 1);
        if (y < stripe_start) return before.get_clamped(x, std::max(y, stripe_start - 2));
        if (y > stripe_end) return before.get_clamped(x, std::min(y, stripe_end + 2));
        return after.get_clamped(x, y);
    }
};

// wiener (src/restoration.rs:259-283).
int64_t wiener(const Source& s, int x, int y, const int16_t* vertical, const int16_t* horizontal,
               int depth) {
    int round_h = depth == 12 ? 5 : 3;
    int64_t offset = 1LL << (depth + 7 - round_h - 1);
    int64_t limit = (1LL << (depth + 1 + 7 - round_h)) - 1;
    auto taps = [](const int16_t* t, int64_t* out) {
        int64_t a = t[0], b = t[1], c = t[2];
        int64_t v[7] = {a, b, c, 128 - 2 * (a + b + c), c, b, a};
        std::memcpy(out, v, sizeof v);
    };
    int64_t hv[7], vv[7];
    taps(horizontal, hv);
    taps(vertical, vv);
    int64_t sum = 0;
    for (int row = 0; row < 7; ++row) {
        int64_t h = 0;
        for (int col = 0; col < 7; ++col) h += hv[col] * s.get(x + col - 3, y + row - 3);
        sum += vv[row] * std::min(std::max(round2(h, round_h), -offset), limit - offset);
    }
    return round2(sum, 14 - round_h);
}

// box_ab (src/restoration.rs:314-339).
void box_ab(const Source& s, int x, int y, int radius, int64_t epsilon, int depth, int64_t* a_out,
            int64_t* b_out) {
    int64_t n = (int64_t)(2 * radius + 1) * (2 * radius + 1);
    int64_t n2e = n * n * epsilon;
    int64_t scale = ((1LL << 20) + n2e / 2) / n2e;
    int64_t sum_sq = 0, sum = 0;
    for (int dy = -radius; dy <= radius; ++dy)
        for (int dx = -radius; dx <= radius; ++dx) {
            int64_t sample = s.get(x + dx, y + dy);
            sum_sq += sample * sample;
            sum += sample;
        }
    int64_t a = round2(sum_sq, 2 * (depth - 8));
    int64_t d = round2(sum, depth - 8);
    int64_t variance = std::max(a * n - d * d, (int64_t)0);
    int64_t z = round2(variance * scale, 20);
    int64_t a2 = z >= 255 ? 256 : z == 0 ? 1 : ((z << 8) + z / 2) / (z + 1);
    int64_t reciprocal = ((1LL << 12) + n / 2) / n;
    *a_out = a2;
    *b_out = round2((256 - a2) * sum * reciprocal, 12);
}

// guided_pass (src/restoration.rs:341-371).
int64_t guided_pass(const Source& s, int x, int y, int pass, int radius, int64_t epsilon, int depth) {
    int64_t original = s.after.get_clamped(x, y);
    if (radius == 0) return original << 4;
    int64_t a = 0, b = 0;
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
            int64_t weight;
            if (pass == 0)
                weight = ((y + dy) & 1) == 0 ? 0 : dx == 0 ? 6 : 5;
            else
                weight = (dx == 0 || dy == 0) ? 4 : 3;
            if (weight != 0) {
                int64_t aa, bb;
                box_ab(s, x + dx, y + dy, radius, epsilon, depth, &aa, &bb);
                a += weight * aa;
                b += weight * bb;
            }
        }
    int shift = (pass == 0 && (y & 1) != 0) ? 4 : 5;
    return round2(a * original + b, 8 + shift - 4);
}

// self_guided (src/restoration.rs:373-384).
int64_t self_guided(const Source& s, int x, int y, int set, const int16_t* xqd, int depth) {
    int64_t w0 = xqd[0], w1 = xqd[1];
    int64_t original = (int64_t)s.after.get_clamped(x, y) << 4;
    int64_t first = guided_pass(s, x, y, 0, kSgr[set][0][0], kSgr[set][0][1], depth);
    int64_t second = guided_pass(s, x, y, 1, kSgr[set][1][0], kSgr[set][1][1], depth);
    return round2(w0 * first + w1 * original + (128 - w0 - w1) * second, 11);
}

// restore_plane (src/restoration.rs:178-207) with PlaneConfig::validate (:135-168).
int restore_plane(const PlaneRef& before, const PlaneRef& after, const LrConfig& cfg,
                  const vaco_av1_lr_unit* units, int unit_count, PlaneMut out, int threads) {
    bool depth_ok = cfg.bit_depth == 8 || cfg.bit_depth == 10 || cfg.bit_depth == 12;
    bool size_ok = cfg.unit_size == 32 || cfg.unit_size == 64 || cfg.unit_size == 128 ||
                   cfg.unit_size == 256;
    if (!depth_ok || !size_ok || cfg.width <= 0 || cfg.height <= 0 || cfg.width > before.width ||
        cfg.width > after.width || cfg.height > before.height || cfg.height > after.height)
        return VACO_AV1_MSG_LR_GEOMETRY;
    int cols, rows;
    cfg.counts(&cols, &rows);
    if ((long)cols * rows != unit_count) return VACO_AV1_MSG_LR_UNIT_COUNT;
    for (int i = 0; i < unit_count; ++i)
        if (!unit_valid(units[i])) return VACO_AV1_MSG_LR_COEFFICIENT;
    const uint16_t max = (uint16_t)((1u << cfg.bit_depth) - 1);
    for (const PlaneRef* p : {&before, &after})
        for (int y = 0; y < cfg.height; ++y)
            for (int x = 0; x < cfg.width; ++x)
                if (p->get_clamped(x, y) > max) return VACO_AV1_MSG_LR_SAMPLE;
    const long segs = (cfg.width + 63) / 64;  // 64-sample row segments
    parallel_for((long)cfg.height * segs, threads, [&](long lo, long hi, int) {
        for (long i = lo; i < hi; ++i) {
            const int y = (int)(i / segs), x0 = (int)(i % segs) * 64;
            Source src(before, after, cfg, y);
            for (int x = x0; x < std::min(x0 + 64, cfg.width); ++x) {
                const vaco_av1_lr_unit& u = units[cfg.unit_index(x, y, cols, rows)];
                int64_t value;
                if (u.type == VACO_AV1_LR_WIENER)
                    value = wiener(src, x, y, u.vertical, u.horizontal, cfg.bit_depth);
                else if (u.type == VACO_AV1_LR_SGRPROJ)
                    value = self_guided(src, x, y, u.set, u.xqd, cfg.bit_depth);
                else
                    value = after.get_clamped(x, y);
                value = std::min(std::max(value, (int64_t)0), (int64_t)max);
                out.set(x, y, (uint16_t)value);
            }
        }
    });
    return 0;
}

// ------------------------------------------------------------------ deblocking (AV1 7.14)

// Tx_Width / Tx_Height for the AV1 TX_SIZE enum.
const int kTxW[19] = {4, 8, 16, 32, 64, 4, 8, 8, 16, 16, 32, 32, 64, 4, 16, 8, 32, 16, 64};
const int kTxH[19] = {4, 8, 16, 32, 64, 8, 4, 16, 8, 32, 16, 64, 32, 16, 4, 32, 8, 64, 16};

struct Strength {
    int lvl, limit, blimit, thresh;
};

// 7.14.4 limit/blimit/thresh from a level and loop_filter_sharpness.
Strength filter_strength(int lvl, int sharpness) {
    int shift = sharpness > 4 ? 2 : sharpness > 0 ? 1 : 0;
    int limit = sharpness > 0 ? std::min(std::max(lvl >> shift, 1), 9 - sharpness)
                              : std::max(1, lvl >> shift);
    Strength s;
    s.lvl = lvl;
    s.limit = limit;
    s.blimit = 2 * (lvl + 2) + limit;
    s.thresh = lvl >> 4;
    return s;
}

struct Deblocker {
    const vaco_av1_frame_info& info;
    const uint8_t* tx_luma;
    const uint8_t* tx_chroma;
    const uint8_t* lvl_map;
    const vaco_av1_deblock_params& params;
    int cmi_rows, cmi_cols;

    int level(int plane, int pass, int row, int col) const {
        int i = plane == 0 ? pass : plane + 1;
        if (lvl_map) return lvl_map[((long)row * info.mi_cols + col) * 4 + i];
        return params.levels[i];
    }
    int tx(int plane, int r, int c) const {
        if (plane == 0) return tx_luma[(long)r * info.mi_cols + c];
        return tx_chroma[(long)r * cmi_cols + c];
    }

    // 7.14.6.2-7.14.6.4 on one line of samples across an edge.  get(k) reads
    // the sample k positions past the edge (k < 0 is the p side).
    template <class Get, class Put>
    void filter_line(Get get, Put put, int plane, int filter_size, const Strength& s) const {
        const int bd = info.bit_depth;
        int q[7], p[7];
        int reach = filter_size == 16 ? 7 : 4;
        for (int k = 0; k < reach; ++k) {
            q[k] = get(k);
            p[k] = get(-k - 1);
        }
        int filter_len = filter_size == 4 ? 4 : plane != 0 ? 6 : filter_size == 8 ? 8 : 16;
        int limit_bd = s.limit << (bd - 8), blimit_bd = s.blimit << (bd - 8);
        int thresh_bd = s.thresh << (bd - 8);
        bool hev = std::abs(p[1] - p[0]) > thresh_bd || std::abs(q[1] - q[0]) > thresh_bd;
        bool mask = std::abs(p[1] - p[0]) > limit_bd || std::abs(q[1] - q[0]) > limit_bd ||
                    std::abs(p[0] - q[0]) * 2 + std::abs(p[1] - q[1]) / 2 > blimit_bd;
        if (filter_len >= 6)
            mask = mask || std::abs(p[2] - p[1]) > limit_bd || std::abs(q[2] - q[1]) > limit_bd;
        if (filter_len >= 8)
            mask = mask || std::abs(p[3] - p[2]) > limit_bd || std::abs(q[3] - q[2]) > limit_bd;
        if (mask) return;
        int one = 1 << (bd - 8);
        bool flat = false, flat2 = false;
        if (filter_size >= 8) {
            bool f = std::abs(p[1] - p[0]) > one || std::abs(q[1] - q[0]) > one ||
                     std::abs(p[2] - p[0]) > one || std::abs(q[2] - q[0]) > one;
            if (filter_len >= 8) f = f || std::abs(p[3] - p[0]) > one || std::abs(q[3] - q[0]) > one;
            flat = !f;
        }
        if (filter_size >= 16) {
            bool f = std::abs(p[6] - p[0]) > one || std::abs(q[6] - q[0]) > one ||
                     std::abs(p[5] - p[0]) > one || std::abs(q[5] - q[0]) > one ||
                     std::abs(p[4] - p[0]) > one || std::abs(q[4] - q[0]) > one;
            flat2 = !f;
        }
        if (filter_size == 4 || !flat) {
            // 7.14.6.3 narrow filter.
            int half = 0x80 << (bd - 8);
            int lo = -(1 << (bd - 1)), hi = (1 << (bd - 1)) - 1;
            auto c4 = [&](int v) { return std::min(std::max(v, lo), hi); };
            int ps1 = p[1] - half, ps0 = p[0] - half, qs0 = q[0] - half, qs1 = q[1] - half;
            int filter = hev ? c4(ps1 - qs1) : 0;
            filter = c4(filter + 3 * (qs0 - ps0));
            int filter1 = c4(filter + 4) >> 3;
            int filter2 = c4(filter + 3) >> 3;
            put(0, c4(qs0 - filter1) + half);
            put(-1, c4(ps0 + filter2) + half);
            if (!hev) {
                int f = (filter1 + 1) >> 1;
                put(1, c4(qs1 - f) + half);
                put(-2, c4(ps1 + f) + half);
            }
            return;
        }
        // 7.14.6.4 wide filter.
        int log2 = (filter_size == 8 || !flat2) ? 3 : 4;
        int n = log2 == 4 ? 6 : plane == 0 ? 3 : 2;
        int n2 = (log2 == 3 && plane == 0) ? 0 : 1;
        auto F = [&](int k) { return k >= 0 ? q[k] : p[-k - 1]; };
        int out[12];
        for (int i = -n; i < n; ++i) {
            int t = 0;
            for (int j = -n; j <= n; ++j) {
                int pos = std::min(std::max(i + j, -(n + 1)), n);
                int tap = std::abs(j) <= n2 ? 2 : 1;
                t += F(pos) * tap;
            }
            out[i + n] = (t + (1 << (log2 - 1))) >> log2;
        }
        for (int i = -n; i < n; ++i) put(i, out[i + n]);
    }

    // 7.14.2 edge loop filter for one 4x4 (plane units) edge segment.
    void edge(PlaneMut& pl, int plane, int pass, int row, int col) const {
        int ssx = plane ? info.subsampling_x : 0, ssy = plane ? info.subsampling_y : 0;
        int dx = pass == 0, dy = pass == 1;
        long x = (long)col * 4, y = (long)row * 4;
        row |= ssy;
        col |= ssx;
        bool on_screen = !(x >= info.coded_width || y >= info.coded_height || (pass == 0 && x == 0) ||
                           (pass == 1 && y == 0));
        if (!on_screen) return;
        int xp = (int)(x >> ssx), yp = (int)(y >> ssy);
        int prev_row = row - (dy << ssy), prev_col = col - (dx << ssx);
        int tx_sz = tx(plane, row >> ssy, col >> ssx);
        int prev_tx = tx(plane, prev_row >> ssy, prev_col >> ssx);
        bool is_tx_edge = pass == 0 ? xp % kTxW[tx_sz] == 0 : yp % kTxH[tx_sz] == 0;
        if (!is_tx_edge) return;  // intra blocks: applyFilter == isTxEdge
        int base = pass == 0 ? std::min(kTxW[prev_tx], kTxW[tx_sz]) : std::min(kTxH[prev_tx], kTxH[tx_sz]);
        int filter_size = plane == 0 ? std::min(16, base) : std::min(8, base);
        int lvl = level(plane, pass, row, col);
        if (lvl == 0) lvl = level(plane, pass, prev_row, prev_col);
        if (lvl == 0) return;
        Strength s = filter_strength(lvl, params.sharpness);
        for (int i = 0; i < 4; ++i) {
            long sx = xp + dy * i, sy = yp + dx * i;
            PlaneRef r = pl.ref();
            auto get = [&](int k) { return (int)r.get_clamped(sx + dx * k, sy + dy * k); };
            auto put = [&](int k, int v) { pl.set(sx + dx * k, sy + dy * k, (uint16_t)v); };
            filter_line(get, put, plane, filter_size, s);
        }
    }
};

// 7.14.1 loop filter over the picture, in place on `pic`.
int deblock_frame(PlaneMut pic[3], int num_planes, const vaco_av1_frame_info& info,
                  const uint8_t* tx_luma, const uint8_t* tx_chroma, const uint8_t* lvl_map,
                  const vaco_av1_deblock_params& params, int threads) {
    if (!(info.bit_depth == 8 || info.bit_depth == 10 || info.bit_depth == 12) || params.sharpness > 7)
        return VACO_AV1_MSG_DB_PARAMS;
    for (int k = 0; k < 4; ++k)
        if (params.levels[k] > 63) return VACO_AV1_MSG_DB_PARAMS;
    const int ssx = info.subsampling_x, ssy = info.subsampling_y;
    Deblocker d{info, tx_luma, tx_chroma, lvl_map, params,
                (info.mi_rows + ssy) >> ssy, (info.mi_cols + ssx) >> ssx};
    long n_luma = (long)info.mi_rows * info.mi_cols;
    for (long i = 0; i < n_luma; ++i)
        if (tx_luma[i] > 18 || (lvl_map && (lvl_map[4 * i] > 63 || lvl_map[4 * i + 1] > 63 ||
                                            lvl_map[4 * i + 2] > 63 || lvl_map[4 * i + 3] > 63)))
            return VACO_AV1_MSG_DB_PARAMS;
    if (num_planes > 1)
        for (long i = 0; i < (long)d.cmi_rows * d.cmi_cols; ++i)
            if (tx_chroma[i] > 18) return VACO_AV1_MSG_DB_PARAMS;
    const uint16_t max = (uint16_t)((1u << info.bit_depth) - 1);
    for (int pl = 0; pl < num_planes; ++pl)
        for (int y = 0; y < pic[pl].height; ++y)
            for (int x = 0; x < pic[pl].width; ++x)
                if (pic[pl].data[(long)y * pic[pl].stride + x] > max) return VACO_AV1_MSG_DB_SAMPLE;
    // The whole filter is off when both luma levels are zero (the syntax then
    // codes no chroma levels, AV1 5.9.11).
    if (params.levels[0] == 0 && params.levels[1] == 0) return 0;
    for (int plane = 0; plane < num_planes; ++plane) {
        if (plane != 0 && params.levels[1 + plane] == 0) continue;
        int row_step = plane == 0 ? 1 : 1 << ssy, col_step = plane == 0 ? 1 : 1 << ssx;
        int nrows = (info.mi_rows + row_step - 1) / row_step;
        for (int pass = 0; pass < 2; ++pass) {
            // Edges within one pass never overlap, so rows run independently.
            const long ncols = (info.mi_cols + col_step - 1) / col_step;
            parallel_for((long)nrows * ncols, threads, [&](long lo, long hi, int) {
                for (long i = lo; i < hi; ++i)
                    d.edge(pic[plane], plane, pass, (int)(i / ncols) * row_step, (int)(i % ncols) * col_step);
            });
        }
    }
    return 0;
}

PlaneRef plane_ref(const vaco_av1_picture& p, int k) {
    return PlaneRef{p.planes[k], p.width[k], p.height[k], p.stride[k]};
}
PlaneMut plane_mut(const vaco_av1_picture& p, int k) {
    return PlaneMut{p.planes[k], p.width[k], p.height[k], p.stride[k]};
}

void copy_plane(const PlaneRef& s, PlaneMut d) {
    for (int y = 0; y < std::min(s.height, d.height); ++y)
        std::memcpy(d.data + (long)y * d.stride, s.data + (long)y * s.stride,
                    sizeof(uint16_t) * std::min(s.width, d.width));
}

}  // namespace

// ------------------------------------------------------------------ C entry points (ctypes)

extern "C" {

int vo_find_direction(const uint16_t* blocks, int n, int bit_depth, uint8_t* dirs, uint32_t* vars) {
    for (int i = 0; i < n; ++i)
        if (int m = find_direction(blocks + 64L * i, bit_depth, dirs + i, vars + i)) return m;
    return 0;
}

int vo_filter_block(const uint16_t* inputs, const vaco_av1_cdef_filter_params* params, int n,
                    uint16_t* outputs) {
    for (int i = 0; i < n; ++i)
        if (int m = filter_block(inputs + 144L * i, params[i], outputs + 64L * i)) return m;
    return 0;
}

int vo_adjust_strength(int primary, uint32_t variance) { return adjust_strength(primary, variance); }
int vo_chroma_direction(int d, int sx, int sy) { return chroma_direction(d, sx != 0, sy != 0); }

// apply_cdef over a picture; dst receives a full copy first.
int vo_cdef_picture(const vaco_av1_picture* src, const vaco_av1_picture* dst,
                    const vaco_av1_frame_info* info, const uint8_t* skip, const int32_t* cdef_idx,
                    int cdef_stride, int cdef_count, const vaco_av1_cdef_params* params, int threads) {
    int np = info->monochrome ? 1 : 3;
    PlaneRef s[3];
    PlaneMut d[3];
    for (int k = 0; k < np; ++k) {
        s[k] = plane_ref(*src, k);
        d[k] = plane_mut(*dst, k);
        copy_plane(s[k], d[k]);
    }
    return cdef_frame(s, d, np, *info, skip, cdef_idx, cdef_stride, cdef_count, *params, threads);
}

int vo_upscale_plane(const uint16_t* input, int in_width, int in_height, int in_stride,
                     int visible_width, int output_width, int height, int bit_depth,
                     uint16_t* output, int out_stride, int threads) {
    PlaneRef in{input, in_width, in_height, in_stride};
    PlaneMut out{output, output_width, height, out_stride};
    return upscale_plane(in, visible_width, output_width, height, bit_depth, out, threads);
}

// upscale_picture (src/superres.rs:226-274): luma at (coded_width,
// upscaled_width, coded_height), then U and V at the ceil-divided chroma
// geometry, each through upscale_plane in that order, so the first failing
// plane's error is the one returned.  A missing U or V plane fails with
// vaco's "missing U/V plane" message once luma has succeeded.
int vo_upscale_picture(const vaco_av1_picture* in, const vaco_av1_picture* out,
                       const vaco_av1_superres_picture_config* cfg, int threads) {
    const int np = cfg->monochrome ? 1 : 3;
    for (int k = 0; k < np; ++k) {
        const int sx = k ? cfg->subsampling_x : 0, sy = k ? cfg->subsampling_y : 0;
        const int vis = (cfg->coded_width + (1 << sx) - 1) >> sx;
        const int outw = (cfg->upscaled_width + (1 << sx) - 1) >> sx;
        const int h = (cfg->coded_height + (1 << sy) - 1) >> sy;
        if (!in->planes[k]) return k == 1 ? VACO_AV1_MSG_SR_MISSING_U : VACO_AV1_MSG_SR_MISSING_V;
        PlaneRef src{in->planes[k], in->width[k], in->height[k], in->stride[k]};
        PlaneMut dst{out->planes[k], outw, h, out->stride[k]};
        if (int m = upscale_plane(src, vis, outw, h, cfg->bit_depth, dst, threads)) return m;
    }
    return 0;
}

// Lines across a deblocking edge through the 7.14.6 sample filter, for
// cross-checks of the filter arithmetic: lines[16 i + 8 + k] is sample k past
// the edge (k < 0 on the p side) of line i, which filters at level lvls[i];
// out receives each line after filtering (a copy where nothing is written).
int vo_deblock_lines(const uint16_t* lines, int n, int plane, int filter_size, const uint8_t* lvls, int sharpness,
                     int bit_depth, uint16_t* out) {
    vaco_av1_frame_info info{};
    info.bit_depth = bit_depth;
    vaco_av1_deblock_params params{};
    params.sharpness = (uint8_t)sharpness;
    Deblocker d{info, nullptr, nullptr, nullptr, params, 0, 0};
    for (int i = 0; i < n; ++i) {
        const uint16_t* line = lines + 16L * i;
        uint16_t* o = out + 16L * i;
        for (int k = 0; k < 16; ++k) o[k] = line[k];
        auto get = [&](int k) { return (int)line[std::min(std::max(8 + k, 0), 15)]; };
        auto put = [&](int k, int v) {
            if (8 + k >= 0 && 8 + k < 16) o[8 + k] = (uint16_t)v;
        };
        d.filter_line(get, put, plane, filter_size, filter_strength(lvls[i], sharpness));
    }
    return 0;
}

int vo_restore_plane(const uint16_t* before, int bw, int bh, int bstride, const uint16_t* after,
                     int aw, int ah, int astride, const vaco_av1_lr_plane_config* cfg,
                     const vaco_av1_lr_unit* units, int unit_count, uint16_t* output,
                     int out_stride, int threads) {
    PlaneRef b{before, bw, bh, bstride}, a{after, aw, ah, astride};
    LrConfig c{cfg->width, cfg->height, cfg->bit_depth, cfg->unit_size, cfg->subsampling_y ? 1 : 0};
    PlaneMut out{output, cfg->width > 0 ? cfg->width : 0, cfg->height > 0 ? cfg->height : 0, out_stride};
    return restore_plane(b, a, c, units, unit_count, out, threads);
}

int vo_deblock_picture(const vaco_av1_picture* src, const vaco_av1_picture* dst,
                       const vaco_av1_frame_info* info, const uint8_t* tx_luma,
                       const uint8_t* tx_chroma, const uint8_t* lvl_map,
                       const vaco_av1_deblock_params* params, int threads) {
    int np = info->monochrome ? 1 : 3;
    PlaneMut d[3];
    for (int k = 0; k < np; ++k) {
        d[k] = plane_mut(*dst, k);
        copy_plane(plane_ref(*src, k), d[k]);
    }
    return deblock_frame(d, np, *info, tx_luma, tx_chroma, lvl_map, *params, threads);
}

// The whole chain, as decode_frame (src/decode.rs:553-559) orders it with a
// deblocking step in front: deblock -> keep the pre-CDEF copy -> CDEF ->
// superres of both images -> restoration per plane -> visible output.
int vo_postfilter_frame(const vaco_av1_frame_job* job, int threads) {
    const vaco_av1_frame_info& info = job->info;
    const int np = info.monochrome ? 1 : 3;
    const int ssx = info.subsampling_x, ssy = info.subsampling_y;
    std::vector<uint16_t> pre[3], cdef[3], up_pre[3], up_cdef[3];
    PlaneMut pre_p[3], cdef_p[3];
    for (int k = 0; k < np; ++k) {
        int w = job->src.width[k], h = job->src.height[k];
        pre[k].assign((size_t)w * h, 0);
        cdef[k].assign((size_t)w * h, 0);
        pre_p[k] = PlaneMut{pre[k].data(), w, h, w};
        cdef_p[k] = PlaneMut{cdef[k].data(), w, h, w};
        copy_plane(plane_ref(job->src, k), pre_p[k]);
    }
    if (int m = deblock_frame(pre_p, np, info, job->tx_luma, job->tx_chroma, job->lvl_map, job->deblock,
                              threads))
        return m;
    PlaneRef pre_r[3];
    for (int k = 0; k < np; ++k) {
        pre_r[k] = pre_p[k].ref();
        copy_plane(pre_r[k], cdef_p[k]);
    }
    if (int m = cdef_frame(pre_r, cdef_p, np, info, job->skip, job->cdef_idx, job->cdef_stride,
                           job->cdef_count, job->cdef, threads))
        return m;
    const bool superres = info.upscaled_width != info.coded_width;
    bool lr_active = false;
    for (int k = 0; k < np; ++k) lr_active = lr_active || job->lr_type[k] != VACO_AV1_FRAME_LR_NONE;
    PlaneRef before[3], after[3];
    for (int k = 0; k < np; ++k) {
        before[k] = pre_r[k];
        after[k] = cdef_p[k].ref();
    }
    if (superres) {
        for (int k = 0; k < np; ++k) {
            bool ch = k != 0;
            int sx = ch ? ssx : 0, sy = ch ? ssy : 0;
            int vis = (info.coded_width + sx) >> sx, outw = (info.upscaled_width + sx) >> sx;
            int h = (info.coded_height + sy) >> sy;
            up_cdef[k].assign((size_t)outw * h, 0);
            if (int m = upscale_plane(after[k], vis, outw, h, info.bit_depth,
                                      PlaneMut{up_cdef[k].data(), outw, h, outw}, threads))
                return m;
            after[k] = PlaneRef{up_cdef[k].data(), outw, h, outw};
            if (lr_active) {
                up_pre[k].assign((size_t)outw * h, 0);
                if (int m = upscale_plane(before[k], vis, outw, h, info.bit_depth,
                                          PlaneMut{up_pre[k].data(), outw, h, outw}, threads))
                    return m;
                before[k] = PlaneRef{up_pre[k].data(), outw, h, outw};
            }
        }
    }
    for (int k = 0; k < np; ++k) {
        bool ch = k != 0;
        int sx = ch ? ssx : 0, sy = ch ? ssy : 0;
        int w = info.upscaled_width >> sx, h = info.coded_height >> sy;
        PlaneMut out = plane_mut(job->dst, k);
        if (job->lr_type[k] == VACO_AV1_FRAME_LR_NONE) {
            // copy_visible_plane (src/decode.rs:673-681).
            for (int y = 0; y < h; ++y)
                for (int x = 0; x < w; ++x) out.set(x, y, after[k].get_clamped(x, y));
            continue;
        }
        if (job->lr_unit_size[k] == 0) return VACO_AV1_MSG_LR_NO_UNIT_SIZE;
        LrConfig c{w, h, info.bit_depth, job->lr_unit_size[k], ch && ssy ? 1 : 0};
        if (int m = restore_plane(before[k], after[k], c, job->lr_units[k], job->lr_unit_count[k], out,
                                  threads))
            return m;
    }
    return 0;
}

}  // extern "C"

// Struct sizes as gcc lays them out from include/vaco_av1_gpu.h, for the
// ctypes layout test.
// pic_to_frame / blit (src/decode.rs:3795-3891): the pixel format from
// (bit depth, monochrome, subsampling), then per plane the frame extents
// (upscaled_width x coded_height, chroma rounded up) cut to the source
// plane, each sample written as one byte (u8::try_from(v).unwrap_or(0): a
// value above 255 becomes 0) or as two little-endian bytes above 8 bits.
extern "C" int vo_emit_frame(const vaco_av1_picture* pic, const vaco_av1_frame_info* info,
                             const vaco_av1_frame_buffer* out) {
    const int bd = info->bit_depth;
    const bool mono = info->monochrome != 0, sx = info->subsampling_x != 0, sy = info->subsampling_y != 0;
    // The names of decode.rs:3802-3817; vaco-pixfmt knows all but yuv440p8le.
    const bool known = (bd == 8 || bd == 10 || bd == 12) && !(bd == 8 && !mono && !sx && sy);
    if (!known) return VACO_AV1_MSG_PIXEL_FORMAT;
    const long w = info->upscaled_width, h = info->coded_height;
    const long cw = (w + (1L << sx) - 1) >> sx, ch = (h + (1L << sy) - 1) >> sy;
    const bool two_bytes = bd > 8;
    for (int k = 0; k < (mono ? 1 : 3); ++k) {
        PlaneRef src = plane_ref(*pic, k);
        const long width = std::min<long>(k ? cw : w, src.width), height = std::min<long>(k ? ch : h, src.height);
        uint8_t* dst = static_cast<uint8_t*>(out->planes[k]);
        for (long y = 0; y < height; ++y) {
            uint8_t* row = dst + y * out->linesize[k];
            for (long x = 0; x < width; ++x) {
                const uint16_t v = src.get_clamped((int)x, (int)y);
                if (two_bytes) {
                    row[2 * x] = (uint8_t)(v & 0xFF);
                    row[2 * x + 1] = (uint8_t)(v >> 8);
                } else {
                    row[x] = v > 255 ? 0 : (uint8_t)v;
                }
            }
        }
    }
    return 0;
}

// ------------------------------------------------------------ film grain
//
// AV1 spec 7.18.3 (film grain synthesis), restated step by step: vaco parses
// the parameters (src/frame_header.rs:1125-1210) but has no synthesis, so
// this part has no vaco code or golden vector behind it (parity unpinned).
// The Gaussian sequence is the caller's table.

namespace fg {

struct Grain {
    const vaco_av1_film_grain_params& p;
    const int16_t* gauss;
    int bd, sub_x, sub_y, mono;
    unsigned reg = 0;
    int luma[73][82] = {}, cb[73][82] = {}, cr[73][82] = {};
    int lut[3][256] = {};
    int grain_min = 0, grain_max = 0;

    Grain(const vaco_av1_film_grain_params& p_, const int16_t* g, int bd_, int sx, int sy, int mono_)
        : p(p_), gauss(g), bd(bd_), sub_x(sx), sub_y(sy), mono(mono_) {
        const int center = 128 << (bd - 8);
        grain_min = -center;
        grain_max = (256 << (bd - 8)) - 1 - center;
    }

    static int round2(int x, int n) { return n == 0 ? x : (x + (1 << (n - 1))) >> n; }
    static int clip3(int lo, int hi, int x) { return x < lo ? lo : x > hi ? hi : x; }

    // 7.18.3.2 random number process
    int random(int bits) {
        unsigned r = reg;
        const unsigned bit = ((r >> 0) ^ (r >> 1) ^ (r >> 3) ^ (r >> 12)) & 1;
        r = (r >> 1) | (bit << 15);
        reg = r;
        return (int)((r >> (16 - bits)) & ((1u << bits) - 1));
    }

    // 7.18.3.3 generate grain process
    void generate() {
        int shift = 12 - bd + p.grain_scale_shift;
        reg = p.grain_seed;
        for (int y = 0; y < 73; ++y)
            for (int x = 0; x < 82; ++x) {
                const int g = p.num_y_points > 0 ? gauss[random(11)] : 0;
                luma[y][x] = round2(g, shift);
            }
        const int ar_shift = p.ar_coeff_shift_minus_6 + 6;
        const int lag = p.ar_coeff_lag;
        for (int y = 3; y < 73; ++y)
            for (int x = 3; x < 82 - 3; ++x) {
                int sum = 0, pos = 0;
                for (int dr = -lag; dr <= 0; ++dr)
                    for (int dc = -lag; dc <= lag; ++dc) {
                        if (dr == 0 && dc == 0) break;
                        sum += luma[y + dr][x + dc] * (p.ar_coeffs_y_plus_128[pos] - 128);
                        ++pos;
                    }
                luma[y][x] = clip3(grain_min, grain_max, luma[y][x] + round2(sum, ar_shift));
            }
        if (mono) return;
        const int cw = sub_x ? 44 : 82, ch = sub_y ? 38 : 73;
        const bool cb_on = p.num_cb_points || p.chroma_scaling_from_luma;
        const bool cr_on = p.num_cr_points || p.chroma_scaling_from_luma;
        reg = p.grain_seed ^ 0xb524u;
        for (int y = 0; y < ch; ++y)
            for (int x = 0; x < cw; ++x) cb[y][x] = round2(cb_on ? gauss[random(11)] : 0, shift);
        reg = p.grain_seed ^ 0x49d8u;
        for (int y = 0; y < ch; ++y)
            for (int x = 0; x < cw; ++x) cr[y][x] = round2(cr_on ? gauss[random(11)] : 0, shift);
        for (int y = 3; y < ch; ++y)
            for (int x = 3; x < cw - 3; ++x) {
                int sum0 = 0, sum1 = 0, pos = 0;
                for (int dr = -lag; dr <= 0; ++dr)
                    for (int dc = -lag; dc <= lag; ++dc) {
                        const int c0 = p.ar_coeffs_cb_plus_128[pos] - 128, c1 = p.ar_coeffs_cr_plus_128[pos] - 128;
                        if (dr == 0 && dc == 0) {
                            if (p.num_y_points > 0) {
                                int l = 0;
                                const int ly = ((y - 3) << sub_y) + 3, lx = ((x - 3) << sub_x) + 3;
                                for (int i = 0; i <= sub_y; ++i)
                                    for (int j = 0; j <= sub_x; ++j) l += luma[ly + i][lx + j];
                                l = round2(l, sub_x + sub_y);
                                sum0 += l * c0;
                                sum1 += l * c1;
                            }
                            break;
                        }
                        sum0 += c0 * cb[y + dr][x + dc];
                        sum1 += c1 * cr[y + dr][x + dc];
                        ++pos;
                    }
                if (cb_on) cb[y][x] = clip3(grain_min, grain_max, cb[y][x] + round2(sum0, ar_shift));
                if (cr_on) cr[y][x] = clip3(grain_min, grain_max, cr[y][x] + round2(sum1, ar_shift));
            }
    }

    // 7.18.3.4 scaling lookup initialization
    void init_luts() {
        for (int plane = 0; plane < (mono ? 1 : 3); ++plane) {
            const uint8_t *v, *sc;
            int n;
            if (plane == 0 || p.chroma_scaling_from_luma) {
                n = p.num_y_points, v = p.point_y_value, sc = p.point_y_scaling;
            } else if (plane == 1) {
                n = p.num_cb_points, v = p.point_cb_value, sc = p.point_cb_scaling;
            } else {
                n = p.num_cr_points, v = p.point_cr_value, sc = p.point_cr_scaling;
            }
            int* l = lut[plane];
            if (n == 0) {
                for (int x = 0; x < 256; ++x) l[x] = 0;
                continue;
            }
            for (int x = 0; x < v[0]; ++x) l[x] = sc[0];
            for (int i = 0; i < n - 1; ++i) {
                const int dy = sc[i + 1] - sc[i], dx = v[i + 1] - v[i];
                const int delta = dy * ((65536 + (dx >> 1)) / dx);
                for (int x = 0; x < dx; ++x) l[v[i] + x] = sc[i] + ((x * delta + 32768) >> 16);
            }
            for (int x = v[n - 1]; x < 256; ++x) l[x] = sc[n - 1];
        }
    }

    int scale_lut(int plane, int index) const {
        const int shift = bd - 8, x = index >> shift, rem = index - (x << shift);
        if (bd == 8 || x == 255) return lut[plane][x];
        const int start = lut[plane][x], end = lut[plane][x + 1];
        return start + round2((end - start) * rem, shift);
    }
};

}  // namespace fg

// 7.18.3.5 add noise synthesis process over the whole frame.
extern "C" int vo_film_grain(const vaco_av1_picture* in, const vaco_av1_picture* out,
                             const vaco_av1_frame_info* info, const vaco_av1_film_grain_params* p,
                             const int16_t* gauss) {
    const int bd = info->bit_depth;
    const int mono = info->monochrome != 0, sx = info->subsampling_x, sy = info->subsampling_y;
    const int np = mono ? 1 : 3;
    if (!(bd == 8 || bd == 10 || bd == 12)) return VACO_AV1_MSG_FG_PARAMS;
    auto increasing = [](const uint8_t* v, int n) {
        for (int i = 1; i < n; ++i)
            if (v[i] <= v[i - 1]) return false;
        return true;
    };
    if (p->num_y_points > 14 || p->num_cb_points > 10 || p->num_cr_points > 10 || p->ar_coeff_lag > 3 ||
        p->grain_scaling_minus_8 > 3 || p->ar_coeff_shift_minus_6 > 3 || p->grain_scale_shift > 3 ||
        p->cb_offset > 511 || p->cr_offset > 511 || !increasing(p->point_y_value, p->num_y_points) ||
        !increasing(p->point_cb_value, p->num_cb_points) || !increasing(p->point_cr_value, p->num_cr_points))
        return VACO_AV1_MSG_FG_PARAMS;
    const int w = info->upscaled_width, h = info->coded_height;
    if (w <= 0 || h <= 0) return VACO_AV1_MSG_FRAME_GEOMETRY;
    int pw[3], ph[3];
    for (int k = 0; k < np; ++k) {
        pw[k] = k ? (w + sx) >> sx : w;
        ph[k] = k ? (h + sy) >> sy : h;
        if (in->width[k] < pw[k] || in->height[k] < ph[k] || out->width[k] < pw[k] || out->height[k] < ph[k])
            return VACO_AV1_MSG_FRAME_GEOMETRY;
    }
    const int maxv = (1 << bd) - 1;
    auto at = [](const vaco_av1_picture* pic, int k, int x, int y) -> uint16_t& {
        return pic->planes[k][(long)y * pic->stride[k] + x];
    };
    for (int k = 0; k < np; ++k)
        for (int y = 0; y < ph[k]; ++y)
            for (int x = 0; x < pw[k]; ++x)
                if (at(in, k, x, y) > maxv) return VACO_AV1_MSG_FG_SAMPLE;
    if (!p->apply_grain) {
        for (int k = 0; k < np; ++k)
            for (int y = 0; y < ph[k]; ++y)
                for (int x = 0; x < pw[k]; ++x) at(out, k, x, y) = at(in, k, x, y);
        return 0;
    }
    auto* g = new fg::Grain(*p, gauss, bd, sx, sy, mono);
    g->generate();
    g->init_luts();
    // Noise stripes: 34 rows (17 when subsampled) of every plane per stripe of
    // 32 luma rows; columns up to the last block's reach.
    const int nstripes = ((h + 1) / 2 + 15) / 16;
    const int stripe_w = ((w + 1) / 2 + 15) / 16 * 32 + 34;
    std::vector<int> stripe((size_t)nstripes * 3 * 34 * stripe_w, 0);
    auto ns = [&](int s, int plane, int i, int x) -> int& {
        return stripe[(((size_t)s * 3 + plane) * 34 + i) * stripe_w + x];
    };
    int luma_num = 0;
    for (int y = 0; y < (h + 1) / 2; y += 16) {
        g->reg = p->grain_seed;
        g->reg ^= ((luma_num * 37 + 178) & 255) << 8;
        g->reg ^= ((luma_num * 173 + 105) & 255);
        for (int x = 0; x < (w + 1) / 2; x += 16) {
            const int rnd = g->random(8);
            const int off_x = rnd >> 4, off_y = rnd & 15;
            for (int plane = 0; plane < np; ++plane) {
                const int psx = plane ? sx : 0, psy = plane ? sy : 0;
                const int pox = psx ? 6 + off_x : 9 + off_x * 2, poy = psy ? 6 + off_y : 9 + off_y * 2;
                for (int i = 0; i < (34 >> psy); ++i)
                    for (int j = 0; j < (34 >> psx); ++j) {
                        const int(*tmpl)[82] = plane == 0 ? g->luma : plane == 1 ? g->cb : g->cr;
                        int v = tmpl[poy + i][pox + j];
                        if (psx == 0) {
                            if (j < 2 && p->overlap_flag && x > 0) {
                                const int old = ns(luma_num, plane, i, x * 2 + j);
                                v = j == 0 ? old * 27 + v * 17 : old * 17 + v * 27;
                                v = fg::Grain::clip3(g->grain_min, g->grain_max, fg::Grain::round2(v, 5));
                            }
                            ns(luma_num, plane, i, x * 2 + j) = v;
                        } else {
                            if (j == 0 && p->overlap_flag && x > 0) {
                                const int old = ns(luma_num, plane, i, x + j);
                                v = old * 23 + v * 22;
                                v = fg::Grain::clip3(g->grain_min, g->grain_max, fg::Grain::round2(v, 5));
                            }
                            ns(luma_num, plane, i, x + j) = v;
                        }
                    }
            }
        }
        ++luma_num;
    }
    // Noise image with the vertical overlap, then blending.
    int min_v, max_luma, max_chroma;
    if (p->clip_to_restricted_range) {
        min_v = 16 << (bd - 8);
        max_luma = 235 << (bd - 8);
        max_chroma = p->mc_identity ? max_luma : 240 << (bd - 8);
    } else {
        min_v = 0;
        max_luma = max_chroma = (256 << (bd - 8)) - 1;
    }
    const int scaling_shift = p->grain_scaling_minus_8 + 8;
    auto noise = [&](int plane, int y, int x) {
        const int psy = plane ? sy : 0;
        const int num = y >> (5 - psy), i = y - (num << (5 - psy));
        int v = ns(num, plane, i, x);
        if (psy == 0) {
            if (i < 2 && num > 0 && p->overlap_flag) {
                const int old = ns(num - 1, plane, i + 32, x);
                v = i == 0 ? old * 27 + v * 17 : old * 17 + v * 27;
                v = fg::Grain::clip3(g->grain_min, g->grain_max, fg::Grain::round2(v, 5));
            }
        } else if (i < 1 && num > 0 && p->overlap_flag) {
            const int old = ns(num - 1, plane, i + 16, x);
            v = old * 23 + v * 22;
            v = fg::Grain::clip3(g->grain_min, g->grain_max, fg::Grain::round2(v, 5));
        }
        return v;
    };
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const int orig = at(in, 0, x, y);
            int v = orig;
            if (p->num_y_points > 0) {
                const int n = fg::Grain::round2(g->scale_lut(0, orig) * noise(0, y, x), scaling_shift);
                v = fg::Grain::clip3(min_v, max_luma, orig + n);
            }
            at(out, 0, x, y) = (uint16_t)v;
        }
    for (int plane = 1; plane < np; ++plane) {
        const bool on = (plane == 1 ? p->num_cb_points : p->num_cr_points) > 0 || p->chroma_scaling_from_luma;
        const int mult = plane == 1 ? p->cb_mult : p->cr_mult, lmult = plane == 1 ? p->cb_luma_mult : p->cr_luma_mult;
        const int offset = plane == 1 ? p->cb_offset : p->cr_offset;
        for (int y = 0; y < ph[plane]; ++y)
            for (int x = 0; x < pw[plane]; ++x) {
                const int orig = at(in, plane, x, y);
                int v = orig;
                if (on) {
                    const int ly = y << sy, lx = x << sx, lnx = std::min(lx + 1, w - 1);
                    const int avg = sx ? fg::Grain::round2(at(in, 0, lx, ly) + at(in, 0, lnx, ly), 1) : at(in, 0, lx, ly);
                    int merged;
                    if (p->chroma_scaling_from_luma) {
                        merged = avg;
                    } else {
                        const int combined = avg * (lmult - 128) + orig * (mult - 128);
                        merged = fg::Grain::clip3(0, maxv, (combined >> 6) + ((offset - 256) << (bd - 8)));
                    }
                    const int n = fg::Grain::round2(g->scale_lut(plane, merged) * noise(plane, y, x), scaling_shift);
                    v = fg::Grain::clip3(min_v, max_chroma, orig + n);
                }
                at(out, plane, x, y) = (uint16_t)v;
            }
    }
    delete g;
    return 0;
}

extern "C" int vo_sizeof(const char* name) {
    struct Entry {
        const char* n;
        int s;
    };
    static const Entry kSizes[] = {
        {"vaco_av1_picture", (int)sizeof(vaco_av1_picture)},
        {"vaco_av1_frame_info", (int)sizeof(vaco_av1_frame_info)},
        {"vaco_av1_cdef_params", (int)sizeof(vaco_av1_cdef_params)},
        {"vaco_av1_cdef_filter_params", (int)sizeof(vaco_av1_cdef_filter_params)},
        {"vaco_av1_lr_unit", (int)sizeof(vaco_av1_lr_unit)},
        {"vaco_av1_lr_plane_config", (int)sizeof(vaco_av1_lr_plane_config)},
        {"vaco_av1_deblock_params", (int)sizeof(vaco_av1_deblock_params)},
        {"vaco_av1_frame_job", (int)sizeof(vaco_av1_frame_job)},
        {"vaco_av1_tuning", (int)sizeof(vaco_av1_tuning)},
        {"vaco_av1_frame_buffer", (int)sizeof(vaco_av1_frame_buffer)},
        {"vaco_av1_film_grain_params", (int)sizeof(vaco_av1_film_grain_params)},
        {"vaco_av1_superres_picture_config", (int)sizeof(vaco_av1_superres_picture_config)},
    };
    for (const Entry& e : kSizes)
        if (std::strcmp(e.n, name) == 0) return e.s;
    return -1;
}
