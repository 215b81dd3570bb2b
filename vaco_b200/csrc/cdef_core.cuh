// cdef_core.cuh -- CDEF device functions shared by the CDEF kernels and the
// fused deblock+CDEF kernel.  Mirrors vaco crates/codec/vaco-codec-av1/src/cdef.rs
// (find_direction :79, constrain :126, filter_block :142, adjust_strength
// :209, chroma_direction :224).
//
// Unavailable neighbours (outside the plane, apply_cdef's availability rule,
// src/decode.rs:828-831) are stored as the sentinel kSent: constrain() of a
// sentinel difference is 0 for every valid strength/damping pair and the
// maximum masks it out with kMaxMask, so no tap needs a bounds check.
#pragma once

#include "common.cuh"

namespace vaco {
namespace cdefk {

constexpr int kSent = 0xC000;      // > any 12-bit sample; & kMaxMask == 0
constexpr int kMaxMask = 0x3FFF;

// (row, col) step per direction and distance (src/cdef.rs:57-66).
struct DirTable {
    int8_t v[8][2][2];
};
constexpr DirTable kDir = {{
    {{-1, 1}, {-2, 2}}, {{0, 1}, {-1, 2}}, {{0, 1}, {0, 2}},  {{0, 1}, {1, 2}},
    {{1, 1}, {2, 2}},   {{1, 0}, {2, 1}},  {{1, 0}, {2, 0}},  {{1, 0}, {2, -1}},
}};
// The table packed into one 24-bit immediate per (distance, axis): 3 bits
// per direction, biased by 2.  A lookup with a per-lane direction is then a
// shift and a mask instead of a divergent constant-memory read.
__host__ __device__ constexpr uint32_t dir_packed(int k, int axis) {
    uint32_t m = 0;
    for (int d = 0; d < 8; ++d) m |= (uint32_t)(kDir.v[d][k][axis] + 2) << (3 * d);
    return m;
}
template <int K, int AXIS>
__device__ __forceinline__ int dir_step(int d) {
    constexpr uint32_t m = dir_packed(K, AXIS);
    return (int)((m >> (3 * d)) & 7u) - 2;
}
// Sample offset of tap distance K along direction d in a plane of `pitch`.
template <int K>
__device__ __forceinline__ int dir_offset(int d, int pitch) {
    return dir_step<K, 0>(d) * pitch + dir_step<K, 1>(d);
}

// Line index of pixel (i, j) for direction d (src/cdef.rs:88-97).
__host__ __device__ constexpr int dir_bin(int d, int i, int j) {
    return d == 0 ? i + j : d == 1 ? i + j / 2 : d == 2 ? i : d == 3 ? 3 + i - j / 2
         : d == 4 ? 7 + i - j : d == 5 ? 3 + j - i / 2 : d == 6 ? j : i / 2 + j;
}
__host__ __device__ constexpr int dir_count(int d, int b) {
    int n = 0;
    for (int i = 0; i < 8; ++i)
        for (int j = 0; j < 8; ++j) n += dir_bin(d, i, j) == b;
    return n;
}
__host__ __device__ constexpr int dir_weight(int d, int b) {
    return dir_count(d, b) ? 840 / dir_count(d, b) : 0;
}

// Costs of directions P and P+4 for one 8x8 block at `blk` (row pitch in
// samples, rows 16-byte aligned).  Fully unrolled: every bin is a register.
template <int P>
__device__ __forceinline__ void dir_costs(const uint16_t* blk, int pitch, int shift, int& c_lo, int& c_hi) {
    int a[15], b[15];
#pragma unroll
    for (int k = 0; k < 15; ++k) a[k] = b[k] = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        uint4 row = *reinterpret_cast<const uint4*>(blk + i * pitch);
        uint32_t w[4] = {row.x, row.y, row.z, row.w};
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            int s = (j & 1) ? (w[j >> 1] >> 16) : (w[j >> 1] & 0xFFFF);
            int v = (s >> shift) - 128;
            a[dir_bin(P, i, j)] += v;
            b[dir_bin(P + 4, i, j)] += v;
        }
    }
    int lo = 0, hi = 0;
#pragma unroll
    for (int k = 0; k < 15; ++k) {
        if (dir_weight(P, k)) lo += a[k] * a[k] * dir_weight(P, k);
        if (dir_weight(P + 4, k)) hi += b[k] * b[k] * dir_weight(P + 4, k);
    }
    c_lo = lo;
    c_hi = hi;
}

__device__ __forceinline__ void dir_costs_pair(int pair, const uint16_t* blk, int pitch, int shift, int& lo, int& hi) {
    switch (pair) {
        case 0: dir_costs<0>(blk, pitch, shift, lo, hi); break;
        case 1: dir_costs<1>(blk, pitch, shift, lo, hi); break;
        case 2: dir_costs<2>(blk, pitch, shift, lo, hi); break;
        default: dir_costs<3>(blk, pitch, shift, lo, hi); break;
    }
}

__device__ __forceinline__ void best_direction(const int* cost8, int& best, uint32_t& var) {
    int b = 0;
#pragma unroll
    for (int d = 1; d < 8; ++d)
        if (cost8[d] > cost8[b]) b = d;
    best = b;
    var = (uint32_t)((cost8[b] - cost8[(b + 4) & 7]) >> 10);
}

// constrain (src/cdef.rs:126-133); threshold 0 yields 0 for any shift.
__device__ __forceinline__ int constrain(int d, int t, int shift) {
    int a = abs(d);
    int c = min(a, max(0, t - (a >> shift)));
    return d < 0 ? -c : c;
}

__device__ __forceinline__ int ilog2u(unsigned v) { return 31 - __clz(v); }

// adjust_strength (src/cdef.rs:209-220).
__device__ __forceinline__ int adjust_strength(int primary, uint32_t variance) {
    if (variance == 0) return 0;
    uint32_t scaled = variance >> 6;
    uint32_t lg = scaled == 0 ? 0 : min((uint32_t)ilog2u(scaled), 12u);
    return (int)(((uint32_t)primary * (4 + lg) + 8) >> 4);
}

// chroma_direction (src/cdef.rs:224-230).
__device__ __forceinline__ int chroma_direction(int d, int sx, int sy) {
    const uint32_t k10 = 0x66654207u;  // nibbles of [7,0,2,4,5,6,6,6]
    const uint32_t k01 = 0x06432221u;  // nibbles of [1,2,2,2,3,4,6,0]
    if (sx && !sy) return (k10 >> (4 * (d & 7))) & 0xF;
    if (!sx && sy) return (k01 >> (4 * (d & 7))) & 0xF;
    return d & 7;
}

// Per-block filter parameters, offsets in shared-memory samples.
struct BlockFilter {
    int off[6];   // primary d0,d1; secondary (dir+2) d0,d1; secondary (dir+6) d0,d1
    short pri, sec;
    uint8_t pri_shift, sec_shift, pt0, pt1;
};

__device__ __forceinline__ BlockFilter make_filter(int dir, int pri, int sec, int damping, int shift, int pitch) {
    BlockFilter f;
    f.off[0] = dir_offset<0>(dir, pitch);
    f.off[1] = dir_offset<1>(dir, pitch);
    f.off[2] = dir_offset<0>((dir + 2) & 7, pitch);
    f.off[3] = dir_offset<1>((dir + 2) & 7, pitch);
    f.off[4] = dir_offset<0>((dir + 6) & 7, pitch);
    f.off[5] = dir_offset<1>((dir + 6) & 7, pitch);
    f.pri = (short)pri;
    f.sec = (short)sec;
    f.pri_shift = (uint8_t)(pri ? max(0, damping - ilog2u(pri)) : 0);
    f.sec_shift = (uint8_t)(sec ? max(0, damping - ilog2u(sec)) : 0);
    bool odd = ((pri >> shift) & 1) != 0;
    f.pt0 = odd ? 3 : 4;
    f.pt1 = odd ? 3 : 2;
    return f;
}

// One output sample of filter_block (src/cdef.rs:167-202) at smem position s.
__device__ __forceinline__ int filter_px(const uint16_t* s, const BlockFilter& f) {
    const int cur = s[0];
    int mn = cur, mx = cur, sum = 0;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int ptap = k ? f.pt1 : f.pt0;
        const int stap = 2 - k;
        int p0 = s[f.off[k]], p1 = s[-f.off[k]];
        int s0 = s[f.off[2 + k]], s1 = s[-f.off[2 + k]];
        int s2 = s[f.off[4 + k]], s3 = s[-f.off[4 + k]];
        mn = min(mn, min(min(p0, p1), min(min(s0, s1), min(s2, s3))));
        mx = max(mx, max(max(p0 & kMaxMask, p1 & kMaxMask),
                         max(max(s0 & kMaxMask, s1 & kMaxMask), max(s2 & kMaxMask, s3 & kMaxMask))));
        sum += ptap * (constrain(p0 - cur, f.pri, f.pri_shift) + constrain(p1 - cur, f.pri, f.pri_shift));
        sum += stap * (constrain(s0 - cur, f.sec, f.sec_shift) + constrain(s1 - cur, f.sec, f.sec_shift) +
                       constrain(s2 - cur, f.sec, f.sec_shift) + constrain(s3 - cur, f.sec, f.sec_shift));
    }
    int v = cur + ((8 + sum - (sum < 0)) >> 4);
    return min(max(v, mn), mx);
}


}  // namespace cdefk
}  // namespace vaco

namespace vaco {
namespace cdefk {

// ---------------------------------------------------------------- two pixels per register
//
// filter_px() for a horizontal pair of pixels held as two 16-bit lanes of one
// 32-bit word (low lane = left pixel), using the sm_90+ packed min/max.  Every
// per-lane quantity below stays in [0, 65535], so plain 32-bit adds and
// subtracts never carry or borrow across lanes:
//   hi = max(v, cur), lo = min(v, cur), |d| = hi - lo, d+ = hi - cur
//   m  = t - min(|d| >> s, t)               (= max(0, t - (|d| >> s)))
//   c  = min(|d|, m), c+ = min(c, d+)       (c+: constrain's positive part)
//   acc+ += tap * c+, acc += tap * c        (each <= 24 * 240 = 5760), and
//   at the end acc- = acc - acc+ (the negative parts' sum)
// Output: with pos/neg the non-negative parts of acc+ - acc-,
//   r+ = (pos + 8) >> 4, r- = (neg + 8) >> 4  (vaco's signed rounding)
//   out = min(max(cur + r+, mn + r-) - r-, mx) = clamp(cur + r+ - r-, mn, mx).
__device__ __forceinline__ uint32_t vmin2(uint32_t a, uint32_t b) {
    uint32_t d;
    asm("min.u16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
__device__ __forceinline__ uint32_t vmax2(uint32_t a, uint32_t b) {
    uint32_t d;
    asm("max.u16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}

// Per-block tap description for the pair filter.
struct PairBlock {
    int16_t off[6];       // tap offsets (samples): primary d0,d1; dir+2 d0,d1; dir+6 d0,d1
    uint16_t pri, sec;
    uint8_t pri_shift, sec_shift, pt0, pt1;
};

__device__ __forceinline__ PairBlock make_pair_block(int dir, int pri, int sec, int damping, int shift, int pitch) {
    PairBlock f;
    f.off[0] = (int16_t)dir_offset<0>(dir, pitch);
    f.off[1] = (int16_t)dir_offset<1>(dir, pitch);
    f.off[2] = (int16_t)dir_offset<0>((dir + 2) & 7, pitch);
    f.off[3] = (int16_t)dir_offset<1>((dir + 2) & 7, pitch);
    f.off[4] = (int16_t)dir_offset<0>((dir + 6) & 7, pitch);
    f.off[5] = (int16_t)dir_offset<1>((dir + 6) & 7, pitch);
    f.pri = (uint16_t)pri;
    f.sec = (uint16_t)sec;
    f.pri_shift = (uint8_t)(pri ? max(0, damping - ilog2u(pri)) : 0);
    f.sec_shift = (uint8_t)(sec ? max(0, damping - ilog2u(sec)) : 0);
    const bool odd = ((pri >> shift) & 1) != 0;
    f.pt0 = odd ? 3 : 4;
    f.pt1 = odd ? 3 : 2;
    return f;
}

// The pair of samples starting at sample index `i` (any parity) of a plane
// staged at 4-byte alignment: two aligned word loads and a byte permute.
struct PairTap {
    const uint32_t* w;  // aligned word holding sample i & ~1
    uint32_t sel;       // byte selector: 0x3210 (i even) or 0x5432 (i odd)
};

__device__ __forceinline__ PairTap pair_tap(const uint16_t* base, int i) {
    PairTap t;
    t.w = reinterpret_cast<const uint32_t*>(base + (i & ~1));
    t.sel = (i & 1) ? 0x5432u : 0x3210u;
    return t;
}

__device__ __forceinline__ uint32_t load_pair(const PairTap& t, int word_off) {
    return __byte_perm(t.w[word_off], t.w[word_off + 1], t.sel);
}

// A tap whose pair is one aligned word: of the plane itself when the pair
// starts on an even sample, of a copy shifted by one sample when it starts
// on an odd one.
struct WordTap {
    const uint32_t* w;
};

__device__ __forceinline__ uint32_t load_pair(const WordTap& t, int word_off) { return t.w[word_off]; }

template <bool MASK_MAX>
__device__ __forceinline__ void pair_tap_step(uint32_t v, uint32_t cur, uint32_t t2, int s, uint32_t smask, uint32_t w,
                                              uint32_t& accp, uint32_t& acct, uint32_t& mn, uint32_t& mx) {
    const uint32_t hi = vmax2(v, cur), lo = vmin2(v, cur);
    const uint32_t ad = hi - lo;
    const uint32_t sh = (ad >> s) & smask;
    const uint32_t m = t2 - vmin2(sh, t2);
    const uint32_t c = vmin2(ad, m);
    const uint32_t cp = vmin2(c, hi - cur);
    accp += w * cp;
    acct += w * c;
    mn = vmin2(mn, v);
    mx = vmax2(mx, MASK_MAX ? (v & 0x3FFF3FFFu) : v);
}

// Which tap sets a tile's blocks use.  vaco's filter_block clamps the result
// to the min/max of every available tap, but when only one tap set has a
// non-zero strength that clamp never binds: the set's weights sum to 12 <= 16
// and |constrain(d)| <= |d|, so cur + Round(sum/16) stays inside the taps'
// range (for sum > 0: (8 + 12 D) >> 4 <= D for every D >= 0, D = max - cur;
// for sum < 0: (7 - 12 E) >> 4 >= -E, E = cur - min).  A zero strength also
// makes every constrain() of its set 0.  So the taps of a set whose preset
// strength is zero are skipped altogether (pri_on / sec_on, uniform over a
// tile), bit-exactly: the clamp over the remaining set is a no-op.

// Filter the pixel pair whose left sample is at `s` (4-byte aligned).  `taps`
// are the 12 tap positions of the block for this lane, `row` the word offset
// of the current row relative to the block's first row.  MASK_MAX: the tile
// touches a plane edge, so sentinel samples must not raise the maximum.
template <bool MASK_MAX, class Tap>
__device__ __forceinline__ uint32_t filter_pair(uint32_t cur, const Tap* taps, int row, const PairBlock& f,
                                                bool pri_on, bool sec_on) {
    const uint32_t tp = f.pri | ((uint32_t)f.pri << 16), ts = f.sec | ((uint32_t)f.sec << 16);
    const uint32_t pm = (0xFFFFu >> f.pri_shift) * 0x10001u, sm = (0xFFFFu >> f.sec_shift) * 0x10001u;
    uint32_t accp = 0, acct = 0, mn = cur, mx = cur;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const uint32_t wp = k ? f.pt1 : f.pt0, ws = 2 - k;
        if (pri_on) {
            pair_tap_step<MASK_MAX>(load_pair(taps[2 * k], row), cur, tp, f.pri_shift, pm, wp, accp, acct, mn, mx);
            pair_tap_step<MASK_MAX>(load_pair(taps[2 * k + 1], row), cur, tp, f.pri_shift, pm, wp, accp, acct, mn, mx);
        }
        if (sec_on) {
            pair_tap_step<MASK_MAX>(load_pair(taps[4 + 2 * k], row), cur, ts, f.sec_shift, sm, ws, accp, acct, mn, mx);
            pair_tap_step<MASK_MAX>(load_pair(taps[4 + 2 * k + 1], row), cur, ts, f.sec_shift, sm, ws, accp, acct, mn,
                                    mx);
            pair_tap_step<MASK_MAX>(load_pair(taps[8 + 2 * k], row), cur, ts, f.sec_shift, sm, ws, accp, acct, mn, mx);
            pair_tap_step<MASK_MAX>(load_pair(taps[8 + 2 * k + 1], row), cur, ts, f.sec_shift, sm, ws, accp, acct, mn,
                                    mx);
        }
    }
    const uint32_t accn = acct - accp;
    const uint32_t both = vmin2(accp, accn);
    const uint32_t rp = ((accp - both + 0x00080008u) >> 4) & 0x0FFF0FFFu;
    const uint32_t rn = ((accn - both + 0x00080008u) >> 4) & 0x0FFF0FFFu;
    return vmin2(vmax2(cur + rp, mn + rn) - rn, mx);
}

}  // namespace cdefk
}  // namespace vaco
