// deblock_core.cuh -- AV1 loop-filter device functions (spec 7.14.4-7.14.6)
// shared by the standalone deblocking kernels and the fused deblock+CDEF
// kernel.  vaco has no deblocking filter (crates/codec/vaco-codec-av1/src/lib.rs:16-18).
#pragma once

#include "common.cuh"
#include "kernels.cuh"

namespace vaco {
namespace dbk {

struct Strength {
    int limit, blimit, thresh;
};

// 7.14.4: limit / blimit / thresh from the level and sharpness.
__device__ __forceinline__ Strength strength_of(int lvl, int sharpness) {
    int shift = sharpness > 4 ? 2 : sharpness > 0 ? 1 : 0;
    int limit = sharpness > 0 ? clampi(lvl >> shift, 1, 9 - sharpness) : max(1, lvl >> shift);
    return Strength{limit, 2 * (lvl + 2) + limit, lvl >> 4};
}

// One line of samples across an edge; q0 at `q`, samples `step` apart.
// nq / np: samples that exist on the q / p side inside the plane (reads past
// them repeat the last one, writes past them are dropped).
__device__ __forceinline__ void filter_line(uint16_t* q, long step, int nq, int np, int plane, int size,
                                            const Strength& s, int bd) {
    const int reach = size == 16 ? 7 : 4;
    int Q[7], Pp[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        if (k < reach) {
            Q[k] = q[step * min(k, nq - 1)];
            Pp[k] = q[-step * min(k + 1, np)];
        } else {
            Q[k] = Pp[k] = 0;
        }
    }
    const int len = size == 4 ? 4 : plane != 0 ? 6 : size == 8 ? 8 : 16;
    const int sh = bd - 8;
    const int limit = s.limit << sh, blimit = s.blimit << sh, thresh = s.thresh << sh;
    const bool hev = abs(Pp[1] - Pp[0]) > thresh || abs(Q[1] - Q[0]) > thresh;
    bool mask = abs(Pp[1] - Pp[0]) > limit || abs(Q[1] - Q[0]) > limit ||
                abs(Pp[0] - Q[0]) * 2 + abs(Pp[1] - Q[1]) / 2 > blimit;
    if (len >= 6) mask = mask || abs(Pp[2] - Pp[1]) > limit || abs(Q[2] - Q[1]) > limit;
    if (len >= 8) mask = mask || abs(Pp[3] - Pp[2]) > limit || abs(Q[3] - Q[2]) > limit;
    if (mask) return;
    const int one = 1 << sh;
    bool flat = false, flat2 = false;
    if (size >= 8) {
        bool f = abs(Pp[1] - Pp[0]) > one || abs(Q[1] - Q[0]) > one || abs(Pp[2] - Pp[0]) > one ||
                 abs(Q[2] - Q[0]) > one;
        if (len >= 8) f = f || abs(Pp[3] - Pp[0]) > one || abs(Q[3] - Q[0]) > one;
        flat = !f;
    }
    if (size >= 16) {
        bool f = abs(Pp[6] - Pp[0]) > one || abs(Q[6] - Q[0]) > one || abs(Pp[5] - Pp[0]) > one ||
                 abs(Q[5] - Q[0]) > one || abs(Pp[4] - Pp[0]) > one || abs(Q[4] - Q[0]) > one;
        flat2 = !f;
    }
    auto put = [&](int k, int v) {
        if (k >= 0 ? k < nq : -k <= np) q[step * k] = (uint16_t)v;
    };
    if (size == 4 || !flat) {
        // 7.14.6.3 narrow filter
        const int half = 0x80 << sh, lo = -(1 << (bd - 1)), hi = (1 << (bd - 1)) - 1;
        const int ps1 = Pp[1] - half, ps0 = Pp[0] - half, qs0 = Q[0] - half, qs1 = Q[1] - half;
        int f = hev ? clampi(ps1 - qs1, lo, hi) : 0;
        f = clampi(f + 3 * (qs0 - ps0), lo, hi);
        const int f1 = clampi(f + 4, lo, hi) >> 3;
        const int f2 = clampi(f + 3, lo, hi) >> 3;
        put(0, clampi(qs0 - f1, lo, hi) + half);
        put(-1, clampi(ps0 + f2, lo, hi) + half);
        if (!hev) {
            const int f3 = (f1 + 1) >> 1;
            put(1, clampi(qs1 - f3, lo, hi) + half);
            put(-2, clampi(ps1 + f3, lo, hi) + half);
        }
        return;
    }
    // 7.14.6.4 wide filters: F[k] = q_k (k >= 0), p_{-k-1} (k < 0)
    if (size == 8 || !flat2) {
        if (plane == 0) {  // 8-tap, n = 3, center tap weight 2
            const int p3 = Pp[3], p2 = Pp[2], p1 = Pp[1], p0 = Pp[0], q0 = Q[0], q1 = Q[1], q2 = Q[2], q3 = Q[3];
            put(-3, (3 * p3 + 2 * p2 + p1 + p0 + q0 + 4) >> 3);
            put(-2, (2 * p3 + p2 + 2 * p1 + p0 + q0 + q1 + 4) >> 3);
            put(-1, (p3 + p2 + p1 + 2 * p0 + q0 + q1 + q2 + 4) >> 3);
            put(0, (p2 + p1 + p0 + 2 * q0 + q1 + q2 + q3 + 4) >> 3);
            put(1, (p1 + p0 + q0 + 2 * q1 + q2 + 2 * q3 + 4) >> 3);
            put(2, (p0 + q0 + q1 + 2 * q2 + 3 * q3 + 4) >> 3);
        } else {  // 6-tap chroma, n = 2, taps within |j| <= 1 weigh 2
            const int p2 = Pp[2], p1 = Pp[1], p0 = Pp[0], q0 = Q[0], q1 = Q[1], q2 = Q[2];
            put(-2, (3 * p2 + 2 * p1 + 2 * p0 + q0 + 4) >> 3);
            put(-1, (p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3);
            put(0, (p1 + 2 * p0 + 2 * q0 + 2 * q1 + q2 + 4) >> 3);
            put(1, (p0 + 2 * q0 + 2 * q1 + 3 * q2 + 4) >> 3);
        }
        return;
    }
    // 14-tap, n = 6, log2 size 4
    int F[14];
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        F[7 + k] = Q[k];
        F[6 - k] = Pp[k];
    }
    int out[12];
#pragma unroll
    for (int i = -6; i < 6; ++i) {
        int t = 0;
#pragma unroll
        for (int j = -6; j <= 6; ++j) {
            int pos = min(max(i + j, -7), 6);
            t += F[pos + 7] * ((j >= -1 && j <= 1) ? 2 : 1);
        }
        out[i + 6] = (t + 8) >> 4;
    }
#pragma unroll
    for (int i = -6; i < 6; ++i) put(i, out[i + 6]);
}

__device__ __forceinline__ int level_at(const DeblockLaunch& L, int plane, int pass, int row, int col) {
    const int i = plane == 0 ? pass : plane + 1;
    if (L.lvl_map) return L.lvl_map[((long)row * L.mi_cols + col) * 4 + i];
    return L.levels[i];
}

}  // namespace dbk
}  // namespace vaco

namespace vaco {
namespace dbk {

// ---------------------------------------------------------------- size-class line filters
//
// The same arithmetic as filter_line(), split by filter size so that a warp
// runs one class at a time.  q points at q0; sample k of the line (k < 0 is
// the p side) lives at q[k * step].  nq / np count the samples that exist on
// each side inside the plane: when both reach past the filter's span the
// loads need no clamping, otherwise reads repeat the last sample and writes
// past the plane are dropped (the get_clamped / set semantics of the oracle).

template <int R, int STEP>
__device__ __forceinline__ void load_line(const uint16_t* q, long step_rt, int nq, int np, int* Pv, int* Qv) {
    const long step = STEP ? STEP : step_rt;
    if (nq >= R && np >= R) {
#pragma unroll
        for (int k = 0; k < R; ++k) {
            Qv[k] = q[k * step];
            Pv[k] = q[-(k + 1) * step];
        }
    } else {
#pragma unroll
        for (int k = 0; k < R; ++k) {
            Qv[k] = q[min(k, nq - 1) * step];
            Pv[k] = q[-min(k + 1, np) * step];
        }
    }
}

template <int STEP>
__device__ __forceinline__ void store_at(uint16_t* q, long step_rt, int nq, int np, int k, int v) {
    const long step = STEP ? STEP : step_rt;
    if (k >= 0 ? k < nq : -k <= np) q[k * step] = (uint16_t)v;
}

// 7.14.6.3 narrow filter on p1, p0, q0, q1.
template <int STEP>
__device__ __forceinline__ void narrow_apply(uint16_t* q, long step_rt, int nq, int np, int p1, int p0, int q0, int q1,
                                             bool hev, int bd) {
    const int sh = bd - 8, half = 0x80 << sh, lo = -(1 << (bd - 1)), hi = (1 << (bd - 1)) - 1;
    const int ps1 = p1 - half, ps0 = p0 - half, qs0 = q0 - half, qs1 = q1 - half;
    int f = hev ? clampi(ps1 - qs1, lo, hi) : 0;
    f = clampi(f + 3 * (qs0 - ps0), lo, hi);
    const int f1 = clampi(f + 4, lo, hi) >> 3;
    const int f2 = clampi(f + 3, lo, hi) >> 3;
    store_at<STEP>(q, step_rt, nq, np, 0, clampi(qs0 - f1, lo, hi) + half);
    store_at<STEP>(q, step_rt, nq, np, -1, clampi(ps0 + f2, lo, hi) + half);
    if (!hev) {
        const int f3 = (f1 + 1) >> 1;
        store_at<STEP>(q, step_rt, nq, np, 1, clampi(qs1 - f3, lo, hi) + half);
        store_at<STEP>(q, step_rt, nq, np, -2, clampi(ps1 + f3, lo, hi) + half);
    }
}

// Filter size 4 (luma or chroma): mask over p1..q1, narrow filter.
template <int STEP>
__device__ __forceinline__ void line_size4(uint16_t* q, long step_rt, int nq, int np, const Strength& s, int bd) {
    int P[2], Q[2];
    load_line<2, STEP>(q, step_rt, nq, np, P, Q);
    const int sh = bd - 8;
    const int limit = s.limit << sh, blimit = s.blimit << sh, thresh = s.thresh << sh;
    const int d_p = abs(P[1] - P[0]), d_q = abs(Q[1] - Q[0]);
    if (max(d_p, d_q) > limit || abs(P[0] - Q[0]) * 2 + abs(P[1] - Q[1]) / 2 > blimit) return;
    narrow_apply<STEP>(q, step_rt, nq, np, P[1], P[0], Q[0], Q[1], max(d_p, d_q) > thresh, bd);
}

// Filter size 8 on a chroma plane (filter length 6).
template <int STEP>
__device__ __forceinline__ void line_size6(uint16_t* q, long step_rt, int nq, int np, const Strength& s, int bd) {
    int P[3], Q[3];
    load_line<3, STEP>(q, step_rt, nq, np, P, Q);
    const int sh = bd - 8;
    const int limit = s.limit << sh, blimit = s.blimit << sh, thresh = s.thresh << sh;
    const int d_p = abs(P[1] - P[0]), d_q = abs(Q[1] - Q[0]);
    const int m = max(max(d_p, d_q), max(abs(P[2] - P[1]), abs(Q[2] - Q[1])));
    if (m > limit || abs(P[0] - Q[0]) * 2 + abs(P[1] - Q[1]) / 2 > blimit) return;
    const int one = 1 << sh;
    const bool flat = max(max(d_p, d_q), max(abs(P[2] - P[0]), abs(Q[2] - Q[0]))) <= one;
    if (!flat) {
        narrow_apply<STEP>(q, step_rt, nq, np, P[1], P[0], Q[0], Q[1], max(d_p, d_q) > thresh, bd);
        return;
    }
    const int p2 = P[2], p1 = P[1], p0 = P[0], q0 = Q[0], q1 = Q[1], q2 = Q[2];
    store_at<STEP>(q, step_rt, nq, np, -2, (3 * p2 + 2 * p1 + 2 * p0 + q0 + 4) >> 3);
    store_at<STEP>(q, step_rt, nq, np, -1, (p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3);
    store_at<STEP>(q, step_rt, nq, np, 0, (p1 + 2 * p0 + 2 * q0 + 2 * q1 + q2 + 4) >> 3);
    store_at<STEP>(q, step_rt, nq, np, 1, (p0 + 2 * q0 + 2 * q1 + 3 * q2 + 4) >> 3);
}

template <int STEP>
__device__ __forceinline__ void apply8(uint16_t* q, long step_rt, int nq, int np, const int* P, const int* Q) {
    const int p3 = P[3], p2 = P[2], p1 = P[1], p0 = P[0], q0 = Q[0], q1 = Q[1], q2 = Q[2], q3 = Q[3];
    store_at<STEP>(q, step_rt, nq, np, -3, (3 * p3 + 2 * p2 + p1 + p0 + q0 + 4) >> 3);
    store_at<STEP>(q, step_rt, nq, np, -2, (2 * p3 + p2 + 2 * p1 + p0 + q0 + q1 + 4) >> 3);
    store_at<STEP>(q, step_rt, nq, np, -1, (p3 + p2 + p1 + 2 * p0 + q0 + q1 + q2 + 4) >> 3);
    store_at<STEP>(q, step_rt, nq, np, 0, (p2 + p1 + p0 + 2 * q0 + q1 + q2 + q3 + 4) >> 3);
    store_at<STEP>(q, step_rt, nq, np, 1, (p1 + p0 + q0 + 2 * q1 + q2 + 2 * q3 + 4) >> 3);
    store_at<STEP>(q, step_rt, nq, np, 2, (p0 + q0 + q1 + 2 * q2 + 3 * q3 + 4) >> 3);
}

// Filter size 8 on luma (filter length 8).
template <int STEP>
__device__ __forceinline__ void line_size8(uint16_t* q, long step_rt, int nq, int np, const Strength& s, int bd) {
    int P[4], Q[4];
    load_line<4, STEP>(q, step_rt, nq, np, P, Q);
    const int sh = bd - 8;
    const int limit = s.limit << sh, blimit = s.blimit << sh, thresh = s.thresh << sh;
    const int d_p = abs(P[1] - P[0]), d_q = abs(Q[1] - Q[0]);
    const int m = max(max(max(d_p, d_q), max(abs(P[2] - P[1]), abs(Q[2] - Q[1]))),
                      max(abs(P[3] - P[2]), abs(Q[3] - Q[2])));
    if (m > limit || abs(P[0] - Q[0]) * 2 + abs(P[1] - Q[1]) / 2 > blimit) return;
    const int one = 1 << sh;
    const int fl = max(max(max(d_p, d_q), max(abs(P[2] - P[0]), abs(Q[2] - Q[0]))),
                       max(abs(P[3] - P[0]), abs(Q[3] - Q[0])));
    if (fl > one) {
        narrow_apply<STEP>(q, step_rt, nq, np, P[1], P[0], Q[0], Q[1], max(d_p, d_q) > thresh, bd);
        return;
    }
    apply8<STEP>(q, step_rt, nq, np, P, Q);
}

// Filter size 16 on luma: narrow, 8-tap or 14-tap by the flat masks.
template <int STEP>
__device__ __forceinline__ void line_size16(uint16_t* q, long step_rt, int nq, int np, const Strength& s, int bd) {
    int P[7], Q[7];
    load_line<7, STEP>(q, step_rt, nq, np, P, Q);
    const int sh = bd - 8;
    const int limit = s.limit << sh, blimit = s.blimit << sh, thresh = s.thresh << sh;
    const int d_p = abs(P[1] - P[0]), d_q = abs(Q[1] - Q[0]);
    const int m = max(max(max(d_p, d_q), max(abs(P[2] - P[1]), abs(Q[2] - Q[1]))),
                      max(abs(P[3] - P[2]), abs(Q[3] - Q[2])));
    if (m > limit || abs(P[0] - Q[0]) * 2 + abs(P[1] - Q[1]) / 2 > blimit) return;
    const int one = 1 << sh;
    const int fl = max(max(max(d_p, d_q), max(abs(P[2] - P[0]), abs(Q[2] - Q[0]))),
                       max(abs(P[3] - P[0]), abs(Q[3] - Q[0])));
    if (fl > one) {
        narrow_apply<STEP>(q, step_rt, nq, np, P[1], P[0], Q[0], Q[1], max(d_p, d_q) > thresh, bd);
        return;
    }
    const int fl2 = max(max(max(abs(P[6] - P[0]), abs(Q[6] - Q[0])), max(abs(P[5] - P[0]), abs(Q[5] - Q[0]))),
                        max(abs(P[4] - P[0]), abs(Q[4] - Q[0])));
    if (fl2 > one) {
        apply8<STEP>(q, step_rt, nq, np, P, Q);
        return;
    }
    // 14-tap (7.14.6.4, log2Size 4): out[i] = Round2(T_i + U_i, 4) with
    // T_i the 13-sample window sum (edge-clamped) and U_i = F[i-1]+F[i]+F[i+1].
    int F[14];
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        F[6 - k] = P[k];
        F[7 + k] = Q[k];
    }
    int T = 6 * F[0];
#pragma unroll
    for (int k = 1; k <= 7; ++k) T += F[k];  // window of i = -6: F[0]x7 .. F[7]
    int out[12];
#pragma unroll
    for (int i = -6; i < 6; ++i) {
        const int c = i + 7;  // F index of output i
        out[i + 6] = (T + F[c - 1] + F[c] + F[c + 1] + 8) >> 4;
        if (i < 5) T += F[min(c + 7, 13)] - F[max(c - 6, 0)];
    }
#pragma unroll
    for (int i = -6; i < 6; ++i) store_at<STEP>(q, step_rt, nq, np, i, out[i + 6]);
}

// ---------------------------------------------------------------- two lines per register
//
// The size-class filters above for two adjacent lines of one edge segment at
// once: sample k of both lines sits in one 32-bit word, the first line in the
// low 16 bits.  Both lines share the segment's filter size and strengths;
// each keeps its own masks (filterMask, hev, flat, flat2 of 7.14.6.2), which
// select per 16-bit half between the original samples and the narrow, 8-tap
// or 14-tap results, so the lines never diverge.  Every per-half quantity
// stays in [0, 65535], so plain 32-bit adds and subtracts never carry or
// borrow across halves:
//   - samples are at most 4095 (12-bit); |a - b| = max(a, b) - min(a, b);
//   - the wide filters' weighted sums are at most 16 x 4095 + 8;
//   - the narrow filter's signed intermediates (7.14.6.3) are held biased by
//     kNarrowBias = 2^14, whose magnitude exceeds every negative value they
//     take (|ps1 - qs1| + 3 |qs0 - ps0| <= 4 x 4095), and whose multiples of
//     8 and 16 keep the arithmetic shifts exact: (v + 2^14) >> 3 =
//     (v >> 3) + 2^11 for any v > -2^14.
// The callers use these only where the segment reaches R samples into the
// plane on both sides (no clamped reads, no dropped writes); nearer the plane
// edge they run the per-line filters above.

__device__ __forceinline__ uint32_t pmin2(uint32_t a, uint32_t b) {
    uint32_t d;
    asm("min.u16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
__device__ __forceinline__ uint32_t pmax2(uint32_t a, uint32_t b) {
    uint32_t d;
    asm("max.u16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
__device__ __forceinline__ constexpr uint32_t pk2(int v) { return (uint32_t)v * 0x10001u; }
__device__ __forceinline__ uint32_t absd2(uint32_t a, uint32_t b) { return pmax2(a, b) - pmin2(a, b); }
// Per half: non-zero iff a > t.
__device__ __forceinline__ uint32_t over2(uint32_t a, uint32_t t) { return pmax2(a, t) - t; }
// Per half: 0xFFFF where x's half is non-zero, else 0.
__device__ __forceinline__ uint32_t mask2(uint32_t x) { return pmin2(x, 0x00010001u) * 0xFFFFu; }
// Per half: m ? a : b.
__device__ __forceinline__ uint32_t sel2(uint32_t m, uint32_t a, uint32_t b) { return (a & m) | (b & ~m); }

constexpr int kNarrowBias = 1 << 14;

// Packed limit / blimit / thresh / flatness bound of a segment (7.14.4),
// scaled to the bit depth (sh = bit depth - 8).
struct __align__(16) PairStrength {
    uint32_t limit, blimit, thresh, one;
};

__device__ __forceinline__ PairStrength pair_strength(const Strength& s, int sh) {
    return PairStrength{pk2(s.limit << sh), pk2(s.blimit << sh), pk2(s.thresh << sh), pk2(1 << sh)};
}

// 2 |p0 - q0| + |p1 - q1| / 2, the blimit side of filterMask.
__device__ __forceinline__ uint32_t blimit_term2(const uint32_t* P, const uint32_t* Q) {
    return absd2(P[0], Q[0]) * 2u + ((absd2(P[1], Q[1]) >> 1) & 0x7FFF7FFFu);
}

// 7.14.6.3 narrow filter of both halves (hevm: 0xFFFF where hev), in place.
__device__ __forceinline__ void narrow2(uint32_t& p1, uint32_t& p0, uint32_t& q0, uint32_t& q1, uint32_t hevm,
                                        int sh) {
    const int half = 0x80 << sh;
    const uint32_t lo = pk2(kNarrowBias - half), hi = pk2(kNarrowBias + half - 1);
    // f = hev ? clamp(ps1 - qs1) : 0, then clamp(f + 3 (qs0 - ps0)); biased
    uint32_t f = sel2(hevm, pmin2(pmax2(p1 + pk2(kNarrowBias) - q1, lo), hi), pk2(kNarrowBias));
    f = pmin2(pmax2(f + 3u * q0 - 3u * p0, lo), hi);
    // f1 = clamp(f + 4) >> 3, f2 = clamp(f + 3) >> 3, f3 = (f1 + 1) >> 1, each
    // plus the bias shifted alike (2^11 for f1 and f2, 2^10 for f3)
    const uint32_t f1 = (pmin2(f + pk2(4), hi) >> 3) & 0x1FFF1FFFu;
    const uint32_t f2 = (pmin2(f + pk2(3), hi) >> 3) & 0x1FFF1FFFu;
    const uint32_t f3 = ((f1 + pk2(1)) >> 1) & 0x7FFF7FFFu;
    // clamp(qs0 - f1) + half and so on: the biased value minus (bias - half)
    const uint32_t nq0 = pmin2(pmax2(q0 + pk2(kNarrowBias + kNarrowBias / 8 - half) - f1, lo), hi) - lo;
    const uint32_t np0 = pmin2(pmax2(p0 + f2 + pk2(kNarrowBias - half - kNarrowBias / 8), lo), hi) - lo;
    const uint32_t nq1 = pmin2(pmax2(q1 + pk2(kNarrowBias + kNarrowBias / 16 - half) - f3, lo), hi) - lo;
    const uint32_t np1 = pmin2(pmax2(p1 + f3 + pk2(kNarrowBias - half - kNarrowBias / 16), lo), hi) - lo;
    q0 = nq0;
    p0 = np0;
    q1 = sel2(hevm, q1, nq1);
    p1 = sel2(hevm, p1, np1);
}

// Samples -R .. R-1 of the lane's two lines, q at sample 0 of the first line
// (4-byte aligned).  PASS 1 (horizontal edge): the lines are adjacent
// columns, so sample k of both is one word k rows away.  PASS 0 (vertical
// edge): the lines are adjacent rows; words of two samples along each row
// are interleaved into (row 0, row 1) pairs.  P[k] is sample -(k+1).
template <int PASS, int R>
__device__ __forceinline__ void load_pair(const uint16_t* q, int pitch, uint32_t* P, uint32_t* Q) {
    if (PASS == 1) {
        const uint32_t* w = reinterpret_cast<const uint32_t*>(q);
        const int wp = pitch >> 1;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            Q[k] = w[k * wp];
            P[k] = w[-(k + 1) * wp];
        }
    } else {
        const uint32_t* r0 = reinterpret_cast<const uint32_t*>(q);
        const uint32_t* r1 = reinterpret_cast<const uint32_t*>(q + pitch);
#pragma unroll
        for (int j = 0; j < (R + 1) / 2; ++j) {
            uint32_t a = r0[j], b = r1[j];  // samples 2j, 2j+1
            Q[2 * j] = __byte_perm(a, b, 0x5410);
            if (2 * j + 1 < R) Q[2 * j + 1] = __byte_perm(a, b, 0x7632);
            a = r0[-(j + 1)];  // samples -2j-2, -2j-1
            b = r1[-(j + 1)];
            P[2 * j] = __byte_perm(a, b, 0x7632);
            if (2 * j + 1 < R) P[2 * j + 1] = __byte_perm(a, b, 0x5410);
        }
    }
}

// Stores samples -NP .. NQ-1 of both lines (the layout of load_pair).  For
// PASS 0, NP and NQ are even: whole words along each row.
template <int PASS, int NP, int NQ>
__device__ __forceinline__ void store_pair(uint16_t* q, int pitch, const uint32_t* P, const uint32_t* Q) {
    if (PASS == 1) {
        uint32_t* w = reinterpret_cast<uint32_t*>(q);
        const int wp = pitch >> 1;
#pragma unroll
        for (int k = 0; k < NQ; ++k) w[k * wp] = Q[k];
#pragma unroll
        for (int k = 0; k < NP; ++k) w[-(k + 1) * wp] = P[k];
    } else {
        uint32_t* r0 = reinterpret_cast<uint32_t*>(q);
        uint32_t* r1 = reinterpret_cast<uint32_t*>(q + pitch);
#pragma unroll
        for (int j = 0; j < NQ / 2; ++j) {
            r0[j] = __byte_perm(Q[2 * j], Q[2 * j + 1], 0x5410);
            r1[j] = __byte_perm(Q[2 * j], Q[2 * j + 1], 0x7632);
        }
#pragma unroll
        for (int j = 0; j < NP / 2; ++j) {
            r0[-(j + 1)] = __byte_perm(P[2 * j + 1], P[2 * j], 0x5410);
            r1[-(j + 1)] = __byte_perm(P[2 * j + 1], P[2 * j], 0x7632);
        }
    }
}

// The 8-tap outputs (samples -3 .. 2) of apply8 into w[0..5].
__device__ __forceinline__ void wide8_2(const uint32_t* P, const uint32_t* Q, uint32_t* w) {
    const uint32_t p3 = P[3], p2 = P[2], p1 = P[1], p0 = P[0], q0 = Q[0], q1 = Q[1], q2 = Q[2], q3 = Q[3];
    const uint32_t r = pk2(4), m = 0x1FFF1FFFu;
    w[0] = ((3u * p3 + 2u * p2 + p1 + p0 + q0 + r) >> 3) & m;
    w[1] = ((2u * p3 + p2 + 2u * p1 + p0 + q0 + q1 + r) >> 3) & m;
    w[2] = ((p3 + p2 + p1 + 2u * p0 + q0 + q1 + q2 + r) >> 3) & m;
    w[3] = ((p2 + p1 + p0 + 2u * q0 + q1 + q2 + q3 + r) >> 3) & m;
    w[4] = ((p1 + p0 + q0 + 2u * q1 + q2 + 2u * q3 + r) >> 3) & m;
    w[5] = ((p0 + q0 + q1 + 2u * q2 + 3u * q3 + r) >> 3) & m;
}

// Filter size 4: mask over p1..q1, narrow filter.
template <int PASS>
__device__ __forceinline__ void pair_size4(uint16_t* q, int pitch, const PairStrength& s, int sh) {
    uint32_t P[2], Q[2];
    load_pair<PASS, 2>(q, pitch, P, Q);
    const uint32_t dpq = pmax2(absd2(P[1], P[0]), absd2(Q[1], Q[0]));
    const uint32_t keep = mask2(over2(dpq, s.limit) | over2(blimit_term2(P, Q), s.blimit));
    if (keep == 0xFFFFFFFFu) return;
    uint32_t p1 = P[1], p0 = P[0], q0 = Q[0], q1 = Q[1];
    narrow2(p1, p0, q0, q1, mask2(over2(dpq, s.thresh)), sh);
    P[1] = sel2(keep, P[1], p1);
    P[0] = sel2(keep, P[0], p0);
    Q[0] = sel2(keep, Q[0], q0);
    Q[1] = sel2(keep, Q[1], q1);
    store_pair<PASS, 2, 2>(q, pitch, P, Q);
}

// Filter size 8 on a chroma plane (filter length 6).
template <int PASS>
__device__ __forceinline__ void pair_size6(uint16_t* q, int pitch, const PairStrength& s, int sh) {
    uint32_t P[3], Q[3];
    load_pair<PASS, 3>(q, pitch, P, Q);
    const uint32_t dpq = pmax2(absd2(P[1], P[0]), absd2(Q[1], Q[0]));
    const uint32_t m = pmax2(dpq, pmax2(absd2(P[2], P[1]), absd2(Q[2], Q[1])));
    const uint32_t keep = mask2(over2(m, s.limit) | over2(blimit_term2(P, Q), s.blimit));
    if (keep == 0xFFFFFFFFu) return;
    const uint32_t steep = mask2(over2(pmax2(dpq, pmax2(absd2(P[2], P[0]), absd2(Q[2], Q[0]))), s.one));
    uint32_t p1 = P[1], p0 = P[0], q0 = Q[0], q1 = Q[1];
    narrow2(p1, p0, q0, q1, mask2(over2(dpq, s.thresh)), sh);
    if ((~steep & ~keep) != 0) {  // a flat line: the 6-tap filter
        const uint32_t p2 = P[2], q2 = Q[2], r = pk2(4), mk = 0x1FFF1FFFu;
        p1 = sel2(steep, p1, ((3u * p2 + 2u * P[1] + 2u * P[0] + Q[0] + r) >> 3) & mk);
        const uint32_t w0 = ((p2 + 2u * P[1] + 2u * P[0] + 2u * Q[0] + Q[1] + r) >> 3) & mk;
        const uint32_t w1 = ((P[1] + 2u * P[0] + 2u * Q[0] + 2u * Q[1] + q2 + r) >> 3) & mk;
        q1 = sel2(steep, q1, ((P[0] + 2u * Q[0] + 2u * Q[1] + 3u * q2 + r) >> 3) & mk);
        p0 = sel2(steep, p0, w0);
        q0 = sel2(steep, q0, w1);
    }
    P[1] = sel2(keep, P[1], p1);
    P[0] = sel2(keep, P[0], p0);
    Q[0] = sel2(keep, Q[0], q0);
    Q[1] = sel2(keep, Q[1], q1);
    store_pair<PASS, 2, 2>(q, pitch, P, Q);
}

// filterMask and the flat mask over p3..q3 (filter sizes 8 and 16 on luma).
__device__ __forceinline__ void masks8_2(const uint32_t* P, const uint32_t* Q, const PairStrength& s, uint32_t& dpq,
                                         uint32_t& keep, uint32_t& steep) {
    dpq = pmax2(absd2(P[1], P[0]), absd2(Q[1], Q[0]));
    const uint32_t m = pmax2(pmax2(dpq, pmax2(absd2(P[2], P[1]), absd2(Q[2], Q[1]))),
                             pmax2(absd2(P[3], P[2]), absd2(Q[3], Q[2])));
    keep = mask2(over2(m, s.limit) | over2(blimit_term2(P, Q), s.blimit));
    const uint32_t fl = pmax2(pmax2(dpq, pmax2(absd2(P[2], P[0]), absd2(Q[2], Q[0]))),
                              pmax2(absd2(P[3], P[0]), absd2(Q[3], Q[0])));
    steep = mask2(over2(fl, s.one));
}

// Filter size 8 on luma (filter length 8).
template <int PASS>
__device__ __forceinline__ void pair_size8(uint16_t* q, int pitch, const PairStrength& s, int sh) {
    uint32_t P[4], Q[4];
    load_pair<PASS, 4>(q, pitch, P, Q);
    uint32_t dpq, keep, steep;
    masks8_2(P, Q, s, dpq, keep, steep);
    if (keep == 0xFFFFFFFFu) return;
    uint32_t p1 = P[1], p0 = P[0], q0 = Q[0], q1 = Q[1];
    narrow2(p1, p0, q0, q1, mask2(over2(dpq, s.thresh)), sh);
    const uint32_t n[4] = {p1, p0, q0, q1};
    if ((~steep & ~keep) == 0) {  // narrow lines only: samples -2 .. 1
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            P[k] = sel2(keep, P[k], n[1 - k]);
            Q[k] = sel2(keep, Q[k], n[2 + k]);
        }
        store_pair<PASS, 2, 2>(q, pitch, P, Q);
        return;
    }
    uint32_t w[6];
    wide8_2(P, Q, w);
    const uint32_t flat = ~steep & ~keep, narrow = steep & ~keep;
#pragma unroll
    for (int k = 0; k < 3; ++k) {  // samples -(k+1) and k
        uint32_t pv = sel2(flat, w[2 - k], P[k]), qv = sel2(flat, w[3 + k], Q[k]);
        if (k < 2) {
            pv = sel2(narrow, n[1 - k], pv);
            qv = sel2(narrow, n[2 + k], qv);
        }
        P[k] = pv;
        Q[k] = qv;
    }
    store_pair<PASS, PASS == 0 ? 4 : 3, PASS == 0 ? 4 : 3>(q, pitch, P, Q);
}

// Filter size 16 on luma: narrow, 8-tap or 14-tap by the flat masks.
template <int PASS>
__device__ __forceinline__ void pair_size16(uint16_t* q, int pitch, const PairStrength& s, int sh) {
    uint32_t P[7], Q[7];
    load_pair<PASS, 7>(q, pitch, P, Q);
    uint32_t dpq, keep, steep;
    masks8_2(P, Q, s, dpq, keep, steep);
    if (keep == 0xFFFFFFFFu) return;
    uint32_t p1 = P[1], p0 = P[0], q0 = Q[0], q1 = Q[1];
    narrow2(p1, p0, q0, q1, mask2(over2(dpq, s.thresh)), sh);
    const uint32_t n[4] = {p1, p0, q0, q1};
    const uint32_t flat = ~steep & ~keep, narrow = steep & ~keep;
    if (flat == 0) {  // narrow lines only: samples -2 .. 1
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            P[k] = sel2(keep, P[k], n[1 - k]);
            Q[k] = sel2(keep, Q[k], n[2 + k]);
        }
        store_pair<PASS, 2, 2>(q, pitch, P, Q);
        return;
    }
    const uint32_t fl2 = pmax2(pmax2(pmax2(absd2(P[6], P[0]), absd2(Q[6], Q[0])),
                                     pmax2(absd2(P[5], P[0]), absd2(Q[5], Q[0]))),
                               pmax2(absd2(P[4], P[0]), absd2(Q[4], Q[0])));
    const uint32_t flat2 = flat & ~mask2(over2(fl2, s.one)), flat1 = flat & ~flat2;
    uint32_t w[6];
    wide8_2(P, Q, w);
    uint32_t o[12];  // outputs of samples -6 .. 5
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        o[5 - k] = P[k];
        o[6 + k] = Q[k];
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) o[3 + k] = sel2(flat1, w[k], o[3 + k]);
#pragma unroll
    for (int k = 0; k < 4; ++k) o[4 + k] = sel2(narrow, n[k], o[4 + k]);
    if (flat2 != 0) {
        // 14-tap (log2Size 4): out[i] = (T_i + F[i-1] + F[i] + F[i+1] + 8) >> 4
        // with T_i the edge-clamped 13-sample window sum, as line_size16
        uint32_t F[14];
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            F[6 - k] = P[k];
            F[7 + k] = Q[k];
        }
        uint32_t T = 6u * F[0];
#pragma unroll
        for (int k = 1; k <= 7; ++k) T += F[k];
#pragma unroll
        for (int i = -6; i < 6; ++i) {
            const int c = i + 7;
            o[i + 6] = sel2(flat2, ((T + F[c - 1] + F[c] + F[c + 1] + pk2(8)) >> 4) & 0x0FFF0FFFu, o[i + 6]);
            if (i < 5) T = T + F[min(c + 7, 13)] - F[max(c - 6, 0)];
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            P[k] = o[5 - k];
            Q[k] = o[6 + k];
        }
        store_pair<PASS, 6, 6>(q, pitch, P, Q);
        return;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        P[k] = o[5 - k];
        Q[k] = o[6 + k];
    }
    store_pair<PASS, PASS == 0 ? 4 : 3, PASS == 0 ? 4 : 3>(q, pitch, P, Q);
}

template <int PASS>
__device__ __forceinline__ void filter_pair_class(int cls, uint16_t* q, int pitch, const PairStrength& s, int sh) {
    if (cls == 0) pair_size4<PASS>(q, pitch, s, sh);
    else if (cls == 1) pair_size6<PASS>(q, pitch, s, sh);
    else if (cls == 2) pair_size8<PASS>(q, pitch, s, sh);
    else pair_size16<PASS>(q, pitch, s, sh);
}

// Samples per side a size class reads (and the per-line filters' clamping
// threshold): 4-tap 2, chroma 6-tap 3, luma 8-tap 4, luma 14-tap 7.
__device__ __forceinline__ int class_reach(int cls) { return cls == 0 ? 2 : cls == 1 ? 3 : cls == 2 ? 4 : 7; }

}  // namespace dbk
}  // namespace vaco
