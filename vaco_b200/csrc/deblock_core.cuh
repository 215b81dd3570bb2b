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

}  // namespace dbk
}  // namespace vaco
