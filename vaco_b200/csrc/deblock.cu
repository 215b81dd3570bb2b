// deblock.cu -- AV1 loop filter (spec 7.14) on sm_100a.
//
// vaco has no deblocking filter (crates/codec/vaco-codec-av1/src/lib.rs:16-18),
// so this follows the AV1 specification: edge loop filter (7.14.2), filter
// size (7.14.3), adaptive strength (7.14.4-7.14.5, levels supplied by the
// caller), filter masks (7.14.6.2), narrow filter (7.14.6.3) and wide
// filters (7.14.6.4), for intra frames (vaco decodes intra frames only,
// src/decode.rs:511-515), where an edge is filtered exactly when it is a
// transform edge.
//
// All vertical edges of a plane are filtered before any horizontal edge.
// Within one pass no two edges read or write a common sample (a filter of
// size S sits on an edge that is a multiple of S away from the next one and
// reaches at most S/2 - 1 samples deep on a side), so each pass runs one
// thread per edge line, in place.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"

namespace vaco {

namespace {

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

struct PassArgs {
    DeblockLaunch L;
    int plane_list[3];
    int nplanes;
};

__device__ __forceinline__ int level_at(const DeblockLaunch& L, int plane, int pass, int row, int col) {
    const int i = plane == 0 ? pass : plane + 1;
    if (L.lvl_map) return L.lvl_map[((long)row * L.mi_cols + col) * 4 + i];
    return L.levels[i];
}

// Pass 0: vertical edges.  x = edge index (plane column 4g), y = sample row.
__global__ void deblock_vertical_kernel(PassArgs a) {
    const DeblockLaunch& L = a.L;
    const int plane = a.plane_list[blockIdx.z];
    const DevPlane& P = L.pic[plane];
    const int g = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int yp = blockIdx.y * blockDim.y + threadIdx.y;
    const int xp = 4 * g;
    if (xp >= P.width || yp >= P.height) return;
    const int ssx = plane ? L.ssx : 0, ssy = plane ? L.ssy : 0;
    const int col = g << ssx, row = (yp >> 2) << ssy;
    if (col * 4 >= L.coded_width || row * 4 >= L.coded_height) return;
    const uint8_t* map = plane ? L.tx_chroma : L.tx_luma;
    const int map_cols = plane ? (L.mi_cols + L.ssx) >> L.ssx : L.mi_cols;
    const int cur = map[(long)(yp >> 2) * map_cols + g], prev = map[(long)(yp >> 2) * map_cols + g - 1];
    const int wl = tx_w_log2(cur);
    if (xp & ((1 << wl) - 1)) return;
    const int base = min(wl, tx_w_log2(prev));
    const int size = min(plane ? 8 : 16, 1 << base);
    const int r = row | ssy, c = col | ssx;
    int lvl = level_at(L, plane, 0, r, c);
    if (lvl == 0) lvl = level_at(L, plane, 0, r, c - (1 << ssx));
    if (lvl == 0) return;
    const Strength s = strength_of(lvl, L.sharpness);
    filter_line(P.data + (long)yp * P.stride + xp, 1, P.width - xp, xp, plane, size, s, L.bit_depth);
}

// Pass 1: horizontal edges.  x = sample column, y = edge index (plane row 4e).
__global__ void deblock_horizontal_kernel(PassArgs a) {
    const DeblockLaunch& L = a.L;
    const int plane = a.plane_list[blockIdx.z];
    const DevPlane& P = L.pic[plane];
    const int xp = blockIdx.x * blockDim.x + threadIdx.x;
    const int e = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int yp = 4 * e;
    if (xp >= P.width || yp >= P.height) return;
    const int ssx = plane ? L.ssx : 0, ssy = plane ? L.ssy : 0;
    const int col = (xp >> 2) << ssx, row = e << ssy;
    if (col * 4 >= L.coded_width || row * 4 >= L.coded_height) return;
    const uint8_t* map = plane ? L.tx_chroma : L.tx_luma;
    const int map_cols = plane ? (L.mi_cols + L.ssx) >> L.ssx : L.mi_cols;
    const int cur = map[(long)e * map_cols + (xp >> 2)], prev = map[(long)(e - 1) * map_cols + (xp >> 2)];
    const int hl = tx_h_log2(cur);
    if (yp & ((1 << hl) - 1)) return;
    const int base = min(hl, tx_h_log2(prev));
    const int size = min(plane ? 8 : 16, 1 << base);
    const int r = row | ssy, c = col | ssx;
    int lvl = level_at(L, plane, 1, r, c);
    if (lvl == 0) lvl = level_at(L, plane, 1, r - (1 << ssy), c);
    if (lvl == 0) return;
    const Strength s = strength_of(lvl, L.sharpness);
    filter_line(P.data + (long)yp * P.stride + xp, P.stride, P.height - yp, yp, plane, size, s, L.bit_depth);
}

// Copy one plane and flag samples above the bit depth.
__global__ void copy_check_kernel(DevPlaneC s, DevPlane d, int maxv, DeviceStatus* st) {
    int bad = 0;
    const long total = (long)s.width * s.height;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        int y = (int)(i / s.width), x = (int)(i - (long)y * s.width);
        int v = __ldg(s.data + (long)y * s.stride + x);
        bad |= v > maxv;
        d.data[(long)y * d.stride + x] = (uint16_t)v;
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) report_error(st, STAGE_DEBLOCK, 1, VACO_AV1_MSG_DB_SAMPLE);
}

// Row-vectorised variant: 8 samples per thread, 16-byte aligned rows.
__global__ void copy_check_vec_kernel(DevPlaneC s, DevPlane d, int maxv, DeviceStatus* st) {
    int bad = 0;
    const int vpr = s.width / 8;
    const long total = (long)vpr * s.height;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        int y = (int)(i / vpr), v8 = (int)(i - (long)y * vpr);
        uint4 q = __ldg(reinterpret_cast<const uint4*>(s.data + (long)y * s.stride) + v8);
        uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) bad |= ((int)(w[k] & 0xFFFF) > maxv) | ((int)(w[k] >> 16) > maxv);
        reinterpret_cast<uint4*>(d.data + (long)y * d.stride)[v8] = q;
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) report_error(st, STAGE_DEBLOCK, 1, VACO_AV1_MSG_DB_SAMPLE);
}

__global__ void side_check_kernel(const uint8_t* tx_luma, long n_luma, const uint8_t* tx_chroma, long n_chroma,
                                  const uint8_t* lvl_map, DeviceStatus* st) {
    int bad = 0;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n_luma; i += stride) {
        bad |= tx_luma[i] > 18;
        if (lvl_map) {
            uint32_t w = *reinterpret_cast<const uint32_t*>(lvl_map + 4 * i);
            bad |= ((w & 0xFF) > 63) | (((w >> 8) & 0xFF) > 63) | (((w >> 16) & 0xFF) > 63) | ((w >> 24) > 63);
        }
    }
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n_chroma; i += stride) bad |= tx_chroma[i] > 18;
    if (__syncthreads_or(bad) && threadIdx.x == 0) report_error(st, STAGE_DEBLOCK, 0, VACO_AV1_MSG_DB_PARAMS);
}

}  // namespace

cudaError_t launch_deblock_prepare(const DevPlaneC* src, const DevPlane* dst, int num_planes, int bit_depth,
                                   const uint8_t* tx_luma, long n_luma, const uint8_t* tx_chroma, long n_chroma,
                                   const uint8_t* lvl_map, DeviceStatus* status, cudaStream_t stream) {
    const int maxv = (1 << bit_depth) - 1;
    if (n_luma + n_chroma > 0) {
        side_check_kernel<<<148 * 2, 256, 0, stream>>>(tx_luma, n_luma, tx_chroma, n_chroma, lvl_map, status);
    }
    for (int p = 0; p < num_planes; ++p) {
        const DevPlaneC& s = src[p];
        const DevPlane& d = dst[p];
        bool vec = s.width % 8 == 0 && s.stride % 8 == 0 && d.stride % 8 == 0 && ((uintptr_t)s.data % 16) == 0 &&
                   ((uintptr_t)d.data % 16) == 0;
        long units = vec ? (long)(s.width / 8) * s.height : (long)s.width * s.height;
        int blocks = (int)std::min<long>((units + 255) / 256, 148L * 8);
        if (blocks <= 0) continue;
        if (vec)
            copy_check_vec_kernel<<<blocks, 256, 0, stream>>>(s, d, maxv, status);
        else
            copy_check_kernel<<<blocks, 256, 0, stream>>>(s, d, maxv, status);
    }
    return cudaGetLastError();
}

cudaError_t launch_deblock_passes(const DeblockLaunch& L, cudaStream_t stream) {
    if (L.levels[0] == 0 && L.levels[1] == 0) return cudaSuccess;
    PassArgs a;
    a.L = L;
    a.nplanes = 0;
    int max_w = 0, max_h = 0;
    for (int p = 0; p < L.num_planes; ++p) {
        if (p != 0 && L.levels[1 + p] == 0) continue;
        a.plane_list[a.nplanes++] = p;
        max_w = max(max_w, L.pic[p].width);
        max_h = max(max_h, L.pic[p].height);
    }
    if (a.nplanes == 0) return cudaSuccess;
    dim3 blk(32, 8);
    dim3 grid_v(div_up(div_up(max_w, 4), 32), div_up(max_h, 8), a.nplanes);
    deblock_vertical_kernel<<<grid_v, blk, 0, stream>>>(a);
    dim3 grid_h(div_up(max_w, 32), div_up(div_up(max_h, 4), 8), a.nplanes);
    deblock_horizontal_kernel<<<grid_h, blk, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace vaco
