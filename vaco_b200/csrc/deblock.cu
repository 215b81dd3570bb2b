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
#include "deblock_core.cuh"
#include "kernels.cuh"

namespace vaco {

namespace {

using namespace dbk;

struct PassArgs {
    DeblockLaunch L;
    int plane_list[3];
    int nplanes;
};

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
