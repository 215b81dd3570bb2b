// cdef.cu -- AV1 CDEF (spec 7.15) on sm_100a.
//
// Mirrors vaco crates/codec/vaco-codec-av1/src/cdef.rs (find_direction :79,
// constrain :126, filter_block :142, adjust_strength :209, chroma_direction
// :224) and the frame pass apply_cdef (src/decode.rs:739-862).
//
// Frame kernel layout: one CTA per 64x64 luma filter block (one cdef_idx
// entry), 256 threads.  The CTA stages the source tile with a 2-row / 8-column
// halo in shared memory (pitch keeps every 8-sample block row 16-byte aligned
// so rows move as uint4).  Samples outside the plane are stored as a sentinel
// that no tap can use: constrain() of a sentinel difference is 0 and the
// maximum masks it out, which is exactly vaco's "unavailable border samples
// are ignored" rule (the availability edges of apply_cdef are the plane
// bounds, decode.rs:828-831).
#include "cdef_core.cuh"
#include "common.cuh"
#include "kernels.cuh"

namespace vaco {

namespace {

using namespace cdefk;

// ---------------------------------------------------------------- frame kernel

constexpr int kThreads = 256;
constexpr int kLumaPitch = 80;   // cols x0-8 .. x0+72
constexpr int kLumaRows = 68;    // rows y0-2 .. y0+66

struct CdefFrameArgs {
    DevPlaneC src[3];
    DevPlane dst[3];
    int num_planes, ssx, ssy, bit_depth, shift, bd_ok;
    int mi_rows, mi_cols;
    const uint8_t* skip;
    const int32_t* cdef_idx;
    int cdef_stride, cdef_count;
    int damping;
    uint8_t y_pri[8], y_sec[8], uv_pri[8], uv_sec[8];
    DeviceStatus* status;
    int vec_ok;  // all plane bases/strides allow 16-byte row vectors
};

// Stage tile rows [y0-2, y0+h+2) x cols [x0-8, x0+w+8) of plane p into smem.
// Returns (via *bad) whether an in-plane sample exceeds the bit depth.
__device__ __forceinline__ void load_tile(uint16_t* sm, int pitch, int rows, const DevPlaneC& p, int x0,
                                          int y0, int limit, bool vec, int* bad) {
    const int vecs_per_row = pitch / 8;
    int local_bad = 0;
    for (int v = threadIdx.x; v < rows * vecs_per_row; v += blockDim.x) {
        int r = v / vecs_per_row, cv = v - r * vecs_per_row;
        int y = y0 - 2 + r, x = x0 - 8 + cv * 8;
        uint16_t* d = sm + r * pitch + cv * 8;
        bool row_in = y >= 0 && y < p.height;
        if (vec && row_in && x >= 0 && x + 8 <= p.width) {
            uint4 q = __ldg(reinterpret_cast<const uint4*>(p.data + (long)y * p.stride + x));
            *reinterpret_cast<uint4*>(d) = q;
            uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int k = 0; k < 4; ++k) local_bad |= ((int)(w[k] & 0xFFFF) > limit) | ((int)(w[k] >> 16) > limit);
        } else {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                int xx = x + k;
                int s = kSent;
                if (row_in && xx >= 0 && xx < p.width) {
                    s = __ldg(p.data + (long)y * p.stride + xx);
                    local_bad |= s > limit;
                }
                d[k] = (uint16_t)s;
            }
        }
    }
    if (local_bad) atomicOr(bad, 1);
}

__global__ void __launch_bounds__(kThreads) cdef_frame_kernel(CdefFrameArgs a) {
    extern __shared__ __align__(16) uint16_t smem[];
    const int cw = 64 >> a.ssx, ch = 64 >> a.ssy;               // chroma tile extent
    const int cpitch = cw + 16, crows = ch + 4;
    uint16_t* tile[3];
    tile[0] = smem;
    tile[1] = smem + kLumaRows * kLumaPitch;
    tile[2] = tile[1] + crows * cpitch;
    __shared__ int s_cost[64][8];
    __shared__ BlockFilter s_filter[3][64];
    __shared__ uint8_t s_active[64];
    __shared__ int s_bad, s_any;

    const int mi_r0 = blockIdx.y * 16, mi_c0 = blockIdx.x * 16;
    const int x0 = mi_c0 * 4, y0 = mi_r0 * 4;
    const int tid = threadIdx.x;

    // Which 8x8 blocks of this 64x64 unit are filtered (decode.rs:772-779).
    long slot = (long)(mi_r0 >> 4) * a.cdef_stride + (mi_c0 >> 4);
    const int index = (slot < a.cdef_count) ? __ldg(a.cdef_idx + slot) : -1;
    if (tid == 0) {
        s_bad = 0;
        s_any = 0;
    }
    __syncthreads();
    if (tid < 64) {
        int r = mi_r0 + (tid >> 3) * 2, c = mi_c0 + (tid & 7) * 2;
        bool act = false;
        if (r < a.mi_rows && c < a.mi_cols && index >= 0) {
            auto sk = [&](int rr, int cc) {
                return rr < a.mi_rows && cc < a.mi_cols && a.skip[(long)rr * a.mi_cols + cc] != 0;
            };
            act = !(sk(r, c) && sk(r + 1, c) && sk(r, c + 1) && sk(r + 1, c + 1));
        }
        s_active[tid] = act;
        if (act) s_any = 1;
    }
    __syncthreads();

    const int limit = a.bd_ok ? (1 << a.bit_depth) - 1 : 0xFFFF;
    const bool vec = a.vec_ok != 0;
    if (s_any) {
        load_tile(tile[0], kLumaPitch, kLumaRows, a.src[0], x0, y0, limit, vec, &s_bad);
        for (int p = 1; p < a.num_planes; ++p)
            load_tile(tile[p], cpitch, crows, a.src[p], x0 >> a.ssx, y0 >> a.ssy, limit, vec, &s_bad);
    }
    __syncthreads();

    if (!s_any) {
        // Nothing filtered: the output is the source (apply_cdef copies first).
        for (int p = 0; p < a.num_planes; ++p) {
            int px0 = p ? x0 >> a.ssx : x0, py0 = p ? y0 >> a.ssy : y0;
            int tw = p ? cw : 64, th = p ? ch : 64;
            const DevPlaneC& s = a.src[p];
            const DevPlane& d = a.dst[p];
            for (int i = tid; i < tw * th; i += kThreads) {
                int yy = py0 + i / tw, xx = px0 + i % tw;
                if (yy < s.height && xx < s.width) d.data[(long)yy * d.stride + xx] = s.data[(long)yy * s.stride + xx];
            }
        }
        return;
    }

    // Direction search: warp w handles direction pair (w & 3) for blocks
    // (w >> 2)*32 + lane, so every branch below is warp-uniform.
    if (a.bd_ok) {
        const int warp = tid >> 5, lane = tid & 31;
        const int pair = warp & 3, b = ((warp >> 2) << 5) + lane;
        if (s_active[b]) {
            const uint16_t* blk = tile[0] + (2 + (b >> 3) * 8) * kLumaPitch + 8 + (b & 7) * 8;
            int lo, hi;
            dir_costs_pair(pair, blk, kLumaPitch, a.shift, lo, hi);
            s_cost[b][pair] = lo;
            s_cost[b][pair + 4] = hi;
        }
    }
    __syncthreads();

    // Per-block parameters (decode.rs:780-841) and vaco's checks.
    if (tid < 64 && s_active[tid]) {
        const int b = tid;
        int dir = 0;
        uint32_t var = 0;
        if (a.bd_ok) best_direction(s_cost[b], dir, var);
        bool param_bad[3] = {false, false, false};
        for (int p = 0; p < a.num_planes; ++p) {
            bool chroma = p != 0;
            int sp = 0, ss = 0;
            if (index < 8) {
                sp = chroma ? a.uv_pri[index] : a.y_pri[index];
                ss = chroma ? a.uv_sec[index] : a.y_sec[index];
            }
            int primary = (sp << a.shift) & 0xFFFF, secondary = (ss << a.shift) & 0xFFFF;
            int chosen = primary == 0 ? 0 : chroma ? chroma_direction(dir, a.ssx, a.ssy) : dir;
            if (!chroma) primary = adjust_strength(primary, var);
            int damping = (a.damping + a.shift - (chroma ? 1 : 0)) & 0xFF;
            param_bad[p] = index >= 8 || damping > 12 || primary > (15 << a.shift) || secondary > (4 << a.shift);
            int pitch = chroma ? cpitch : kLumaPitch;
            s_filter[p][b] = make_filter(chosen, primary, secondary, min(damping, 12), a.shift, pitch);
        }
        if (!a.bd_ok || param_bad[0] || param_bad[1] || param_bad[2]) atomicOr(&s_bad, 2);
    }
    __syncthreads();

    if (s_bad) {
        // Rare path: find the first failing check of each block exactly as
        // vaco's raster walk would meet it, and report the earliest.
        if (tid < 64 && s_active[tid]) {
            const int b = tid, by = b >> 3, bx = b & 7;
            const int r = mi_r0 + by * 2, c = mi_c0 + bx * 2;
            const unsigned long long pos = ((unsigned long long)r * a.mi_cols + c) * 4;
            int msg = 0, stage = 0;
            if (!a.bd_ok) {
                msg = VACO_AV1_MSG_CDEF_BIT_DEPTH;
            } else {
                for (int i = 0; i < 64 && !msg; ++i)
                    if (tile[0][(2 + by * 8 + i / 8) * kLumaPitch + 8 + bx * 8 + i % 8] > limit)
                        msg = VACO_AV1_MSG_CDEF_SAMPLE;
                for (int p = 0; p < a.num_planes && !msg; ++p) {
                    bool chroma = p != 0;
                    int sx = chroma ? a.ssx : 0, sy = chroma ? a.ssy : 0;
                    int bw = 8 >> sx, bh = 8 >> sy, pitch = chroma ? cpitch : kLumaPitch;
                    int lx = bx * bw, ly = by * bh;  // tile-local block origin
                    bool bad = index >= 8;
                    if (bad) {
                        msg = VACO_AV1_MSG_CDEF_STRENGTH_INDEX;
                        stage = 1 + p;
                        break;
                    }
                    int sp = chroma ? a.uv_pri[index] : a.y_pri[index];
                    int ss = chroma ? a.uv_sec[index] : a.y_sec[index];
                    int primary = (sp << a.shift) & 0xFFFF, secondary = (ss << a.shift) & 0xFFFF;
                    if (!chroma) {
                        int dir;
                        uint32_t var;
                        best_direction(s_cost[b], dir, var);
                        primary = adjust_strength(primary, var);
                    }
                    int damping = (a.damping + a.shift - (chroma ? 1 : 0)) & 0xFF;
                    bad = damping > 12 || primary > (15 << a.shift) || secondary > (4 << a.shift);
                    const DevPlaneC& sp_ = a.src[p];
                    int gx0 = (p ? x0 >> a.ssx : x0) + lx, gy0 = (p ? y0 >> a.ssy : y0) + ly;
                    for (int yy = -2; yy < bh + 2 && !bad; ++yy)
                        for (int xx = -2; xx < bw + 2 && !bad; ++xx) {
                            int gx = gx0 + xx, gy = gy0 + yy;
                            if (gx < 0 || gy < 0 || gx >= sp_.width || gy >= sp_.height) continue;
                            bad = tile[p][(2 + ly + yy) * pitch + 8 + lx + xx] > limit;
                        }
                    if (bad) {
                        msg = VACO_AV1_MSG_CDEF_BLOCK_PARAMS;
                        stage = 1 + p;
                    }
                }
            }
            if (msg) report_error(a.status, STAGE_CDEF, pos + stage, msg);
        }
        if (!a.bd_ok) return;
    }

    // Filtering: one lane per column and warps walking contiguous rows, so the
    // taps of a warp read consecutive shared-memory samples (no bank
    // conflicts) and every output row is one coalesced store.  Each lane
    // handles whole block columns: the tap addresses of a block are formed
    // once and the rows inside the block use immediate offsets.
    const int warp = tid >> 5, lane = tid & 31;
    for (int p = 0; p < a.num_planes; ++p) {
        const int sx = p ? a.ssx : 0, sy = p ? a.ssy : 0;
        const int tw = 64 >> sx, th = 64 >> sy;   // tile extent in this plane
        const int bw = 8 >> sx, bh = 8 >> sy;     // block extent
        const int pitch = p ? cpitch : kLumaPitch;
        const DevPlane& d = a.dst[p];
        const int px0 = p ? x0 >> a.ssx : x0, py0 = p ? y0 >> a.ssy : y0;
        const int strips = tw >> 5;               // 32-column strips (2 or 1)
        const int wps = (kThreads / 32) / strips; // warps per strip
        const int rpw = th / wps;                 // rows per warp (a multiple of bh)
        const int c = (warp / wps) * 32 + lane;   // tile column of this lane
        const int gx = px0 + c, bx = c / bw;
        const bool col_in = gx < d.width;
        for (int r0 = (warp % wps) * rpw; r0 < (warp % wps + 1) * rpw; r0 += bh) {
            if (py0 + r0 >= d.height) break;
            const int b = (r0 / bh) * 8 + bx;
            const uint16_t* s = tile[p] + (2 + r0) * pitch + 8 + c;
            uint16_t* o = d.data + (long)(py0 + r0) * d.stride + gx;
            const int rows = min(bh, d.height - (py0 + r0));
            if (s_active[b]) {
                const BlockFilter f = s_filter[p][b];
                if (bh == 8) {
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const int v = filter_px(s + j * pitch, f);
                        if (col_in && j < rows) o[(long)j * d.stride] = (uint16_t)v;
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int v = filter_px(s + j * pitch, f);
                        if (col_in && j < rows) o[(long)j * d.stride] = (uint16_t)v;
                    }
                }
            } else if (col_in) {
                for (int j = 0; j < rows; ++j) o[(long)j * d.stride] = s[j * pitch];
            }
        }
    }
}

// ---------------------------------------------------------------- batch kernels (cdef.rs API)

// find_direction over n blocks: 64 blocks per CTA staged at pitch 8.
__global__ void __launch_bounds__(kThreads) find_direction_kernel(const uint16_t* __restrict__ blocks, int n,
                                                                  int bit_depth, uint8_t* dirs, uint32_t* vars,
                                                                  DeviceStatus* status) {
    __shared__ __align__(16) uint16_t sm[64 * 64];
    __shared__ int s_cost[64][8];
    const int base = blockIdx.x * 64;
    const int tid = threadIdx.x;
    const bool bd_ok = bit_depth == 8 || bit_depth == 10 || bit_depth == 12;
    const int limit = bd_ok ? (1 << bit_depth) - 1 : 0;
    for (int i = tid; i < 64 * 64; i += kThreads) {
        long g = (long)base * 64 + i;
        int v = (g < (long)n * 64) ? blocks[g] : 0;
        sm[i] = (uint16_t)v;
        if (g < (long)n * 64 && (!bd_ok || v > limit))
            report_error(status, 0, (unsigned long long)(g / 64),
                         bd_ok ? VACO_AV1_MSG_CDEF_SAMPLE : VACO_AV1_MSG_CDEF_BIT_DEPTH);
    }
    __syncthreads();
    if (!bd_ok) return;
    const int warp = tid >> 5, lane = tid & 31;
    const int pair = warp & 3, b = ((warp >> 2) << 5) + lane;
    int lo, hi;
    dir_costs_pair(pair, sm + b * 64, 8, bit_depth - 8, lo, hi);
    s_cost[b][pair] = lo;
    s_cost[b][pair + 4] = hi;
    __syncthreads();
    if (tid < 64 && base + tid < n) {
        int d;
        uint32_t v;
        best_direction(s_cost[tid], d, v);
        dirs[base + tid] = (uint8_t)d;
        vars[base + tid] = v;
    }
}

// filter_block over n 12x12 neighborhoods; 64 cases per CTA, 4 threads per case.
__global__ void __launch_bounds__(kThreads) filter_block_kernel(const uint16_t* __restrict__ inputs,
                                                                const vaco_av1_cdef_filter_params* __restrict__ params,
                                                                int n, uint16_t* outputs, DeviceStatus* status) {
    constexpr int P = 16;  // smem pitch per case (12 used)
    __shared__ __align__(16) uint16_t sm[64][12 * P];
    const int base = blockIdx.x * 64;
    const int tid = threadIdx.x;
    // Stage each case with unavailable positions replaced by the sentinel.
    for (int i = tid; i < 64 * 144; i += kThreads) {
        int c = i / 144, k = i - c * 144;
        int id = base + c;
        if (id >= n) continue;
        vaco_av1_cdef_filter_params p = params[id];
        int y = k / 12 - 2, x = k % 12 - 2;
        int x_min = (p.edges & 1) ? -2 : 0, x_max = p.width + ((p.edges & 2) ? 2 : 0);
        int y_min = (p.edges & 4) ? -2 : 0, y_max = p.height + ((p.edges & 8) ? 2 : 0);
        int v = inputs[(long)id * 144 + k];
        bool avail = x >= x_min && x < x_max && y >= y_min && y < y_max;
        sm[c][(y + 2) * P + x + 2] = avail ? (uint16_t)v : (uint16_t)kSent;
        bool bd_ok = p.bit_depth == 8 || p.bit_depth == 10 || p.bit_depth == 12;
        if (!bd_ok) {
            report_error(status, 0, id, VACO_AV1_MSG_CDEF_BIT_DEPTH);
        } else if (v >= (1 << p.bit_depth)) {
            report_error(status, 0, id, VACO_AV1_MSG_CDEF_BLOCK_PARAMS);
        } else if (k == 0) {
            int shift = p.bit_depth - 8;
            bool bad = !(p.width == 4 || p.width == 8) || !(p.height == 4 || p.height == 8) || p.direction > 7 ||
                       p.edges > 15 || p.damping > 12 || p.primary > (15 << shift) || p.secondary > (4 << shift);
            if (bad) report_error(status, 0, id, VACO_AV1_MSG_CDEF_BLOCK_PARAMS);
        }
    }
    __syncthreads();
    const int c = tid >> 2, id = base + c;
    if (id >= n) return;
    vaco_av1_cdef_filter_params p = params[id];
    bool bd_ok = p.bit_depth == 8 || p.bit_depth == 10 || p.bit_depth == 12;
    if (!bd_ok || p.direction > 7 || p.damping > 12) return;
    int shift = p.bit_depth - 8;
    BlockFilter f = make_filter(p.direction, p.primary, p.secondary, p.damping, shift, P);
    for (int row = (tid & 3) * 2; row < (tid & 3) * 2 + 2; ++row)
        for (int x = 0; x < 8; ++x) {
            int v = (row < p.height && x < p.width) ? filter_px(&sm[c][(row + 2) * P + x + 2], f) : 0;
            outputs[(long)id * 64 + row * 8 + x] = (uint16_t)v;
        }
}

}  // namespace

// ---------------------------------------------------------------- launchers

cudaError_t launch_cdef_frame(const CdefLaunch& L, cudaStream_t stream) {
    CdefFrameArgs a;
    const int np = L.info.monochrome ? 1 : 3;
    bool vec = true;
    for (int p = 0; p < 3; ++p) {
        a.src[p] = DevPlaneC{L.src.planes[p], L.src.width[p], L.src.height[p], L.src.stride[p]};
        a.dst[p] = DevPlane{L.dst.planes[p], L.dst.width[p], L.dst.height[p], L.dst.stride[p]};
        if (p < np) {
            vec = vec && (L.src.stride[p] % 8 == 0) && (L.dst.stride[p] % 8 == 0) &&
                  ((uintptr_t)L.src.planes[p] % 16 == 0) && ((uintptr_t)L.dst.planes[p] % 16 == 0);
        }
    }
    a.num_planes = np;
    a.ssx = np > 1 ? L.info.subsampling_x : 0;
    a.ssy = np > 1 ? L.info.subsampling_y : 0;
    a.bit_depth = L.info.bit_depth;
    a.bd_ok = L.info.bit_depth == 8 || L.info.bit_depth == 10 || L.info.bit_depth == 12;
    a.shift = a.bd_ok ? L.info.bit_depth - 8 : 0;
    a.mi_rows = L.info.mi_rows;
    a.mi_cols = L.info.mi_cols;
    a.skip = L.skip;
    a.cdef_idx = L.cdef_idx;
    a.cdef_stride = L.cdef_stride;
    a.cdef_count = L.cdef_count;
    a.damping = L.params.damping;
    for (int k = 0; k < 8; ++k) {
        a.y_pri[k] = L.params.y_primary[k];
        a.y_sec[k] = L.params.y_secondary[k];
        a.uv_pri[k] = L.params.uv_primary[k];
        a.uv_sec[k] = L.params.uv_secondary[k];
    }
    a.status = L.status;
    a.vec_ok = vec;
    dim3 grid(div_up(L.info.mi_cols, 16), div_up(L.info.mi_rows, 16));
    const int cw = 64 >> a.ssx, ch = 64 >> a.ssy;
    size_t smem = sizeof(uint16_t) * (kLumaRows * kLumaPitch + (np > 1 ? 2 * (ch + 4) * (cw + 16) : 0));
    cdef_frame_kernel<<<grid, kThreads, smem, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_find_direction(const uint16_t* blocks, int n, int bit_depth, uint8_t* dirs, uint32_t* vars,
                                  DeviceStatus* status, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    find_direction_kernel<<<div_up(n, 64), kThreads, 0, stream>>>(blocks, n, bit_depth, dirs, vars, status);
    return cudaGetLastError();
}

cudaError_t launch_filter_block(const uint16_t* inputs, const vaco_av1_cdef_filter_params* params, int n,
                                uint16_t* outputs, DeviceStatus* status, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    filter_block_kernel<<<div_up(n, 64), kThreads, 0, stream>>>(inputs, params, n, outputs, status);
    return cudaGetLastError();
}

}  // namespace vaco
