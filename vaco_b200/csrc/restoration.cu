// restoration.cu -- AV1 loop restoration (spec 7.17) on sm_100a.
//
// Mirrors vaco crates/codec/vaco-codec-av1/src/restoration.rs:178-384
// (restore_plane, Source, wiener, box_ab, guided_pass, self_guided).
//
// Tiling: a CTA owns a tile that lies inside exactly one restoration unit and
// one 64-row (luma) stripe: rows are blocks of min(unit, stripe) samples of
// (y + stripe offset) -- unit rows and stripes share the same 8-row offset
// (restoration.rs:124-133, :218-231) -- and columns are blocks of
// min(unit, 64).  The CTA stages Source::get() of its tile plus a 3-sample
// halo (the reach of the 7-tap Wiener filter and of a radius-2 box around a
// radius-1 neighbourhood) in shared memory, so the stripe rule and the frame
// clamps are applied once per staged sample instead of once per tap.
//   Wiener: the reference's 7x7 sum is separable sample-for-sample (the
//           horizontal rounding/clip depends only on the source row), so it
//           runs as a horizontal pass into an int16 buffer then a vertical pass.
//   Self-guided: box sums per neighbour position are computed once per tile
//           position (vaco recomputes them for every pixel that needs them),
//           with a2 from a 256-entry table of ((z << 8) + z/2) / (z + 1).
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"

namespace vaco {

namespace {

constexpr int kLrThreads = 256;
constexpr int kMaxTile = 64;
constexpr int kSPitch = kMaxTile + 8;                 // staged source pitch (>= C + 6)
constexpr int kSRows = kMaxTile + 6;
constexpr int kBoxPitch = kMaxTile + 2;
constexpr int kBoxRows = kMaxTile + 2;

// Sgr_Params (radius, epsilon) per set and pass (restoration.rs:286-303).
__constant__ int8_t c_sgr_r[16][2] = {{2, 1}, {2, 1}, {2, 1}, {2, 1}, {2, 1}, {2, 1}, {2, 1}, {2, 1},
                                      {2, 1}, {2, 1}, {0, 1}, {0, 1}, {0, 1}, {0, 1}, {2, 0}, {2, 0}};
__constant__ uint8_t c_sgr_e[16][2] = {{12, 4},  {15, 6},  {18, 8},  {21, 9},  {24, 10}, {29, 11},
                                       {36, 12}, {45, 13}, {56, 14}, {68, 15}, {0, 5},   {0, 8},
                                       {0, 11},  {0, 14},  {30, 0},  {75, 0}};

struct LrArgs {
    LrPlane p[3];
    int count;
    int bit_depth;
    int tile_w[3], tile_h[3], tiles_x[3], tiles_y[3], off[3], stripe_h[3];
    int tile_base[4];
};

// Shared-memory layout (dynamic):
//   S     kSRows x kSPitch uint16   staged Source::get values
//   then either  H  kSRows x kMaxTile int16   (Wiener horizontal pass)
//   or           A0,B0,A1,B1  kBoxRows x kBoxPitch int32 each (self-guided)
//   a2 table     256 uint16
constexpr size_t kSBytes = sizeof(uint16_t) * kSRows * kSPitch;
constexpr size_t kBoxBytes = sizeof(int32_t) * kBoxRows * kBoxPitch;
constexpr size_t kLrSmem = kSBytes + 4 * kBoxBytes + 256 * sizeof(uint16_t);

__device__ __forceinline__ int round2i(int v, int s) { return s == 0 ? v : (v + (1 << (s - 1))) >> s; }

__global__ void __launch_bounds__(kLrThreads) restoration_kernel(LrArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint16_t* S = reinterpret_cast<uint16_t*>(smem_raw);
    int32_t* A0 = reinterpret_cast<int32_t*>(smem_raw + kSBytes);
    int32_t* B0 = A0 + kBoxRows * kBoxPitch;
    int32_t* A1 = B0 + kBoxRows * kBoxPitch;
    int32_t* B1 = A1 + kBoxRows * kBoxPitch;
    int16_t* H = reinterpret_cast<int16_t*>(A0);
    uint16_t* a2tab = reinterpret_cast<uint16_t*>(smem_raw + kSBytes + 4 * kBoxBytes);

    int pl = 0;
    while (pl + 1 < a.count && (int)blockIdx.x >= a.tile_base[pl + 1]) ++pl;
    const LrPlane& P = a.p[pl];
    const int local = blockIdx.x - a.tile_base[pl];
    const int ty = local / a.tiles_x[pl], tx = local - ty * a.tiles_x[pl];
    const int off = a.off[pl], sh = a.stripe_h[pl];
    const int y_lo = max(ty * a.tile_h[pl] - off, 0);
    const int y_hi = min((ty + 1) * a.tile_h[pl] - off, P.height);
    const int x_lo = tx * a.tile_w[pl];
    const int x_hi = min(x_lo + a.tile_w[pl], P.width);
    if (y_lo >= y_hi || x_lo >= x_hi) return;
    const int R = y_hi - y_lo, Cw = x_hi - x_lo;
    const int tid = threadIdx.x;

    // Unit of this tile (unit_index, restoration.rs:124-133).
    const int urow = min((y_lo + off) / P.unit_size, P.unit_rows - 1);
    const int ucol = min(x_lo / P.unit_size, P.unit_cols - 1);
    const vaco_av1_lr_unit u = P.units[urow * P.unit_cols + ucol];
    const int bd = a.bit_depth, maxv = (1 << bd) - 1;

    if (u.type != VACO_AV1_LR_WIENER && u.type != VACO_AV1_LR_SGRPROJ) {
        for (int i = tid; i < R * Cw; i += kLrThreads) {
            int yy = y_lo + i / Cw, xx = x_lo + i % Cw;
            P.out.data[(long)yy * P.out.stride + xx] = P.after.data[(long)yy * P.after.stride + xx];
        }
        return;
    }

    // Stage Source::get (restoration.rs:233-244) for rows y_lo-3 .. y_hi+2,
    // cols x_lo-3 .. x_hi+2.
    const int stripe = (y_lo + off) / sh;
    const int s_start = stripe * sh - off, s_end = s_start + sh - 1;
    const int srows = R + 6, scols = Cw + 6;
    for (int i = tid; i < srows * scols; i += kLrThreads) {
        int r = i / scols, c = i - r * scols;
        int x = clampi(x_lo - 3 + c, 0, P.width - 1);
        int y = clampi(y_lo - 3 + r, 0, P.height - 1);
        int v;
        if (y < s_start)
            v = __ldg(P.before.data + (long)max(y, s_start - 2) * P.before.stride + x);
        else if (y > s_end)
            v = __ldg(P.before.data + (long)min(y, s_end + 2) * P.before.stride + x);
        else
            v = __ldg(P.after.data + (long)y * P.after.stride + x);
        S[r * kSPitch + c] = (uint16_t)v;
    }
    __syncthreads();

    if (u.type == VACO_AV1_LR_WIENER) {
        // wiener (restoration.rs:264-283), separated.
        const int round_h = bd == 12 ? 5 : 3;
        const int offset = 1 << (bd + 7 - round_h - 1);
        const int limit = (1 << (bd + 1 + 7 - round_h)) - 1;
        int hv[7], vv[7];
        {
            int a0 = u.horizontal[0], b0 = u.horizontal[1], c0 = u.horizontal[2];
            hv[0] = hv[6] = a0; hv[1] = hv[5] = b0; hv[2] = hv[4] = c0; hv[3] = 128 - 2 * (a0 + b0 + c0);
            int a1 = u.vertical[0], b1 = u.vertical[1], c1 = u.vertical[2];
            vv[0] = vv[6] = a1; vv[1] = vv[5] = b1; vv[2] = vv[4] = c1; vv[3] = 128 - 2 * (a1 + b1 + c1);
        }
        for (int i = tid; i < srows * Cw; i += kLrThreads) {
            int r = i / Cw, c = i - r * Cw;
            const uint16_t* s = S + r * kSPitch + c;
            int h = 0;
#pragma unroll
            for (int t = 0; t < 7; ++t) h += hv[t] * s[t];
            H[r * kMaxTile + c] = (int16_t)clampi(round2i(h, round_h), -offset, limit - offset);
        }
        __syncthreads();
        for (int i = tid; i < R * Cw; i += kLrThreads) {
            int k = i / Cw, c = i - k * Cw;
            int sum = 0;
#pragma unroll
            for (int t = 0; t < 7; ++t) sum += vv[t] * H[(k + t) * kMaxTile + c];
            int v = clampi(round2i(sum, 14 - round_h), 0, maxv);
            P.out.data[(long)(y_lo + k) * P.out.stride + x_lo + c] = (uint16_t)v;
        }
        return;
    }

    // ---- self-guided (restoration.rs:314-384)
    const int set = min(max((int)u.set, 0), 15);
    const int r0 = c_sgr_r[set][0], r1 = c_sgr_r[set][1];
    const int e0 = c_sgr_e[set][0], e1 = c_sgr_e[set][1];
    for (int z = tid; z < 256; z += kLrThreads)
        a2tab[z] = (uint16_t)(z >= 255 ? 256 : z == 0 ? 1 : ((z << 8) + z / 2) / (z + 1));
    const int brow = R + 2, bcol = Cw + 2;  // box positions: y_lo-1.., x_lo-1..
    for (int pass = 0; pass < 2; ++pass) {
        const int rad = pass ? r1 : r0;
        if (rad == 0) continue;
        const int eps = pass ? e1 : e0;
        const int n = (2 * rad + 1) * (2 * rad + 1);
        const int n2e = n * n * eps;
        const unsigned scale = (unsigned)(((1 << 20) + n2e / 2) / n2e);
        const unsigned recip = (unsigned)(((1 << 12) + n / 2) / n);
        int32_t* Ab = pass ? A1 : A0;
        int32_t* Bb = pass ? B1 : B0;
        __syncthreads();  // a2tab ready
        for (int i = tid; i < brow * bcol; i += kLrThreads) {
            int br = i / bcol, bc = i - br * bcol;
            int y = y_lo - 1 + br;
            if (pass == 0 && (y & 1) == 0) continue;  // first pass reads odd rows only
            int sum = 0, sum_sq = 0;
            const uint16_t* s = S + (br + 2 - rad) * kSPitch + (bc + 2 - rad);
            for (int dy = 0; dy <= 2 * rad; ++dy)
                for (int dx = 0; dx <= 2 * rad; ++dx) {
                    int v = s[dy * kSPitch + dx];
                    sum += v;
                    sum_sq += v * v;
                }
            int aa = round2i(sum_sq, 2 * (bd - 8));
            int d = round2i(sum, bd - 8);
            int p = max(aa * n - d * d, 0);
            unsigned long long zz = ((unsigned long long)(unsigned)p * scale + (1u << 19)) >> 20;
            int z = zz > 255 ? 255 : (int)zz;
            int a2 = a2tab[z];
            unsigned b = ((unsigned)(256 - a2) * (unsigned)sum * recip + (1u << 11)) >> 12;
            Ab[br * kBoxPitch + bc] = a2;
            Bb[br * kBoxPitch + bc] = (int)b;
        }
    }
    __syncthreads();
    const int w0 = u.xqd[0], w1 = u.xqd[1];
    for (int i = tid; i < R * Cw; i += kLrThreads) {
        int k = i / Cw, c = i - k * Cw;
        int y = y_lo + k;
        int orig = S[(k + 3) * kSPitch + c + 3];
        const int bi = (k + 1) * kBoxPitch + (c + 1);  // box index of (x, y)
        int first, second;
        if (r0 == 0) {
            first = orig << 4;
        } else if (y & 1) {
            int aa = 6 * A0[bi] + 5 * (A0[bi - 1] + A0[bi + 1]);
            int bb = 6 * B0[bi] + 5 * (B0[bi - 1] + B0[bi + 1]);
            first = round2i(aa * orig + bb, 8);
        } else {
            int up = bi - kBoxPitch, dn = bi + kBoxPitch;
            int aa = 6 * (A0[up] + A0[dn]) + 5 * (A0[up - 1] + A0[up + 1] + A0[dn - 1] + A0[dn + 1]);
            int bb = 6 * (B0[up] + B0[dn]) + 5 * (B0[up - 1] + B0[up + 1] + B0[dn - 1] + B0[dn + 1]);
            first = round2i(aa * orig + bb, 9);
        }
        if (r1 == 0) {
            second = orig << 4;
        } else {
            int up = bi - kBoxPitch, dn = bi + kBoxPitch;
            int aa = 4 * (A1[bi] + A1[bi - 1] + A1[bi + 1] + A1[up] + A1[dn]) +
                     3 * (A1[up - 1] + A1[up + 1] + A1[dn - 1] + A1[dn + 1]);
            int bb = 4 * (B1[bi] + B1[bi - 1] + B1[bi + 1] + B1[up] + B1[dn]) +
                     3 * (B1[up - 1] + B1[up + 1] + B1[dn - 1] + B1[dn + 1]);
            second = round2i(aa * orig + bb, 9);
        }
        int v = round2i(w0 * first + w1 * (orig << 4) + (128 - w0 - w1) * second, 11);
        P.out.data[(long)y * P.out.stride + x_lo + c] = (uint16_t)clampi(v, 0, maxv);
    }
}

__global__ void lr_unit_check_kernel(const vaco_av1_lr_unit* units, int n, DeviceStatus* st) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    vaco_av1_lr_unit u = units[i];
    bool ok;
    if (u.type == VACO_AV1_LR_NONE) {
        ok = true;
    } else if (u.type == VACO_AV1_LR_WIENER) {
        const int lo[3] = {-5, -23, -17}, hi[3] = {10, 8, 46};
        ok = true;
        for (int k = 0; k < 3; ++k)
            ok = ok && u.vertical[k] >= lo[k] && u.vertical[k] <= hi[k] && u.horizontal[k] >= lo[k] &&
                 u.horizontal[k] <= hi[k];
    } else if (u.type == VACO_AV1_LR_SGRPROJ) {
        ok = u.set >= 0 && u.set < 16 && u.xqd[0] >= -96 && u.xqd[0] <= 31 && u.xqd[1] >= -32 && u.xqd[1] <= 95;
    } else {
        ok = false;
    }
    if (!ok) report_error(st, STAGE_LR, (unsigned long long)i, VACO_AV1_MSG_LR_COEFFICIENT);
}

__global__ void range_check_kernel(DevPlaneC p, int w, int h, int maxv, DeviceStatus* st, unsigned stage,
                                   unsigned long long position, unsigned msg) {
    int bad = 0;
    long total = (long)w * h;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        int y = (int)(i / w), x = (int)(i - (long)y * w);
        bad |= __ldg(p.data + (long)y * p.stride + x) > maxv;
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) report_error(st, stage, position, msg);
}

}  // namespace

cudaError_t launch_restoration(const LrPlane* planes, int count, int bit_depth, cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    LrArgs a;
    a.count = count;
    a.bit_depth = bit_depth;
    int total = 0;
    for (int k = 0; k < count; ++k) {
        a.p[k] = planes[k];
        const int sh = 64 >> planes[k].sub_y, off = 8 >> planes[k].sub_y;
        a.stripe_h[k] = sh;
        a.off[k] = off;
        a.tile_h[k] = min(planes[k].unit_size, sh);
        a.tile_w[k] = min(planes[k].unit_size, kMaxTile);
        a.tiles_y[k] = div_up(planes[k].height + off, a.tile_h[k]);
        a.tiles_x[k] = div_up(planes[k].width, a.tile_w[k]);
        a.tile_base[k] = total;
        total += a.tiles_x[k] * a.tiles_y[k];
    }
    a.tile_base[count] = total;
    for (int k = count + 1; k < 4; ++k) a.tile_base[k] = total;
    // The opt-in above 48 KB of dynamic shared memory is a per-device attribute.
    static unsigned long long attr_devices = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !(attr_devices & (1ull << dev))) {
        cudaError_t e = cudaFuncSetAttribute(restoration_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kLrSmem);
        if (e != cudaSuccess) return e;
        attr_devices |= 1ull << dev;
    }
    restoration_kernel<<<total, kLrThreads, kLrSmem, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_lr_unit_check(const vaco_av1_lr_unit* units, int n, DeviceStatus* status, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    lr_unit_check_kernel<<<div_up(n, 128), 128, 0, stream>>>(units, n, status);
    return cudaGetLastError();
}

cudaError_t launch_range_check(const DevPlaneC& p, int w, int h, int max_value, DeviceStatus* status,
                               unsigned stage, unsigned long long position, unsigned msg, cudaStream_t stream) {
    if (w <= 0 || h <= 0) return cudaSuccess;
    long total = (long)w * h;
    int blocks = (int)std::min<long>((std::min<long>(total, 1L << 30) + 2047) / 2048, 148L * 16);
    range_check_kernel<<<max(blocks, 1), 256, 0, stream>>>(p, w, h, max_value, status, stage, position, msg);
    return cudaGetLastError();
}

}  // namespace vaco
