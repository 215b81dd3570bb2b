// grain.cu -- AV1 film grain synthesis (spec 7.18.3) on sm_100a.
//
// vaco parses film_grain_params() (crates/codec/vaco-codec-av1/src/
// frame_header.rs:1125-1210) and stops there: grain synthesis is the next
// step after the post-filters.  This file adds it as two kernels.
//
//   grain_template_kernel  one CTA per frame: the per-stripe random block
//       offsets, the three grain templates (82 x 73 luma, up to 82 x 73 per
//       chroma plane) from the caller's Gaussian table, and their
//       auto-regressive filtering, written to a small workspace.
//       - The templates' random indices come from the spec's 16-bit LFSR.
//         Each thread takes 32 consecutive samples and starts from the
//         register value 32 c steps in, which it computes from the seed by
//         GF(2) matrix products with M^(32 * 2^b) (M = one LFSR step; the
//         host builds those eight matrices), so the sequence needs no
//         serial walk.
//       - The AR filter reads up to 3 rows above (columns x-3 .. x+3) and up
//         to 3 samples to the left, so position (y, x) can run at step
//         (x - 3) + 4 (y - 3): every sample it reads was written at an
//         earlier step.  One thread per row, one barrier per step.
//   grain_apply_kernel  the noise of every output sample straight from the
//       templates: the block's offsets pick the template window, the left
//       block's window gives the horizontal overlap and the stripe above
//       the vertical one (the spec's NoiseStripe / NoiseImage values), then
//       the scaling lookup (built per CTA in shared memory), the chroma
//       merge with the co-located luma and the clip.
//
// Samples above the bit depth would index past the scaling table; they are
// reported (VACO_AV1_MSG_FG_SAMPLE) and the index is clamped.
#include <cstring>

#include "common.cuh"
#include "kernels.cuh"

namespace vaco {

namespace {

constexpr int kTW = 82, kTH = 73;     // template width / height (luma; chroma uses a corner)
constexpr int kTSize = kTW * kTH;     // samples per plane template in the workspace
constexpr int kGrainThreads = 256;
constexpr int kApplyThreads = 256;

constexpr size_t templ_bytes(int np) { return (sizeof(int16_t) * kTSize * np + 255) / 256 * 256; }

struct TemplateArgs {
    vaco_av1_film_grain_params p;
    int16_t gauss[2048];
    uint16_t jump[8][16];  // columns of M^(32 * 2^b)
    int bd, sub_x, sub_y, np;
    int nstripes, nbx;
    int16_t* templ;        // np x kTSize, row pitch kTW
    uint8_t* offsets;      // nstripes x nbx
};

__device__ __forceinline__ int round2(int x, int n) { return n == 0 ? x : (x + (1 << (n - 1))) >> n; }

// One LFSR step of get_random_number (7.18.3.2).
__device__ __forceinline__ unsigned lfsr_step(unsigned r) {
    const unsigned bit = (r ^ (r >> 1) ^ (r >> 3) ^ (r >> 12)) & 1u;
    return (r >> 1) | (bit << 15);
}

__device__ __forceinline__ unsigned gf2_apply(const uint16_t* col, unsigned v) {
    unsigned r = 0;
#pragma unroll
    for (int i = 0; i < 16; ++i) r ^= ((v >> i) & 1u) ? col[i] : 0u;
    return r;
}

__global__ void __launch_bounds__(kGrainThreads) grain_template_kernel(const __grid_constant__ TemplateArgs a) {
    __shared__ int16_t s_gauss[2048];
    __shared__ int16_t s_t[3][kTH][kTW];
    const int tid = threadIdx.x;
    const vaco_av1_film_grain_params& p = a.p;
    const int center = 128 << (a.bd - 8);
    const int gmin = -center, gmax = (256 << (a.bd - 8)) - 1 - center;
    for (int i = tid; i < 2048; i += kGrainThreads) s_gauss[i] = a.gauss[i];

    // Random block offsets of every stripe (7.18.3.5): the register is
    // re-seeded per stripe and steps once per 32-column block.
    for (int s = tid; s < a.nstripes; s += kGrainThreads) {
        unsigned r = p.grain_seed;
        r ^= ((unsigned)((s * 37 + 178) & 255)) << 8;
        r ^= (unsigned)((s * 173 + 105) & 255);
        uint8_t* o = a.offsets + (long)s * a.nbx;
        for (int bx = 0; bx < a.nbx; ++bx) {
            r = lfsr_step(r);
            o[bx] = (uint8_t)((r >> 8) & 255);
        }
    }
    __syncthreads();

    // Templates before filtering (7.18.3.3): Round2(Gaussian_Sequence[rand11], shift).
    const int shift = 12 - a.bd + p.grain_scale_shift;
    const int cw = a.sub_x ? 44 : 82, ch = a.sub_y ? 38 : 73;
    const bool cb_on = p.num_cb_points || p.chroma_scaling_from_luma;
    const bool cr_on = p.num_cr_points || p.chroma_scaling_from_luma;
    for (int plane = 0; plane < a.np; ++plane) {
        const int width = plane ? cw : kTW, n = plane ? cw * ch : kTSize;
        const bool on = plane == 0 ? p.num_y_points > 0 : plane == 1 ? cb_on : cr_on;
        const unsigned seed = plane == 0 ? p.grain_seed : p.grain_seed ^ (plane == 1 ? 0xb524u : 0x49d8u);
        for (int c = tid; c < (n + 31) / 32; c += kGrainThreads) {
            unsigned r = seed;
            for (int b = 0; b < 8; ++b)
                if ((c >> b) & 1) r = gf2_apply(a.jump[b], r);
            for (int k = 0; k < 32; ++k) {
                const int idx = c * 32 + k;
                if (idx >= n) break;
                r = lfsr_step(r);
                const int g = on ? s_gauss[(r >> 5) & 2047] : 0;
                const int y = idx / width;
                s_t[plane][y][idx - y * width] = (int16_t)round2(g, shift);
            }
        }
    }
    __syncthreads();

    // Luma auto-regression, wavefront: row 3 + yy takes column 3 + t - 4 yy at step t.
    const int lag = p.ar_coeff_lag, ar_shift = p.ar_coeff_shift_minus_6 + 6;
    for (int t = 0; t < 76 + 4 * 69; ++t) {
        const int yy = tid, xx = t - 4 * yy;
        if (yy < 70 && xx >= 0 && xx < 76) {
            const int y = 3 + yy, x = 3 + xx;
            int sum = 0, pos = 0;
            for (int dr = -lag; dr <= 0; ++dr)
                for (int dc = -lag; dc <= lag; ++dc) {
                    if (dr == 0 && dc == 0) break;
                    sum += s_t[0][y + dr][x + dc] * (p.ar_coeffs_y_plus_128[pos] - 128);
                    ++pos;
                }
            s_t[0][y][x] = (int16_t)clampi(s_t[0][y][x] + round2(sum, ar_shift), gmin, gmax);
        }
        __syncthreads();
    }

    // Chroma auto-regression, both planes at once, with the co-located luma.
    if (a.np > 1) {
        const int rows = ch - 3, cols = cw - 6;
        for (int t = 0; t < cols + 4 * (rows - 1); ++t) {
            const int plane = 1 + (tid >= rows), yy = tid - (plane - 1) * rows, xx = t - 4 * yy;
            if (tid < 2 * rows && xx >= 0 && xx < cols && (plane == 1 ? cb_on : cr_on)) {
                const int y = 3 + yy, x = 3 + xx;
                const uint8_t* coef = plane == 1 ? p.ar_coeffs_cb_plus_128 : p.ar_coeffs_cr_plus_128;
                int sum = 0, pos = 0;
                for (int dr = -lag; dr <= 0; ++dr)
                    for (int dc = -lag; dc <= lag; ++dc) {
                        const int c = coef[pos] - 128;
                        if (dr == 0 && dc == 0) {
                            if (p.num_y_points > 0) {
                                const int ly = ((y - 3) << a.sub_y) + 3, lx = ((x - 3) << a.sub_x) + 3;
                                int l = 0;
                                for (int i = 0; i <= a.sub_y; ++i)
                                    for (int j = 0; j <= a.sub_x; ++j) l += s_t[0][ly + i][lx + j];
                                sum += round2(l, a.sub_x + a.sub_y) * c;
                            }
                            break;
                        }
                        sum += c * s_t[plane][y + dr][x + dc];
                        ++pos;
                    }
                s_t[plane][y][x] = (int16_t)clampi(s_t[plane][y][x] + round2(sum, ar_shift), gmin, gmax);
            }
            __syncthreads();
        }
    }

    for (int i = tid; i < a.np * kTSize; i += kGrainThreads) {
        const int plane = i / kTSize, j = i - plane * kTSize, y = j / kTW;
        a.templ[i] = s_t[plane][y][j - y * kTW];
    }
}

struct ApplyArgs {
    vaco_av1_film_grain_params p;
    DevPlaneC in[3];
    DevPlane out[3];
    int bd, sub_x, sub_y, np, w, h, nbx;
    int pw[3], ph[3];
    int chunks_per_row[3];
    long long chunk_base[4];
    const int16_t* templ;
    const uint8_t* offsets;
    DeviceStatus* status;
};

// NoiseStripe[s][plane][i][x] of 7.18.3.5: the block's template window, with
// the horizontal overlap against the block to its left.
__device__ __forceinline__ int stripe_value(const ApplyArgs& a, const int16_t* T, int psx, int psy, int gmin,
                                            int gmax, int s, int i, int x) {
    const int bw = 32 >> psx, bx = x >> (5 - psx), j = x - bx * bw;
    const int off = __ldg(a.offsets + (long)s * a.nbx + bx);
    const int ox = psx ? 6 + (off >> 4) : 9 + 2 * (off >> 4), oy = psy ? 6 + (off & 15) : 9 + 2 * (off & 15);
    int g = __ldg(T + (oy + i) * kTW + ox + j);
    if (a.p.overlap_flag && bx > 0 && (psx ? j == 0 : j < 2)) {
        const int o2 = __ldg(a.offsets + (long)s * a.nbx + bx - 1);
        const int ox2 = psx ? 6 + (o2 >> 4) : 9 + 2 * (o2 >> 4), oy2 = psy ? 6 + (o2 & 15) : 9 + 2 * (o2 & 15);
        const int old = __ldg(T + (oy2 + i) * kTW + ox2 + j + bw);
        g = psx ? old * 23 + g * 22 : (j == 0 ? old * 27 + g * 17 : old * 17 + g * 27);
        g = clampi(round2(g, 5), gmin, gmax);
    }
    return g;
}

// NoiseImage[plane][y][x]: the stripe value with the vertical overlap.
__device__ __forceinline__ int noise_at(const ApplyArgs& a, int plane, int gmin, int gmax, int y, int x) {
    const int psx = plane ? a.sub_x : 0, psy = plane ? a.sub_y : 0;
    const int16_t* T = a.templ + plane * kTSize;
    const int s = y >> (5 - psy), i = y - (s << (5 - psy));
    int g = stripe_value(a, T, psx, psy, gmin, gmax, s, i, x);
    if (a.p.overlap_flag && s > 0 && (psy ? i == 0 : i < 2)) {
        const int old = stripe_value(a, T, psx, psy, gmin, gmax, s - 1, i + (32 >> psy), x);
        g = psy ? old * 23 + g * 22 : (i == 0 ? old * 27 + g * 17 : old * 17 + g * 27);
        g = clampi(round2(g, 5), gmin, gmax);
    }
    return g;
}

// ScalingLut entry x of a plane (7.18.3.4) from its points.
__device__ int lut_entry(const uint8_t* v, const uint8_t* sc, int n, int x) {
    if (n == 0) return 0;
    if (x < v[0]) return sc[0];
    if (x >= v[n - 1]) return sc[n - 1];
    int i = 0;
    while (x >= v[i + 1]) ++i;
    const int dy = sc[i + 1] - sc[i], dx = v[i + 1] - v[i];
    const int delta = dy * ((65536 + (dx >> 1)) / dx);
    return sc[i] + (((x - v[i]) * delta + 32768) >> 16);
}

__global__ void __launch_bounds__(kApplyThreads) grain_apply_kernel(const __grid_constant__ ApplyArgs a) {
    __shared__ int16_t s_lut[3][256];
    const vaco_av1_film_grain_params& p = a.p;
    for (int i = threadIdx.x; i < a.np * 256; i += kApplyThreads) {
        const int plane = i >> 8, x = i & 255;
        int v;
        if (plane == 0 || p.chroma_scaling_from_luma) v = lut_entry(p.point_y_value, p.point_y_scaling, p.num_y_points, x);
        else if (plane == 1) v = lut_entry(p.point_cb_value, p.point_cb_scaling, p.num_cb_points, x);
        else v = lut_entry(p.point_cr_value, p.point_cr_scaling, p.num_cr_points, x);
        s_lut[plane][x] = (int16_t)v;
    }
    __syncthreads();
    const int bd = a.bd, maxv = (1 << bd) - 1, lshift = bd - 8;
    const int center = 128 << lshift, gmin = -center, gmax = (256 << lshift) - 1 - center;
    int min_v = 0, max_luma = (256 << lshift) - 1, max_chroma = max_luma;
    if (p.clip_to_restricted_range) {
        min_v = 16 << lshift;
        max_luma = 235 << lshift;
        max_chroma = p.mc_identity ? max_luma : 240 << lshift;
    }
    const int scaling_shift = p.grain_scaling_minus_8 + 8;
    auto scale = [&](int plane, int index) {
        int x = index >> lshift;
        x = x > 255 ? 255 : x;  // only reached for a sample above the bit depth, which is reported
        const int rem = index - (x << lshift);
        if (bd == 8 || x == 255) return (int)s_lut[plane][x];
        const int start = s_lut[plane][x], end = s_lut[plane][x + 1];
        return start + round2((end - start) * rem, lshift);
    };
    const long long total = a.chunk_base[a.np];
    for (long long c = (long long)blockIdx.x * kApplyThreads + threadIdx.x; c < total;
         c += (long long)gridDim.x * kApplyThreads) {
        int plane = 0;
        while (plane + 1 < a.np && c >= a.chunk_base[plane + 1]) ++plane;
        const long long j = c - a.chunk_base[plane];
        const int cpr = a.chunks_per_row[plane];
        const int y = (int)(j / cpr), x0 = (int)(j - (long long)y * cpr) * 8;
        const int n = min(8, a.pw[plane] - x0);
        const uint16_t* src = a.in[plane].data + (long)y * a.in[plane].stride;
        uint16_t* dst = a.out[plane].data + (long)y * a.out[plane].stride;
        bool bad = false;
        const bool on = plane == 0 ? p.num_y_points > 0
                                   : (plane == 1 ? p.num_cb_points : p.num_cr_points) > 0 || p.chroma_scaling_from_luma;
        for (int k = 0; k < n; ++k) {
            const int x = x0 + k, orig = src[x];
            bad |= orig > maxv;
            int v = orig;
            if (p.apply_grain && on) {
                int merged = orig;
                if (plane) {
                    const uint16_t* lrow = a.in[0].data + (long)(y << a.sub_y) * a.in[0].stride;
                    const int lx = x << a.sub_x, lnx = min(lx + 1, a.w - 1);
                    const int avg = a.sub_x ? round2(lrow[lx] + lrow[lnx], 1) : lrow[lx];
                    if (p.chroma_scaling_from_luma) {
                        merged = avg;
                    } else {
                        const int mult = plane == 1 ? p.cb_mult : p.cr_mult;
                        const int lmult = plane == 1 ? p.cb_luma_mult : p.cr_luma_mult;
                        const int offset = plane == 1 ? p.cb_offset : p.cr_offset;
                        const int combined = avg * (lmult - 128) + orig * (mult - 128);
                        merged = clampi((combined >> 6) + ((offset - 256) << lshift), 0, maxv);
                    }
                }
                const int noise = round2(scale(plane, merged) * noise_at(a, plane, gmin, gmax, y, x), scaling_shift);
                v = clampi(orig + noise, min_v, plane ? max_chroma : max_luma);
            }
            dst[x] = (uint16_t)v;
        }
        if (bad)
            report_error(a.status, STAGE_GRAIN, ((unsigned long long)plane << 44) | ((unsigned long long)y << 20) | x0,
                         VACO_AV1_MSG_FG_SAMPLE);
    }
}

// Columns of M^(32 * 2^b), M = one LFSR step, for b = 0..7.
void build_jump(uint16_t (&jump)[8][16]) {
    auto step = [](unsigned r) {
        const unsigned bit = (r ^ (r >> 1) ^ (r >> 3) ^ (r >> 12)) & 1u;
        return (r >> 1) | (bit << 15);
    };
    auto apply = [](const uint16_t* col, unsigned v) {
        unsigned r = 0;
        for (int i = 0; i < 16; ++i)
            if ((v >> i) & 1u) r ^= col[i];
        return r;
    };
    for (int i = 0; i < 16; ++i) {
        unsigned r = 1u << i;
        for (int k = 0; k < 32; ++k) r = step(r);
        jump[0][i] = (uint16_t)r;
    }
    for (int b = 1; b < 8; ++b)
        for (int i = 0; i < 16; ++i) jump[b][i] = (uint16_t)apply(jump[b - 1], apply(jump[b - 1], 1u << i));
}

}  // namespace

size_t film_grain_workspace_bytes(int np, int w, int h) {
    const size_t nstripes = (size_t)(((h + 1) / 2 + 15) / 16), nbx = (size_t)(((w + 1) / 2 + 15) / 16);
    return templ_bytes(np) + nstripes * nbx;
}

cudaError_t launch_film_grain(const vaco_av1_film_grain_params& p, const int16_t* gauss, const DevPlaneC* in,
                              const DevPlane* out, int np, int bd, int sub_x, int sub_y, int w, int h,
                              void* workspace, DeviceStatus* status, int sm_count, cudaStream_t stream) {
    const int nstripes = ((h + 1) / 2 + 15) / 16, nbx = ((w + 1) / 2 + 15) / 16;
    int16_t* templ = static_cast<int16_t*>(workspace);
    uint8_t* offsets = static_cast<uint8_t*>(workspace) + templ_bytes(np);
    if (p.apply_grain) {
        static thread_local TemplateArgs t;  // 4.6 KB, off the stack; the launch copies it
        t.p = p;
        memcpy(t.gauss, gauss, sizeof t.gauss);
        build_jump(t.jump);
        t.bd = bd, t.sub_x = sub_x, t.sub_y = sub_y, t.np = np;
        t.nstripes = nstripes, t.nbx = nbx;
        t.templ = templ, t.offsets = offsets;
        grain_template_kernel<<<1, kGrainThreads, 0, stream>>>(t);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    ApplyArgs a;
    memset(&a, 0, sizeof a);
    a.p = p;
    a.bd = bd, a.sub_x = sub_x, a.sub_y = sub_y, a.np = np, a.w = w, a.h = h, a.nbx = nbx;
    a.templ = templ, a.offsets = offsets, a.status = status;
    long long total = 0;
    for (int k = 0; k < np; ++k) {
        a.in[k] = in[k];
        a.out[k] = out[k];
        a.pw[k] = k ? (w + sub_x) >> sub_x : w;
        a.ph[k] = k ? (h + sub_y) >> sub_y : h;
        a.chunks_per_row[k] = (a.pw[k] + 7) / 8;
        a.chunk_base[k] = total;
        total += (long long)a.chunks_per_row[k] * a.ph[k];
    }
    a.chunk_base[np] = total;
    if (total == 0) return cudaSuccess;
    const long long want = (total + kApplyThreads - 1) / kApplyThreads;
    const int grid = (int)(want < (long long)sm_count * 8 ? want : (long long)sm_count * 8);
    grain_apply_kernel<<<grid, kApplyThreads, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace vaco
