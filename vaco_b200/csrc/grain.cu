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
//         earlier step.  One thread per row, a register window of the rows
//         above, one barrier (of the row-owning warps only) per step.
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

// Round2 of the co-located filtered luma of chroma template position (y, x).
__device__ __forceinline__ int luma_term(const int16_t (*L)[kTW], int y, int x, int sub_x, int sub_y) {
    const int ly = ((y - 3) << sub_y) + 3, lx = ((x - 3) << sub_x) + 3;
    int l = 0;
    for (int i = 0; i <= sub_y; ++i)
        for (int j = 0; j <= sub_x; ++j) l += L[ly + i][lx + j];
    return round2(l, sub_x + sub_y);
}

__device__ __forceinline__ void bar_named(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// One plane's auto-regression (7.18.3.3) in place in shared memory, as a
// wavefront: template row 3 + yy takes column 3 + (t - 4 yy) at step t, so
// every sample it reads was written at an earlier step.  The thread keeps
// its row's last LAG outputs and a LAG x (2 LAG + 1) window of the rows
// above in registers, so a step loads only the window's new column.  The
// taps c[] are in the spec's order (rows above from the farthest, then the
// left neighbours); CHROMA adds the co-located luma times c[2 LAG (LAG + 1)].
// Every thread of the first `nthreads` threads of the CTA calls it (named
// barrier 1); `active` says whether the thread owns a row.
template <int LAG, bool CHROMA>
__device__ __forceinline__ void ar_wavefront(int16_t (*T)[kTW], const int16_t (*L)[kTW], int yy, bool active,
                                             int rows, int cols, const int (&c)[25], bool luma_on, int sub_x,
                                             int sub_y, int ar_shift, int gmin, int gmax, int nthreads) {
    constexpr int NA = 2 * LAG + 1, NL = LAG > 0 ? LAG : 1;
    constexpr int kPosLuma = 2 * LAG * (LAG + 1);
    int win[NL][NA];  // win[d - 1][k] = T[y - d][x - LAG + k]
    int left[NL];     // left[k - 1] = T[y][x - k]
    const int y = 3 + yy;
    const int steps = cols + 4 * (rows - 1);
    for (int t = 0; t < steps; ++t) {
        const int xx = t - 4 * yy;
        if (active && xx >= 0 && xx < cols) {
            const int x = 3 + xx;
            if (xx == 0) {
#pragma unroll
                for (int d = 1; d <= LAG; ++d)
#pragma unroll
                    for (int k = 0; k < NA; ++k) win[d - 1][k] = T[y - d][x - LAG + k];
#pragma unroll
                for (int k = 1; k <= LAG; ++k) left[k - 1] = T[y][x - k];
            } else {
#pragma unroll
                for (int d = 1; d <= LAG; ++d) {
#pragma unroll
                    for (int k = 0; k + 1 < NA; ++k) win[d - 1][k] = win[d - 1][k + 1];
                    win[d - 1][NA - 1] = T[y - d][x + LAG];
                }
            }
            const int cur = T[y][x];
            // one independent partial sum per row above, then the left taps
            int part[NL + 1];
#pragma unroll
            for (int d = LAG; d >= 1; --d) {
                int r = 0;
#pragma unroll
                for (int k = 0; k < NA; ++k) r += c[(LAG - d) * NA + k] * win[d - 1][k];
                part[d - 1] = r;
            }
            int lsum = 0;
#pragma unroll
            for (int k = LAG; k >= 1; --k) lsum += c[LAG * NA + (LAG - k)] * left[k - 1];
            part[NL] = lsum;
            int sum = 0;
#pragma unroll
            for (int d = 0; d <= NL; ++d) sum += (d < LAG || d == NL) ? part[d] : 0;
            if (CHROMA && luma_on) sum += c[kPosLuma] * luma_term(L, y, x, sub_x, sub_y);
            const int v = clampi(cur + round2(sum, ar_shift), gmin, gmax);
            T[y][x] = (int16_t)v;
#pragma unroll
            for (int k = LAG - 1; k >= 1; --k) left[k] = left[k - 1];
            if (LAG > 0) left[0] = v;
        }
        bar_named(1, nthreads);
    }
}

template <int LAG>
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

    // Auto-regression: luma, then both chroma planes together (they read the
    // filtered luma).  Only the warps that own rows take part.
    const int ar_shift = p.ar_coeff_shift_minus_6 + 6;
    constexpr int kPosLuma = 2 * LAG * (LAG + 1);
    {
        int c[25];
#pragma unroll
        for (int i = 0; i < 25; ++i) c[i] = i < kPosLuma ? p.ar_coeffs_y_plus_128[i] - 128 : 0;
        if (LAG == 0) {
            for (int i = tid; i < 70 * 76; i += kGrainThreads) {
                const int y = 3 + i / 76, x = 3 + i % 76;
                s_t[0][y][x] = (int16_t)clampi(s_t[0][y][x], gmin, gmax);  // Round2(0) added
            }
        } else if (tid < 96) {
            ar_wavefront<LAG, false>(s_t[0], s_t[0], tid, tid < 70, 70, 76, c, false, 0, 0, ar_shift, gmin, gmax, 96);
        }
    }
    __syncthreads();
    if (a.np > 1) {
        const int rows = ch - 3, cols = cw - 6;
        const int plane = tid < rows ? 1 : 2, yy = tid - (plane - 1) * rows;
        const bool on = plane == 1 ? cb_on : cr_on;
        const uint8_t* coef = plane == 1 ? p.ar_coeffs_cb_plus_128 : p.ar_coeffs_cr_plus_128;
        int c[25];
#pragma unroll
        for (int i = 0; i < 25; ++i) c[i] = i <= kPosLuma ? coef[i] - 128 : 0;
        const bool luma_on = p.num_y_points > 0;
        if (LAG == 0) {
            for (int i = tid; i < 2 * rows * cols; i += kGrainThreads) {
                const int pl = 1 + i / (rows * cols), j = i % (rows * cols);
                const int y = 3 + j / cols, x = 3 + j % cols;
                if (!(pl == 1 ? cb_on : cr_on)) continue;
                const int cl = (pl == 1 ? p.ar_coeffs_cb_plus_128[0] : p.ar_coeffs_cr_plus_128[0]) - 128;
                const int sum = luma_on ? cl * luma_term(s_t[0], y, x, a.sub_x, a.sub_y) : 0;
                s_t[pl][y][x] = (int16_t)clampi(s_t[pl][y][x] + round2(sum, ar_shift), gmin, gmax);
            }
        } else {
            const int nthreads = (2 * rows + 31) / 32 * 32;
            if (tid < nthreads)
                ar_wavefront<LAG, true>(s_t[plane], s_t[0], yy, tid < 2 * rows && on, rows, cols, c, luma_on,
                                        a.sub_x, a.sub_y, ar_shift, gmin, gmax, nthreads);
        }
    }
    __syncthreads();

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
    unsigned cpr_recip[3];  // fast_div_recip(chunks_per_row)
    long long chunk_base[4];
    const int16_t* templ;
    const uint8_t* offsets;
    DeviceStatus* status;
    int vec;  // every plane's rows start 16-byte aligned: 8-sample runs load and store as one vector
};

// NoiseStripe[s][plane][i][x0 .. x0+7] of 7.18.3.5 (x0 a multiple of 8, so
// the run lies in one block): the block's template window, with the
// horizontal overlap against the block to its left on the block's first
// columns.
__device__ __forceinline__ void stripe_run(const ApplyArgs& a, const int16_t* T, int psx, int psy, int gmin,
                                           int gmax, int s, int i, int x0, int (&g)[8]) {
    const int bw = 32 >> psx, bx = x0 >> (5 - psx), j0 = x0 - bx * bw;
    const int off = __ldg(a.offsets + (long)s * a.nbx + bx);
    const int ox = psx ? 6 + (off >> 4) : 9 + 2 * (off >> 4), oy = psy ? 6 + (off & 15) : 9 + 2 * (off & 15);
    const int16_t* r = T + (oy + i) * kTW + ox + j0;
#pragma unroll
    for (int k = 0; k < 8; ++k) g[k] = __ldg(r + k);
    if (a.p.overlap_flag && bx > 0 && j0 == 0) {
        const int o2 = __ldg(a.offsets + (long)s * a.nbx + bx - 1);
        const int ox2 = psx ? 6 + (o2 >> 4) : 9 + 2 * (o2 >> 4), oy2 = psy ? 6 + (o2 & 15) : 9 + 2 * (o2 & 15);
        const int16_t* r2 = T + (oy2 + i) * kTW + ox2 + bw;
        if (psx) {
            g[0] = clampi(round2(__ldg(r2) * 23 + g[0] * 22, 5), gmin, gmax);
        } else {
            g[0] = clampi(round2(__ldg(r2) * 27 + g[0] * 17, 5), gmin, gmax);
            g[1] = clampi(round2(__ldg(r2 + 1) * 17 + g[1] * 27, 5), gmin, gmax);
        }
    }
}

// NoiseImage[plane][y][x0 .. x0+7]: the stripe's run with the vertical
// overlap against the stripe above on the stripe's first rows.
__device__ __forceinline__ void noise_run(const ApplyArgs& a, int plane, int gmin, int gmax, int y, int x0,
                                          int (&g)[8]) {
    const int psx = plane ? a.sub_x : 0, psy = plane ? a.sub_y : 0;
    const int16_t* T = a.templ + plane * kTSize;
    const int s = y >> (5 - psy), i = y - (s << (5 - psy));
    stripe_run(a, T, psx, psy, gmin, gmax, s, i, x0, g);
    if (a.p.overlap_flag && s > 0 && (psy ? i == 0 : i < 2)) {
        int gp[8];
        stripe_run(a, T, psx, psy, gmin, gmax, s - 1, i + (32 >> psy), x0, gp);
        const int wo = psy ? 23 : i == 0 ? 27 : 17, wn = psy ? 22 : i == 0 ? 17 : 27;
#pragma unroll
        for (int k = 0; k < 8; ++k) g[k] = clampi(round2(gp[k] * wo + g[k] * wn, 5), gmin, gmax);
    }
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
        const unsigned j = (unsigned)(c - a.chunk_base[plane]);  // < 2^31 (checked on the host)
        const int cpr = a.chunks_per_row[plane];
        const int y = (int)fast_div(j, cpr, a.cpr_recip[plane]), x0 = (int)(j - (unsigned)y * cpr) * 8;
        const int n = min(8, a.pw[plane] - x0);
        const uint16_t* src = a.in[plane].data + (long)y * a.in[plane].stride + x0;
        uint16_t* dst = a.out[plane].data + (long)y * a.out[plane].stride + x0;
        const bool full = n == 8 && a.vec;
        int orig[8];
        if (full) {
            const uint4 q = __ldg(reinterpret_cast<const uint4*>(src));
            const uint32_t w4[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int k = 0; k < 4; ++k) orig[2 * k] = w4[k] & 0xFFFF, orig[2 * k + 1] = w4[k] >> 16;
        } else {
#pragma unroll
            for (int k = 0; k < 8; ++k) orig[k] = k < n ? src[k] : 0;
        }
        bool bad = false;
#pragma unroll
        for (int k = 0; k < 8; ++k) bad |= orig[k] > maxv;
        int v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = orig[k];
        const bool on = plane == 0 ? p.num_y_points > 0
                                   : (plane == 1 ? p.num_cb_points : p.num_cr_points) > 0 || p.chroma_scaling_from_luma;
        if (p.apply_grain && on) {
            int g[8];
            noise_run(a, plane, gmin, gmax, y, x0, g);
            int merged[8];
            if (plane) {
                const uint16_t* lrow = a.in[0].data + (long)(y << a.sub_y) * a.in[0].stride;
                const int mult = plane == 1 ? p.cb_mult : p.cr_mult;
                const int lmult = plane == 1 ? p.cb_luma_mult : p.cr_luma_mult;
                const int offset = plane == 1 ? p.cb_offset : p.cr_offset;
                int lv[16];  // co-located luma, two per chroma sample when subsampled
                if (full && a.sub_x && 2 * x0 + 16 <= a.w) {
                    const uint4 q0 = __ldg(reinterpret_cast<const uint4*>(lrow + 2 * x0));
                    const uint4 q1 = __ldg(reinterpret_cast<const uint4*>(lrow + 2 * x0 + 8));
                    const uint32_t w8[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
                    for (int k = 0; k < 8; ++k) lv[2 * k] = w8[k] & 0xFFFF, lv[2 * k + 1] = w8[k] >> 16;
                } else {
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        const int lx = min((x0 + k) << a.sub_x, a.w - 1), lnx = min(lx + 1, a.w - 1);
                        lv[2 * k] = __ldg(lrow + lx);
                        lv[2 * k + 1] = __ldg(lrow + lnx);
                    }
                }
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const int avg = a.sub_x ? round2(lv[2 * k] + lv[2 * k + 1], 1) : lv[2 * k];
                    merged[k] = p.chroma_scaling_from_luma
                                    ? avg
                                    : clampi(((avg * (lmult - 128) + orig[k] * (mult - 128)) >> 6) +
                                                 ((offset - 256) << lshift),
                                             0, maxv);
                }
            } else {
#pragma unroll
                for (int k = 0; k < 8; ++k) merged[k] = orig[k];
            }
            const int hi = plane ? max_chroma : max_luma;
#pragma unroll
            for (int k = 0; k < 8; ++k)
                v[k] = clampi(orig[k] + round2(scale(plane, merged[k]) * g[k], scaling_shift), min_v, hi);
        }
        if (full) {
            *reinterpret_cast<uint4*>(dst) = make_uint4(v[0] | v[1] << 16, v[2] | v[3] << 16, v[4] | v[5] << 16,
                                                        v[6] | v[7] << 16);
        } else {
            for (int k = 0; k < n; ++k) dst[k] = (uint16_t)v[k];
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

cudaError_t launch_grain_template(const vaco_av1_film_grain_params& p, const int16_t* gauss, int np, int bd,
                                  int sub_x, int sub_y, int w, int h, void* workspace, cudaStream_t stream) {
    static thread_local TemplateArgs t;  // 4.6 KB, off the stack; the launch copies it
    t.p = p;
    memcpy(t.gauss, gauss, sizeof t.gauss);
    build_jump(t.jump);
    t.bd = bd, t.sub_x = sub_x, t.sub_y = sub_y, t.np = np;
    t.nstripes = ((h + 1) / 2 + 15) / 16, t.nbx = ((w + 1) / 2 + 15) / 16;
    t.templ = static_cast<int16_t*>(workspace);
    t.offsets = static_cast<uint8_t*>(workspace) + templ_bytes(np);
    switch (p.ar_coeff_lag) {
        case 0: grain_template_kernel<0><<<1, kGrainThreads, 0, stream>>>(t); break;
        case 1: grain_template_kernel<1><<<1, kGrainThreads, 0, stream>>>(t); break;
        case 2: grain_template_kernel<2><<<1, kGrainThreads, 0, stream>>>(t); break;
        default: grain_template_kernel<3><<<1, kGrainThreads, 0, stream>>>(t); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_grain_apply(const vaco_av1_film_grain_params& p, const DevPlaneC* in, const DevPlane* out,
                               int np, int bd, int sub_x, int sub_y, int w, int h, const void* workspace,
                               DeviceStatus* status, int sm_count, cudaStream_t stream) {
    ApplyArgs a;
    memset(&a, 0, sizeof a);
    a.p = p;
    a.bd = bd, a.sub_x = sub_x, a.sub_y = sub_y, a.np = np, a.w = w, a.h = h, a.nbx = ((w + 1) / 2 + 15) / 16;
    a.templ = static_cast<const int16_t*>(workspace);
    a.offsets = static_cast<const uint8_t*>(workspace) + templ_bytes(np);
    a.status = status;
    long long total = 0;
    for (int k = 0; k < np; ++k) {
        a.in[k] = in[k];
        a.out[k] = out[k];
        a.pw[k] = k ? (w + sub_x) >> sub_x : w;
        a.ph[k] = k ? (h + sub_y) >> sub_y : h;
        a.chunks_per_row[k] = (a.pw[k] + 7) / 8;
        a.cpr_recip[k] = fast_div_recip((unsigned)a.chunks_per_row[k]);
        a.chunk_base[k] = total;
        if ((long long)a.chunks_per_row[k] * a.ph[k] >= (1LL << 31)) return cudaErrorInvalidValue;
        total += (long long)a.chunks_per_row[k] * a.ph[k];
    }
    a.chunk_base[np] = total;
    a.vec = 1;
    for (int k = 0; k < np; ++k)
        a.vec = a.vec && (reinterpret_cast<uintptr_t>(in[k].data) | reinterpret_cast<uintptr_t>(out[k].data)) % 16 == 0 &&
                in[k].stride % 8 == 0 && out[k].stride % 8 == 0;
    if (total == 0) return cudaSuccess;
    const long long want = (total + kApplyThreads - 1) / kApplyThreads;
    const int grid = (int)(want < (long long)sm_count * 8 ? want : (long long)sm_count * 8);
    grain_apply_kernel<<<grid, kApplyThreads, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace vaco
