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
// clamps are applied once per staged sample instead of once per tap.  Rows
// are staged as aligned 16-byte vectors covering columns x0-8 .. x0+72.
//   Wiener: the reference's 7x7 sum is separable sample-for-sample (the
//           horizontal rounding/clip depends only on the source row), so it
//           runs as a horizontal pass into an int16 buffer then a vertical pass.
//   Self-guided: box sums per neighbour position are computed once per tile
//           position (vaco recomputes them for every pixel that needs them),
//           radius-specialised and unrolled, with a2 from a 256-entry table of
//           ((z << 8) + z/2) / (z + 1).  The two passes run one after the
//           other in the same shared buffers; each thread keeps its pixels'
//           first-pass values in registers.
// Thread mappings put consecutive lanes on consecutive columns, so shared
// memory reads are conflict-free and global writes coalesce.
#include <algorithm>
#include <atomic>
#include <cstring>

#include "common.cuh"
#include "kernels.cuh"

namespace vaco {

namespace {

constexpr int kLrThreads = 256;
constexpr int kWarps = kLrThreads / 32;
constexpr int kMaxTile = 64;
constexpr int kSPitch = kMaxTile + 16;  // staged columns x0-8 .. x0+72
constexpr int kSRows = kMaxTile + 6;    // staged rows y0-3 .. y0+67
constexpr int kSOff = 8;                // staged column of x0
constexpr int kBox = kMaxTile + 2;      // box positions y0-1 .. y0+64 (and x)

// Sgr_Params (radius, epsilon) per set and pass (restoration.rs:286-303).
__constant__ int8_t c_sgr_r[16][2] = {{2, 1}, {2, 1}, {2, 1}, {2, 1}, {2, 1}, {2, 1}, {2, 1}, {2, 1},
                                      {2, 1}, {2, 1}, {0, 1}, {0, 1}, {0, 1}, {0, 1}, {2, 0}, {2, 0}};

struct SgrPassConst {
    unsigned scale, p_lim;
};
struct SgrConstTable {
    SgrPassConst c[16][2];
};
constexpr SgrPassConst sgr_pass_const(int n, int e) {
    if (e == 0) return SgrPassConst{0, 0};
    const unsigned n2e = (unsigned)(n * n * e);
    const unsigned scale = ((1u << 20) + n2e / 2) / n2e;
    return SgrPassConst{scale, ((1u << 28) - (1u << 19) + scale - 1) / scale};
}
constexpr SgrConstTable make_sgr_consts() {
    constexpr uint8_t e[16][2] = {{12, 4}, {15, 6}, {18, 8}, {21, 9}, {24, 10}, {29, 11}, {36, 12}, {45, 13},
                                  {56, 14}, {68, 15}, {0, 5},  {0, 8},  {0, 11}, {0, 14}, {30, 0},  {75, 0}};
    SgrConstTable t{};
    for (int k = 0; k < 16; ++k) {
        t.c[k][0] = sgr_pass_const(25, e[k][0]);  // n = 25 samples in a radius-2 box
        t.c[k][1] = sgr_pass_const(9, e[k][1]);   // n = 9 in a radius-1 box
    }
    return t;
}
__device__ const SgrConstTable g_sgr_const = make_sgr_consts();

// The a2 table of box_ab: ((z << 8) + z / 2) / (z + 1), with 1 at z = 0 and
// 256 from z = 255 (restoration.rs:322-328).
struct alignas(16) A2Table {
    uint16_t v[256];
};
constexpr A2Table make_a2_table() {
    A2Table t{};
    for (int z = 0; z < 256; ++z) t.v[z] = (uint16_t)(z >= 255 ? 256 : z == 0 ? 1 : ((z << 8) + z / 2) / (z + 1));
    return t;
}
__device__ const A2Table g_a2 = make_a2_table();

struct LrArgs {
    LrPlane p[3];
    int count;
    int bit_depth;
    int tile_w[3], tile_h[3], tiles_x[3], tiles_y[3], off[3], stripe_h[3];
    unsigned tiles_x_recip[3], unit_recip[3], stripe_recip[3];  // fast_div_recip of each
    int tile_base[4];
};

// Shared-memory layout (dynamic):
//   S      kSRows x kSPitch uint16        staged Source::get values
//   region either H  kSRows x kMaxTile int16   (Wiener horizontal pass)
//          or     A0 kBox0 x kBox uint16, B0 kBox0 x kBox int32 (radius-2 pass,
//                 box rows of odd y only) and A1 kBox x kBox uint16,
//                 B1 kBox x kBox int32 (radius-1 pass)
//   a2tab  256 uint16
//   V      per warp: 2 x kVCols int32   vertical box sums (sum, sum of squares)
constexpr int kVCols = kBox + 4 + 2;     // vertical box sums per row: box columns + 2*radius (even)
constexpr int kBox0 = kBox / 2 + 1;      // radius-2 box rows (odd y only)
constexpr size_t align16(size_t b) { return (b + 15) / 16 * 16; }
constexpr size_t kSBytes = sizeof(uint16_t) * kSRows * kSPitch;
constexpr size_t kA0Bytes = align16(sizeof(uint16_t) * kBox0 * kBox);
constexpr size_t kB0Bytes = sizeof(int32_t) * kBox0 * kBox;
constexpr size_t kA1Bytes = align16(sizeof(uint16_t) * kBox * kBox);
constexpr size_t kB1Bytes = sizeof(int32_t) * kBox * kBox;
constexpr size_t kSgrBytes = kA0Bytes + kB0Bytes + kA1Bytes + kB1Bytes;
constexpr size_t kHBytes = sizeof(int16_t) * kSRows * kMaxTile;
constexpr size_t kRegion = kSgrBytes > kHBytes ? kSgrBytes : kHBytes;
constexpr size_t kVBytes = sizeof(int32_t) * 2 * kVCols * kWarps;
constexpr size_t kLrSmem = kSBytes + kRegion + 256 * sizeof(uint16_t) + kVBytes;

__device__ __forceinline__ int round2i(int v, int s) { return s == 0 ? v : (v + (1 << (s - 1))) >> s; }

__device__ __forceinline__ bool unit_ok(const vaco_av1_lr_unit& u) {
    if (u.type == VACO_AV1_LR_NONE) return true;
    if (u.type == VACO_AV1_LR_WIENER) {
        const int lo[3] = {-5, -23, -17}, hi[3] = {10, 8, 46};
        bool ok = true;
        for (int k = 0; k < 3; ++k)
            ok = ok && u.vertical[k] >= lo[k] && u.vertical[k] <= hi[k] && u.horizontal[k] >= lo[k] &&
                 u.horizontal[k] <= hi[k];
        return ok;
    }
    if (u.type == VACO_AV1_LR_SGRPROJ)
        return u.set >= 0 && u.set < 16 && u.xqd[0] >= -96 && u.xqd[0] <= 31 && u.xqd[1] >= -32 && u.xqd[1] <= 95;
    return false;
}


// Box sums around every box position (br, bc) -- box rows y_lo-1+br (only
// those of odd y when odd_rows_only), box columns x_lo-1+bc -- and the a2 / b
// terms of box_ab (restoration.rs:314-339).  A warp takes whole box rows:
// its lanes first form the (2 RAD + 1)-row vertical sums (and sums of
// squares) of every column the row's boxes reach, in the warp's own buffer
// V, then each box sum as 2 RAD + 1 of those -- 2 (2 RAD + 1) loads per box
// instead of (2 RAD + 1)^2.
// box_ab's a2 and b (restoration.rs:314-339) from a box sum and sum of
// squares, stored at box position (ar, bc).
// A pass's constants for box_ab: scale and p_lim of its set, and the
// Round2 shifts by 2 (bd - 8) and bd - 8 as (v + half) >> shift.
struct BoxConst {
    unsigned scale, p_lim;
    int sh_sq, half_sq, sh, half;
};

template <int RAD>
__device__ __forceinline__ void box_ab(int sum, int sum_sq, int ar, int bc, uint16_t* __restrict__ A,
                                       int32_t* __restrict__ B, const uint16_t* __restrict__ a2tab,
                                       const BoxConst& k) {
    constexpr int n = (2 * RAD + 1) * (2 * RAD + 1);
    constexpr unsigned recip = ((1 << 12) + n / 2) / n;
    const int aa = (sum_sq + k.half_sq) >> k.sh_sq;
    const int d = (sum + k.half) >> k.sh;
    const unsigned p = (unsigned)max(aa * n - d * d, 0);
    const unsigned z = min((min(p, k.p_lim) * k.scale + (1u << 19)) >> 20, 255u);
    const int a2 = a2tab[z];
    const unsigned b = ((unsigned)(256 - a2) * (unsigned)sum * recip + (1u << 11)) >> 12;
    A[ar * kBox + bc] = (uint16_t)a2;
    B[ar * kBox + bc] = (int)b;
}

// Box sums around every box position (br, bc) -- box rows y_lo-1+br (only
// those of odd y when odd_rows_only), box columns x_lo-1+bc -- and their a2
// / b terms.  A warp takes whole box rows: its lanes first form the
// (2 RAD + 1)-row vertical sums (and sums of squares) of 64 columns in the
// warp's own buffer V -- two full passes of 32 lanes -- then each box sum of
// the columns those cover, bc < 64 - 2 RAD, as 2 RAD + 1 of them.  The last
// few columns of every row (bc >= 64 - 2 RAD) are summed directly afterwards,
// all rows' together, so no pass over a row runs with most lanes idle.
template <int RAD>
__device__ __forceinline__ void box_pass(const uint16_t* __restrict__ S, uint16_t* __restrict__ A,
                                         int32_t* __restrict__ B, const uint16_t* __restrict__ a2tab,
                                         int32_t* __restrict__ V, int R, int C, int y_lo, bool odd_rows_only,
                                         const BoxConst& k) {
    constexpr int kMain = 64 - 2 * RAD;  // box columns the V buffer covers
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rows = R + 2, cols = C + 2;
    const int main_cols = min(cols, kMain);
    // Box rows of odd y (= y_lo - 1 + br) are the even br: tiles start on
    // even rows (stripe and unit boundaries are even).
    const int rstep = odd_rows_only ? 2 : 1;
    for (int br = warp * rstep; br < rows; br += kWarps * rstep) {
        // staged row of box row br is br + 2 (box rows start at y0-1, staged at y0-3)
        const uint16_t* srow = S + (br + 2 - RAD) * kSPitch + (kSOff - 1 - RAD);
        __syncwarp();  // the previous row's sums are consumed
        {
            // columns 2 lane and 2 lane + 1 (an odd count computes one
            // column more, which no box below reads)
            const int cc = 2 * lane;
            if (cc < main_cols + 2 * RAD) {
                int s0 = 0, q0 = 0, s1 = 0, q1 = 0;
#pragma unroll
                for (int dy = 0; dy <= 2 * RAD; ++dy) {
                    const int v0 = srow[dy * kSPitch + cc], v1 = srow[dy * kSPitch + cc + 1];
                    s0 += v0;
                    q0 += v0 * v0;
                    s1 += v1;
                    q1 += v1 * v1;
                }
                *reinterpret_cast<int2*>(V + cc) = make_int2(s0, s1);
                *reinterpret_cast<int2*>(V + kVCols + cc) = make_int2(q0, q1);
            }
        }
        __syncwarp();
        {
            // boxes 2 lane and 2 lane + 1 from one window of 2 RAD + 2
            // vertical sums
            const int bc = 2 * lane;
            if (bc < main_cols) {
                int vs[2 * RAD + 2], vq[2 * RAD + 2];
#pragma unroll
                for (int j = 0; j < RAD + 1; ++j) {
                    const int2 a = *reinterpret_cast<const int2*>(V + bc + 2 * j);
                    const int2 b = *reinterpret_cast<const int2*>(V + kVCols + bc + 2 * j);
                    vs[2 * j] = a.x, vs[2 * j + 1] = a.y;
                    vq[2 * j] = b.x, vq[2 * j + 1] = b.y;
                }
                int sum = 0, sum_sq = 0;
#pragma unroll
                for (int dx = 0; dx <= 2 * RAD; ++dx) {
                    sum += vs[dx];
                    sum_sq += vq[dx];
                }
                const int ar = odd_rows_only ? br >> 1 : br;
                box_ab<RAD>(sum, sum_sq, ar, bc, A, B, a2tab, k);
                if (bc + 1 < main_cols)
                    box_ab<RAD>(sum - vs[0] + vs[2 * RAD + 1], sum_sq - vq[0] + vq[2 * RAD + 1], ar, bc + 1, A, B,
                                a2tab, k);
            }
        }
    }
    // The remaining box columns [kMain, cols) of every row, summed directly.
    const int extra = cols - main_cols;  // at most 2 + 2 RAD
    if (extra > 0) {
        const int nrows = odd_rows_only ? (rows + 1) >> 1 : rows;
        const unsigned mx = ((1u << 20) + extra - 1) / extra;  // i / extra = (i mx) >> 20 for i < 2^20 / extra
        for (int i = threadIdx.x; i < nrows * extra; i += kLrThreads) {
            const int row = (int)(((unsigned)i * mx) >> 20), bc = kMain + (i - row * extra);
            const int br = odd_rows_only ? 2 * row : row;
            const uint16_t* box = S + (br + 2 - RAD) * kSPitch + (kSOff - 1 - RAD) + bc;
            int sum = 0, sum_sq = 0;
#pragma unroll
            for (int dy = 0; dy <= 2 * RAD; ++dy)
#pragma unroll
                for (int dx = 0; dx <= 2 * RAD; ++dx) {
                    const int v = box[dy * kSPitch + dx];
                    sum += v;
                    sum_sq += v * v;
                }
            box_ab<RAD>(sum, sum_sq, row, bc, A, B, a2tab, k);
        }
    }
}

// One restoration tile: `block` indexes the tiles of all planes of `a`.
__device__ __forceinline__ void lr_tile(const LrArgs& a, int block) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint16_t* S = reinterpret_cast<uint16_t*>(smem_raw);
    unsigned char* region = smem_raw + kSBytes;
    int16_t* H = reinterpret_cast<int16_t*>(region);
    uint16_t* A0 = reinterpret_cast<uint16_t*>(region);
    int32_t* B0 = reinterpret_cast<int32_t*>(region + kA0Bytes);
    uint16_t* A1 = reinterpret_cast<uint16_t*>(region + kA0Bytes + kB0Bytes);
    int32_t* B1 = reinterpret_cast<int32_t*>(region + kA0Bytes + kB0Bytes + kA1Bytes);
    uint16_t* a2tab = reinterpret_cast<uint16_t*>(region + kRegion);
    int32_t* Vw = reinterpret_cast<int32_t*>(region + kRegion + 256 * sizeof(uint16_t)) +
                  (threadIdx.x >> 5) * 2 * kVCols;  // this warp's vertical sums

    int pl = 0;
    while (pl + 1 < a.count && block >= a.tile_base[pl + 1]) ++pl;
    const LrPlane& P = a.p[pl];
    const int local = block - a.tile_base[pl];
    const int ty = (int)fast_div(local, a.tiles_x[pl], a.tiles_x_recip[pl]), tx = local - ty * a.tiles_x[pl];
    const int off = a.off[pl], sh = a.stripe_h[pl];
    const int y_lo = max(ty * a.tile_h[pl] - off, 0);
    const int y_hi = min((ty + 1) * a.tile_h[pl] - off, P.height);
    const int x_lo = tx * a.tile_w[pl];
    const int x_hi = min(x_lo + a.tile_w[pl], P.width);
    if (y_lo >= y_hi || x_lo >= x_hi) return;
    const int R = y_hi - y_lo, C = x_hi - x_lo;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // Unit of this tile (unit_index, restoration.rs:124-133).
    const int urow = min((int)fast_div(y_lo + off, P.unit_size, a.unit_recip[pl]), P.unit_rows - 1);
    const int ucol = min((int)fast_div(x_lo, P.unit_size, a.unit_recip[pl]), P.unit_cols - 1);
    vaco_av1_lr_unit u;
    if (P.copy_only) {
        u.type = VACO_AV1_LR_NONE;
    } else {
        const int ui = urow * P.unit_cols + ucol;
        u = P.units[ui];
        // Every unit is covered by at least one tile, so checking each tile's
        // unit validates the whole unit array (RestorationUnit::validate).
        if (P.unit_status && tid == 0 && !unit_ok(u))
            report_error(P.unit_status, STAGE_LR, lr_key_position(P.plane_index, LRC_COEFFICIENT, ui),
                         VACO_AV1_MSG_LR_COEFFICIENT);
    }
    const int bd = a.bit_depth, maxv = (1 << bd) - 1;

    if (P.copy_only || (u.type != VACO_AV1_LR_WIENER && u.type != VACO_AV1_LR_SGRPROJ)) {
        // RestorationUnit::None: the CDEF output, restoration.rs:194.  The
        // tile is at most 64 x 64 samples = 512 16-byte vectors, so each
        // thread has both of its loads in flight before it stores.
        const bool vec = ((P.after.stride | P.out.stride) & 7) == 0 &&
                         ((reinterpret_cast<uintptr_t>(P.after.data) | reinterpret_cast<uintptr_t>(P.out.data)) & 15) == 0;
        const int vpr = (C + 7) >> 3;
        const unsigned mv = ((1u << 20) + vpr - 1) / vpr;  // i / vpr = (i mv) >> 20 for i < 2^20 / vpr
        uint4 q[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int i = tid + j * kLrThreads, r = (int)(((unsigned)i * mv) >> 20), x = x_lo + 8 * (i - r * vpr);
            if (vec && i < R * vpr && x + 8 <= x_hi)
                q[j] = __ldg(reinterpret_cast<const uint4*>(P.after.data + (long)(y_lo + r) * P.after.stride + x));
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int i = tid + j * kLrThreads, r = (int)(((unsigned)i * mv) >> 20), x = x_lo + 8 * (i - r * vpr);
            if (i >= R * vpr) continue;
            uint16_t* dst = P.out.data + (long)(y_lo + r) * P.out.stride + x;
            if (vec && x + 8 <= x_hi) {
                *reinterpret_cast<uint4*>(dst) = q[j];
            } else {
                const uint16_t* src = P.after.data + (long)(y_lo + r) * P.after.stride + x;
                for (int k = 0; k < min(8, x_hi - x); ++k) dst[k] = src[k];
            }
        }
        return;
    }

    // Stage Source::get (restoration.rs:233-244): rows y_lo-3 .. y_hi+2,
    // columns x_lo-8 .. x_lo+72 as 10 aligned 8-sample vectors per row, all
    // in flight at once by cp.async (edge vectors are gathered sample by sample).
    const int stripe = (int)fast_div(y_lo + off, sh, a.stripe_recip[pl]);
    const int s_start = stripe * sh - off, s_end = s_start + sh - 1;
    const int srows = R + 6;
    const bool compact = P.before_rows.data != nullptr;
    const DevPlaneC& BP = compact ? P.before_rows : P.before;
    const bool vec_ok = ((BP.stride | P.after.stride) & 7) == 0 &&
                        ((reinterpret_cast<uintptr_t>(BP.data) | reinterpret_cast<uintptr_t>(P.after.data)) & 15) == 0;
    for (int i = tid; i < srows * (kSPitch / 8); i += kLrThreads) {
        const int r = i / (kSPitch / 8), v = i - r * (kSPitch / 8);
        const int y = clampi(y_lo - 3 + r, 0, P.height - 1);
        const uint16_t* row;
        if (y < s_start) {
            const int yy = max(y, s_start - 2);
            row = BP.data + (long)(compact ? 4 * stripe + (yy - (s_start - 2)) : yy) * BP.stride;
        } else if (y > s_end) {
            const int yy = min(y, s_end + 2);
            row = BP.data + (long)(compact ? 4 * (stripe + 1) + 2 + (yy - (s_end + 1)) : yy) * BP.stride;
        } else {
            row = P.after.data + (long)y * P.after.stride;
        }
        const int x = x_lo - kSOff + 8 * v;
        uint16_t* d = S + r * kSPitch + 8 * v;
        if (vec_ok && x >= 0 && x + 8 <= P.width) {
            const unsigned dst = (unsigned)__cvta_generic_to_shared(d);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(row + x) : "memory");
        } else {
#pragma unroll
            for (int k = 0; k < 8; ++k) d[k] = __ldg(row + clampi(x + k, 0, P.width - 1));
        }
    }
    asm volatile("cp.async.commit_group;\ncp.async.wait_all;\n" ::: "memory");
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
        // Horizontal pass: a lane filters two adjacent columns from the 8
        // samples they share, and stores both as one word (for an odd C the
        // second value lands in an unused column of the row).
        for (int r = warp; r < srows; r += kWarps) {
            const uint16_t* s = S + r * kSPitch + kSOff - 3;
            const int c = 2 * lane;  // C <= 64
            if (c < C) {
                int v[8];
#pragma unroll
                for (int t = 0; t < 8; ++t) v[t] = s[c + t];
                int h0 = 0, h1 = 0;
#pragma unroll
                for (int t = 0; t < 7; ++t) {
                    h0 += hv[t] * v[t];
                    h1 += hv[t] * v[t + 1];
                }
                h0 = clampi(round2i(h0, round_h), -offset, limit - offset);
                h1 = clampi(round2i(h1, round_h), -offset, limit - offset);
                *reinterpret_cast<uint32_t*>(H + r * kMaxTile + c) = (uint32_t)(h0 & 0xFFFF) | ((uint32_t)h1 << 16);
            }
        }
        __syncthreads();
        // Vertical pass: each thread walks rows 8 warp .. 8 warp + 7 of
        // columns 2 lane and 2 lane + 1, reading each intermediate row once,
        // both columns as one word.
        const int k0 = 8 * warp;
        const int c = 2 * lane;
        if (k0 >= R || c >= C) return;
        const bool second = c + 1 < C;
        const bool pair_store = ((P.out.stride | x_lo) & 1) == 0 && (reinterpret_cast<uintptr_t>(P.out.data) & 3) == 0;
        int h[14][2];
#pragma unroll
        for (int t = 0; t < 14; ++t) {
            const uint32_t w = *reinterpret_cast<const uint32_t*>(H + min(k0 + t, kSRows - 1) * kMaxTile + c);
            h[t][0] = (int16_t)(w & 0xFFFF);
            h[t][1] = (int16_t)(w >> 16);
        }
        uint16_t* orow = P.out.data + (long)(y_lo + k0) * P.out.stride + x_lo + c;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (k0 + j >= R) break;
            int v[2];
#pragma unroll
            for (int x = 0; x < 2; ++x) {
                int sum = 0;
#pragma unroll
                for (int t = 0; t < 7; ++t) sum += vv[t] * h[j + t][x];
                v[x] = clampi(round2i(sum, 14 - round_h), 0, maxv);
            }
            if (pair_store && second) {
                *reinterpret_cast<uint32_t*>(orow) = (uint32_t)v[0] | ((uint32_t)v[1] << 16);
            } else {
                orow[0] = (uint16_t)v[0];
                if (second) orow[1] = (uint16_t)v[1];
            }
            orow += P.out.stride;
        }
        return;
    }

    // ---- self-guided (restoration.rs:314-384)
    const int set = min(max((int)u.set, 0), 15);
    const int r0 = c_sgr_r[set][0], r1 = c_sgr_r[set][1];
    if (tid < 256 * 2 / 16)
        reinterpret_cast<uint4*>(a2tab)[tid] = __ldg(reinterpret_cast<const uint4*>(g_a2.v) + tid);
    // Both box passes, into their own buffers, then one final pass.
    __syncthreads();  // a2tab
    const int sh1 = bd - 8, sh2 = 2 * (bd - 8);
    if (r0 != 0) {
        const SgrPassConst c = g_sgr_const.c[set][0];
        const BoxConst k{c.scale, c.p_lim, sh2, sh2 ? 1 << (sh2 - 1) : 0, sh1, sh1 ? 1 << (sh1 - 1) : 0};
        box_pass<2>(S, A0, B0, a2tab, Vw, R, C, y_lo, true, k);
    }
    if (r1 != 0) {
        const SgrPassConst c = g_sgr_const.c[set][1];
        const BoxConst k{c.scale, c.p_lim, sh2, sh2 ? 1 << (sh2 - 1) : 0, sh1, sh1 ? 1 << (sh1 - 1) : 0};
        box_pass<1>(S, A1, B1, a2tab, Vw, R, C, y_lo, false, k);
    }
    __syncthreads();

    // Pixels of this thread: rows k0 .. k0+7 (k0 = 8 warp) of columns 2 lane
    // and 2 lane + 1; pixel row k is box row k + 1.  Walking down its rows, a
    // thread reads each box row of A / B once, the four box columns its two
    // pixels share as two 32-bit (A) and two 64-bit (B) loads.
    //   radius 2 (box rows of odd y only; y_lo is even, so pixel row k0 + j
    //   has odd y when j is odd): with g = 6 A[c] + 5 (A[c-1] + A[c+1]) of a
    //   box row, an odd row takes g of its own box row (shift 8), an even
    //   row g of the box rows above and below (shift 9);
    //   radius 1: 4 (A[c-1] + A[c] + A[c+1]) of the box row itself, 3 x the
    //   same three of the rows above and below, plus A[c] of those two --
    //   weight 4 on the cross, 3 on the corners.  Likewise for b.
    const int w0 = u.xqd[0], w1 = u.xqd[1];
    const int k0 = 8 * warp;
    const int c = 2 * lane;
    if (k0 >= R || c >= C) return;
    const bool second = c + 1 < C;
    // box columns c .. c + 3 of a row (the neighbourhoods of pixels c, c + 1)
    auto quad = [&](const uint16_t* A, const int32_t* B, int i, int (&qa)[4], int (&qb)[4]) {
        const uint32_t a01 = *reinterpret_cast<const uint32_t*>(A + i);
        const uint32_t a23 = *reinterpret_cast<const uint32_t*>(A + i + 2);
        const int2 b01 = *reinterpret_cast<const int2*>(B + i);
        const int2 b23 = *reinterpret_cast<const int2*>(B + i + 2);
        qa[0] = a01 & 0xFFFF, qa[1] = a01 >> 16, qa[2] = a23 & 0xFFFF, qa[3] = a23 >> 16;
        qb[0] = b01.x, qb[1] = b01.y, qb[2] = b23.x, qb[3] = b23.y;
    };
    auto g0 = [&](int br, int (&ga)[2], int (&gb)[2]) {  // br even: compact row br / 2
        int qa[4], qb[4];
        quad(A0, B0, (br >> 1) * kBox + c, qa, qb);
#pragma unroll
        for (int x = 0; x < 2; ++x) {
            ga[x] = 5 * (qa[x] + qa[x + 2]) + 6 * qa[x + 1];
            gb[x] = 5 * (qb[x] + qb[x + 2]) + 6 * qb[x + 1];
        }
    };
    int h3a[3][2], h3b[3][2], ca[3][2], cb[3][2];
    auto row1 = [&](int br, int slot) {
        int qa[4], qb[4];
        quad(A1, B1, br * kBox + c, qa, qb);
#pragma unroll
        for (int x = 0; x < 2; ++x) {
            ca[slot][x] = qa[x + 1];
            cb[slot][x] = qb[x + 1];
            h3a[slot][x] = qa[x] + qa[x + 1] + qa[x + 2];
            h3b[slot][x] = qb[x] + qb[x + 1] + qb[x + 2];
        }
    };
    int pa[2] = {0, 0}, pb[2] = {0, 0}, na[2] = {0, 0}, nb[2] = {0, 0};
    if (r0) g0(k0, pa, pb);
    if (r1) {
        row1(k0, 0);
        row1(k0 + 1, 1);
    }
    const bool pair_store = ((P.out.stride | x_lo) & 1) == 0 && (reinterpret_cast<uintptr_t>(P.out.data) & 3) == 0;
    uint16_t* orow = P.out.data + (long)(y_lo + k0) * P.out.stride + x_lo + c;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int k = k0 + j;
        const uint32_t ow = *reinterpret_cast<const uint32_t*>(S + (k + 3) * kSPitch + kSOff + c);
        const int orig[2] = {(int)(ow & 0xFFFF), (int)(ow >> 16)};
        int f0[2] = {orig[0] << 4, orig[1] << 4}, f1[2] = {orig[0] << 4, orig[1] << 4};
        if (r0) {
            if ((j & 1) == 0) {
                g0(k + 2, na, nb);
#pragma unroll
                for (int x = 0; x < 2; ++x) f0[x] = round2i((pa[x] + na[x]) * orig[x] + (pb[x] + nb[x]), 9);
            } else {
#pragma unroll
                for (int x = 0; x < 2; ++x) {
                    f0[x] = round2i(na[x] * orig[x] + nb[x], 8);
                    pa[x] = na[x];
                    pb[x] = nb[x];
                }
            }
        }
        if (r1) {
            row1(k + 2, (j + 2) % 3);
            const int u_ = j % 3, m_ = (j + 1) % 3, d_ = (j + 2) % 3;
#pragma unroll
            for (int x = 0; x < 2; ++x) {
                const int aa = 4 * h3a[m_][x] + 3 * (h3a[u_][x] + h3a[d_][x]) + ca[u_][x] + ca[d_][x];
                const int bb = 4 * h3b[m_][x] + 3 * (h3b[u_][x] + h3b[d_][x]) + cb[u_][x] + cb[d_][x];
                f1[x] = round2i(aa * orig[x] + bb, 9);
            }
        }
        if (k < R) {
            int v[2];
#pragma unroll
            for (int x = 0; x < 2; ++x)
                v[x] = clampi(round2i(w0 * f0[x] + w1 * (orig[x] << 4) + (128 - w0 - w1) * f1[x], 11), 0, maxv);
            if (pair_store && second) {
                *reinterpret_cast<uint32_t*>(orow) = (uint32_t)v[0] | ((uint32_t)v[1] << 16);
            } else {
                orow[0] = (uint16_t)v[0];
                if (second) orow[1] = (uint16_t)v[1];
            }
        }
        orow += P.out.stride;
    }
}

__global__ void __launch_bounds__(kLrThreads, 4) restoration_kernel(LrArgs a) {
    overlap_prologue();
    lr_tile(a, blockIdx.x);
}

// Batched form: one CTA per tile of all frames of a batch (see dbcdef.cu).
// MIN_CTAS picks the register budget: 4 resident CTAs per SM leave 64
// registers a thread, 3 leave 80.
template <int MIN_CTAS>
__global__ void __launch_bounds__(kLrThreads, MIN_CTAS) restoration_batch_kernel(const LrArgs* __restrict__ frames,
                                                                                const int* __restrict__ tile_prefix,
                                                                                int n) {
    const int f = frame_of_tile(tile_prefix, n, blockIdx.x);
    lr_tile(frames[f], blockIdx.x - tile_prefix[f]);
}

// RestorationUnit::validate (restoration.rs:67-91).
__global__ void lr_unit_check_kernel(const vaco_av1_lr_unit* units, int n, int plane, DeviceStatus* st) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!unit_ok(units[i]))
        report_error(st, STAGE_LR, lr_key_position(plane, LRC_COEFFICIENT, i), VACO_AV1_MSG_LR_COEFFICIENT);
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

// A restoration plane that only copies `after` into `out` (frame-level
// restoration off for the plane): tiled like a 64-sample unit, no units.
LrPlane copy_only_plane(const DevPlaneC& after, const DevPlane& out, int w, int h, int sub_y, int plane_index) {
    LrPlane p{};
    p.before = DevPlaneC{nullptr, 0, 0, 0};
    p.before_rows = DevPlaneC{nullptr, 0, 0, 0};
    p.after = after;
    p.out = out;
    p.width = w;
    p.height = h;
    p.unit_size = 64;
    p.sub_y = sub_y;
    p.units = nullptr;
    p.unit_cols = p.unit_rows = 1;
    p.copy_only = 1;
    p.plane_index = plane_index;
    p.unit_status = nullptr;
    return p;
}

size_t lr_args_size() { return sizeof(LrArgs); }

// Kernel arguments of up to 3 planes; returns the number of tiles.
int build_lr_args(const LrPlane* planes, int count, int bit_depth, void* out) {
    LrArgs a;
    memset(&a, 0, sizeof a);
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
        a.tiles_x_recip[k] = fast_div_recip((unsigned)a.tiles_x[k]);
        a.unit_recip[k] = fast_div_recip((unsigned)planes[k].unit_size);
        a.stripe_recip[k] = fast_div_recip((unsigned)sh);
        a.tile_base[k] = total;
        total += a.tiles_x[k] * a.tiles_y[k];
    }
    for (int k = count; k < 4; ++k) a.tile_base[k] = total;
    memcpy(out, &a, sizeof a);
    return total;
}

// The opt-in above 48 KB of dynamic shared memory is a per-device attribute.
// Atomic, as several host threads may launch on a device at once (a repeated
// cudaFuncSetAttribute is harmless).
std::atomic<unsigned long long> g_lr_attr_devices{0};

cudaError_t lr_kernel_attributes() {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !(g_lr_attr_devices.load(std::memory_order_acquire) & (1ull << dev))) {
        cudaError_t e = cudaFuncSetAttribute(restoration_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kLrSmem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(restoration_batch_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kLrSmem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(restoration_batch_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kLrSmem);
        if (e != cudaSuccess) return e;
        g_lr_attr_devices.fetch_or(1ull << dev, std::memory_order_release);
    }
    return cudaSuccess;
}

cudaError_t launch_restoration(const LrPlane* planes, int count, int bit_depth, cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    LrArgs a;
    const int total = build_lr_args(planes, count, bit_depth, &a);
    cudaError_t e = lr_kernel_attributes();
    if (e != cudaSuccess) return e;
    if (total == 0) return cudaSuccess;
    return launch_overlapped(restoration_kernel, dim3(total), dim3(kLrThreads), kLrSmem, stream, a);
}

cudaError_t launch_restoration_batch(const void* dev_args, const int* dev_prefix, int n, int tiles, int ctas_per_sm,
                                     cudaStream_t stream) {
    if (tiles <= 0) return cudaSuccess;
    cudaError_t e = lr_kernel_attributes();
    if (e != cudaSuccess) return e;
    const LrArgs* args = static_cast<const LrArgs*>(dev_args);
    if (ctas_per_sm <= 3)
        restoration_batch_kernel<3><<<tiles, kLrThreads, kLrSmem, stream>>>(args, dev_prefix, n);
    else
        restoration_batch_kernel<4><<<tiles, kLrThreads, kLrSmem, stream>>>(args, dev_prefix, n);
    return cudaGetLastError();
}

cudaError_t launch_lr_unit_check(const vaco_av1_lr_unit* units, int n, int plane, DeviceStatus* status,
                                 cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    lr_unit_check_kernel<<<div_up(n, 128), 128, 0, stream>>>(units, n, plane, status);
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
