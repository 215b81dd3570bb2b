// dbcdef.cu -- deblocking (AV1 7.14) fused with CDEF (vaco src/decode.rs:739-862)
// in one pass over each 64x64 filter block.
//
// Why fused: the chain needs the deblocked picture only (a) as CDEF's input
// and (b) as restoration's pre-CDEF source, which restoration reads at just
// four rows around every stripe boundary (src/restoration.rs:233-244).  One
// CTA therefore stages its tile with a 16-sample halo, runs both deblocking
// passes in shared memory (all vertical edges of the staged region, then the
// horizontal edges that reach the CDEF window), writes the stripe-boundary
// rows to a compact buffer, and filters CDEF straight from the deblocked tile.
// The deblocked picture never round-trips through HBM.
//
// Halo arithmetic (plane units, tile [x0, x0+tw) x [y0, y0+th)):
//   CDEF reads the deblocked window [x0-2, x0+tw+2) x [y0-2, y0+th+2).
//   An edge of filter size n sits on a multiple of n (7.14.2: it is a
//   transform edge of the block on its q side), and it modifies n/2 samples
//   on either side at most (14-tap: 6, 8-tap: 3, 6-tap: 2, 4-tap: 2).  The
//   edges that reach the window are therefore exactly the 4-aligned ones in
//   [y0, y0+th] (horizontal) and [x0, x0+tw] (vertical); the edge at y0-4,
//   say, is a size-4 edge and stops at y0-3.
//   Those horizontal edges read rows [E-7, E+6] (luma, 14-tap only where E is
//   a multiple of 16) or [E-3, E+2] (chroma, at most 6 taps): rows
//   [y0-7, y0+th+7) for luma and [y0-3, y0+th+3) for chroma, which is where
//   the vertical pass must run.  Vertical edges read columns [X-7, X+6].
// The staged region is [x0-8, x0+tw+8) x [y0-8, y0+th+8).
#include <algorithm>
#include <atomic>
#include <cstring>

#include "cdef_core.cuh"
#include "common.cuh"
#include "deblock_core.cuh"
#include "kernels.cuh"

namespace vaco {

namespace {

using namespace cdefk;
using namespace dbk;

constexpr int kHalo = 8;
// Edge segments (one edge x one 4-sample cell) per pass and plane are at most
// (th/4+4) x (tw/4+1) = 340.  Size-class lists: 0 = size 4 (any plane, up to
// 3 x 340), 1 = chroma size 8 (2 x 340), 2 = luma size 8, 3 = luma size 16.
__constant__ int c_list_off[4] = {0, 1020, 1700, 2040};
constexpr int kListTotal = 2380;
// Rows of the luma CDEF window (th + 4) kept as odd-aligned pairs.
constexpr int kShiftRows = 64 + 4;

// Side-information window of a tile: cells [mi_r0 - kWinTop, +kWinRows) x
// [mi_c0 - kWinLeft, +kWinCols) of the luma maps, and the same shape around
// the tile's own cell origin in the chroma transform map.  Relative to the
// tile, the two passes read transform sizes at cell rows [-2, 17] and
// columns [-1, 16] (previous cells included), and subsampled chroma reads
// levels at luma cells up to row and column 17.
constexpr int kWinTop = 3, kWinLeft = 2, kWinRows = 22, kWinCols = 20, kWinCells = kWinRows * kWinCols;
struct SideWindow {
    uint8_t tx[2][kWinCells];  // luma, chroma TX_SIZE
    uint32_t lvl[kWinCells];   // loop-filter levels (Yv, Yh, U, V) when a level map is given
};

// n / d for the tile loops' small quotients (segments per edge row 9, 10,
// 17, 18; 16-byte vectors per staged row 6, 10; sentinel window widths 36,
// 68) as one multiply and shift: with m = ceil(2^20 / d), (n m) >> 20 is
// n / d for 0 <= n < 2^20 / d, which every loop here stays under (n is at
// most 80 x 10, 20 x 18 or 68 x 68).  m is computed once per loop.
__device__ __forceinline__ unsigned small_div_magic(int d) { return ((1u << 20) + (unsigned)d - 1) / (unsigned)d; }
__device__ __forceinline__ int small_div(int n, unsigned m) { return (int)(((unsigned)n * m) >> 20); }

struct PlaneGeom {
    int tw, th;        // tile extent in this plane
    int pitch, rows;   // staged region
    int sx, sy;
};

__device__ __forceinline__ PlaneGeom plane_geom(int p, int ssx, int ssy) {
    PlaneGeom g;
    g.sx = p ? ssx : 0;
    g.sy = p ? ssy : 0;
    g.tw = 64 >> g.sx;
    g.th = 64 >> g.sy;
    g.pitch = g.tw + 2 * kHalo;
    g.rows = g.th + 2 * kHalo;
    return g;
}

struct DbCdefArgs {
    DevPlaneC src[3];
    DevPlane dst[3];            // CDEF output planes
    DevPlane pre_rows[3];       // stripe-boundary rows of the deblocked picture (may be null)
    int num_planes, ssx, ssy, bit_depth, shift;
    int mi_rows, mi_cols, coded_width, coded_height;
    // deblocking
    const uint8_t* tx_luma;
    const uint8_t* tx_chroma;
    const uint8_t* lvl_map;
    uint8_t levels[4];
    int sharpness;
    int deblock_on;
    // CDEF
    int cdef_on;
    const uint8_t* skip;
    const int32_t* cdef_idx;
    int cdef_stride, cdef_count;
    int damping;
    uint8_t y_pri[8], y_sec[8], uv_pri[8], uv_sec[8];
    DeviceStatus* status;
    int vec_ok;
    int staged_vectors;         // 16-byte vectors of all staged planes together
    DirectPlane direct[3];      // final output written here too (see DirectPlane)
    size_t plane_off[3];        // shared-memory offset (samples) of each staged plane
};

// CDEF output of one plane tile from the staged (deblocked) samples: one warp
// filters block row br; lane l owns pixel pairs at tile column 2*(l % ppr),
// rows l / ppr + RPI*j.  PITCH is the staged pitch, BH the block height.
// pri_on / sec_on: the tile preset's primary / secondary strength is
// non-zero; with neither, every sample stays as it is.
// SHIFT (luma): s1 holds the tile's luma pairs that start on odd samples,
// kShiftRows rows from row kHalo - 2 on the staged pitch, so every tap is a
// single aligned word.
template <int PITCH, int BH, int RPI, bool EDGE, bool SHIFT>
__device__ __forceinline__ void filter_pairs(const uint16_t* t, const uint32_t* s1, const DevPlane& d,
                                             const DirectPlane* D, int px0, int py0, int tw, const uint8_t* active,
                                             const PairBlock* blocks, bool pri_on, bool sec_on, int br, int lane,
                                             int sx) {
    const int ppr = 32 / RPI;              // pairs per row
    const int lp = lane % ppr, lr = lane / ppr;
    const int x = 2 * lp;
    if (x >= tw) return;
    const int bx = x >> (3 - sx);
    const int gx = px0 + x;
    const bool col_in = gx < d.width;
    const int r0 = br * BH;
    if (py0 + r0 >= d.height) return;
    const int rows_here = min(BH, d.height - (py0 + r0));
    const int b = br * 8 + bx;
    const int base_i = (kHalo + r0 + lr) * PITCH + kHalo + x;  // left sample, first row of this lane
    uint32_t* o = reinterpret_cast<uint32_t*>(d.data + (long)(py0 + r0 + lr) * d.stride + gx);
    const long ostride = (long)d.stride * RPI / 2;  // words per RPI rows
    const uint32_t* cw = reinterpret_cast<const uint32_t*>(t + base_i);
    // The final output too, for a plane without restoration (DirectPlane).
    uint16_t* od = nullptr;
    int od_rows = 0;
    bool od_pair = false;
    if (D && D->out.data && gx < D->out.width) {
        od = D->out.data + (long)(py0 + r0 + lr) * D->out.stride + gx;
        od_rows = min(BH, D->out.height - (py0 + r0));
        od_pair = gx + 1 < D->out.width;
    }
    auto put = [&](int j, uint32_t v) {
        if (od && lr + RPI * j < od_rows) {
            uint16_t* q = od + (long)j * RPI * D->out.stride;
            if (od_pair) *reinterpret_cast<uint32_t*>(q) = v;
            else *q = (uint16_t)v;
        }
    };
    if ((pri_on || sec_on) && active[b]) {
        const PairBlock f = blocks[b];
        if (SHIFT) {
            const uint32_t* t32 = reinterpret_cast<const uint32_t*>(t);
            auto word_tap = [&](int i) {  // i: staged index of the pair's first sample
                return WordTap{(i & 1) ? s1 + ((i >> 1) - (kHalo - 2) * (PITCH / 2)) : t32 + (i >> 1)};
            };
            WordTap taps[12];
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                taps[2 * k] = word_tap(base_i + f.off[k]);
                taps[2 * k + 1] = word_tap(base_i - f.off[k]);
            }
#pragma unroll 1  // smaller code: the fused kernel is sensitive to instruction fetch
            for (int j = 0; j < BH / RPI; ++j) {
                const int woff = j * RPI * PITCH / 2;
                const uint32_t v = filter_pair<EDGE>(cw[woff], taps, woff, f, pri_on, sec_on);
                if (col_in && lr + RPI * j < rows_here) o[j * ostride] = v;
                put(j, v);
            }
        } else {
            PairTap taps[12];
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                taps[2 * k] = pair_tap(t, base_i + f.off[k]);
                taps[2 * k + 1] = pair_tap(t, base_i - f.off[k]);
            }
#pragma unroll 1  // smaller code: the fused kernel is sensitive to instruction fetch
            for (int j = 0; j < BH / RPI; ++j) {
                const int woff = j * RPI * PITCH / 2;
                const uint32_t v = filter_pair<EDGE>(cw[woff], taps, woff, f, pri_on, sec_on);
                if (col_in && lr + RPI * j < rows_here) o[j * ostride] = v;
                put(j, v);
            }
        }
    } else if (col_in) {
#pragma unroll
        for (int j = 0; j < BH / RPI; ++j) {
            const uint32_t v = cw[j * RPI * PITCH / 2];
            if (lr + RPI * j < rows_here) o[j * ostride] = v;
            put(j, v);
        }
    }
}

template <int PITCH, int BH, int RPI, bool SHIFT>
__device__ __forceinline__ void filter_pairs_edge(bool edge, const uint16_t* t, const uint32_t* s1, const DevPlane& d,
                                                  const DirectPlane* D,
                                                  int px0, int py0, int tw, const uint8_t* active,
                                                  const PairBlock* blocks, bool pri_on, bool sec_on, int warp,
                                                  int lane, int sx, int nwarps) {
    for (int br = warp; br < 8; br += nwarps) {  // 8 block rows
        if (edge)
            filter_pairs<PITCH, BH, RPI, true, SHIFT>(t, s1, d, D, px0, py0, tw, active, blocks, pri_on, sec_on, br, lane,
                                                     sx);
        else
            filter_pairs<PITCH, BH, RPI, false, SHIFT>(t, s1, d, D, px0, py0, tw, active, blocks, pri_on, sec_on, br,
                                                      lane, sx);
    }
}

// Segment-list entry: level (6 bits) | samples on the q side, capped at 8 (4)
// | on the p side, capped at 8 (4) | staged offset of q0 on the segment's
// first line (13) | plane (2) | first cell of its edge (1) | last cell (1).
// Capping at 8 keeps the clamping of load_line / store_at exact: no filter
// reaches more than 7 samples from its edge.
__device__ __forceinline__ uint32_t seg_entry(int lvl, int nq, int np, int off, int p, bool first, bool last) {
    return (uint32_t)lvl | ((uint32_t)min(nq, 8) << 6) | ((uint32_t)min(np, 8) << 10) | ((uint32_t)off << 14) |
           ((uint32_t)p << 27) | ((uint32_t)first << 29) | ((uint32_t)last << 30);
}

template <int STEP>
__device__ __forceinline__ void filter_line_class(int cls, uint16_t* q, int step, int nq, int np, const Strength& s,
                                                  int bd) {
    if (cls == 0) line_size4<STEP>(q, step, nq, np, s, bd);
    else if (cls == 1) line_size6<STEP>(q, step, nq, np, s, bd);
    else if (cls == 2) line_size8<STEP>(q, step, nq, np, s, bd);
    else line_size16<STEP>(q, step, nq, np, s, bd);
}

// The edge segments of both deblocking passes over the staged tiles of every
// plane, cell by cell.  A cell is a 4x4 block of samples at (xp, yp) =
// (px0 - 4 + 4 cc, py0 - 4 top + 4 cr), top = 2 (luma) or 1 (chroma), on
// (th/4 + 2 top) x (tw/4 + 2) cells.  Its left side is a candidate segment
// of pass 0 (vertical edges X = px0 + 4e, e <= tw/4, on rows from py0-8 or
// py0-4) and its top side one of pass 1 (horizontal edges E = py0 + 4e,
// e <= th/4, on columns from px0-4); the two share the cell's position
// checks, transform size and level word.  Each candidate gets its decision
// (7.14.2-7.14.5: on screen, transform edge, filter size, level) and joins
// its pass's list of its size class: pass 0 at s_list / s_count, pass 1 at
// s_list + kListTotal / s_count + 4.  The decisions read only the side
// information, never samples (s_count zeroed beforehand; the caller's
// barrier publishes the lists).
template <int NT>
__device__ __forceinline__ void deblock_lists(const DbCdefArgs& a, int ssx, int ssy, int x0, int y0,
                                              const SideWindow& side, uint32_t* s_list, int* s_count) {
    const int tid = threadIdx.x;
    const PlaneGeom gl = plane_geom(0, ssx, ssy), gc = plane_geom(1, ssx, ssy);
    const int nrl = gl.th / 4 + 4, ncl = gl.tw / 4 + 2;  // luma cells: rows, columns
    const int nrc = gc.th / 4 + 2, ncc = gc.tw / 4 + 2;  // chroma
    const int n0 = nrl * ncl, nc = a.num_planes > 1 ? nrc * ncc : 0;
    const unsigned m0 = small_div_magic(ncl), mc = small_div_magic(ncc);
    const int mi_r0 = y0 >> 2, mi_c0 = x0 >> 2;
    for (int i = tid; i < n0 + 2 * nc; i += NT) {
        int p = 0, j = i;
        if (j >= n0) {
            j -= n0;
            p = 1;
            if (j >= nc) {
                j -= nc;
                p = 2;
            }
        }
        if (p != 0 && a.levels[1 + p] == 0) continue;
        const PlaneGeom g = p ? gc : gl;
        const int nr = p ? nrc : nrl, ncol = p ? ncc : ncl, top = p ? 1 : 2;
        const int cr = small_div(j, p ? mc : m0), cc = j - cr * ncol;
        const DevPlane& P = a.dst[p];
        const int px0 = x0 >> g.sx, py0 = y0 >> g.sy;
        const int yp = py0 + 4 * (cr - top), xp = px0 - 4 + 4 * cc;
        const int col = (xp >> 2) << g.sx, row = (yp >> 2) << g.sy;
        if (!(xp >= 0 && yp >= 0 && xp < P.width && yp < P.height && col * 4 < a.coded_width &&
              row * 4 < a.coded_height))
            continue;
        const bool vert = cc >= 1 && xp > 0;                              // pass 0 candidate
        const bool horz = cr >= top && cr - top <= g.th / 4 && yp > 0;    // pass 1 candidate
        if (!vert && !horz) continue;
        const uint8_t* map = side.tx[p ? 1 : 0];
        const int w = (((yp - py0) >> 2) + kWinTop) * kWinCols + ((xp - px0) >> 2) + kWinLeft;  // multiples of 4
        const int cur = map[w];
        const int r = row | g.sy, c = col | g.sx;
        const int lw = (r - mi_r0 + kWinTop) * kWinCols + c - mi_c0 + kWinLeft;
        const uint32_t lv = a.lvl_map ? side.lvl[lw] : 0;
        const int off = (yp - py0 + kHalo) * g.pitch + (xp - px0 + kHalo);
        if (vert) {
            const int cl = tx_w_log2(cur), pl = tx_w_log2(map[w - 1]);
            if ((xp & ((1 << cl) - 1)) == 0) {
                const int li = p == 0 ? 0 : p + 1;  // level index (7.14.5)
                int lvl;
                if (a.lvl_map) {
                    lvl = (lv >> (8 * li)) & 0xFF;
                    if (lvl == 0) lvl = (side.lvl[lw - (1 << g.sx)] >> (8 * li)) & 0xFF;
                } else {
                    lvl = a.levels[li];
                }
                if (lvl != 0) {
                    const int size = min(p ? 8 : 16, 1 << min(cl, pl));
                    const int cls = size == 4 ? 0 : p ? 1 : size == 8 ? 2 : 3;
                    const int at = atomicAdd(&s_count[cls], 1);
                    s_list[c_list_off[cls] + at] = seg_entry(lvl, P.width - xp, xp, off, p, cr == 0, cr == nr - 1);
                }
            }
        }
        if (horz) {
            const int cl = tx_h_log2(cur), pl = tx_h_log2(map[w - kWinCols]);
            if ((yp & ((1 << cl) - 1)) == 0) {
                const int li = p == 0 ? 1 : p + 1;
                int lvl;
                if (a.lvl_map) {
                    lvl = (lv >> (8 * li)) & 0xFF;
                    if (lvl == 0) lvl = (side.lvl[lw - (kWinCols << g.sy)] >> (8 * li)) & 0xFF;
                } else {
                    lvl = a.levels[li];
                }
                if (lvl != 0) {
                    const int size = min(p ? 8 : 16, 1 << min(cl, pl));
                    const int cls = size == 4 ? 0 : p ? 1 : size == 8 ? 2 : 3;
                    const int at = atomicAdd(&s_count[4 + cls], 1);
                    s_list[kListTotal + c_list_off[cls] + at] =
                        seg_entry(lvl, P.height - yp, yp, off, p, cc == 0, cc == ncol - 1);
                }
            }
        }
    }
}

// The lines of one pass, filtered in one loop over its class lists laid end
// to end, so a warp changes filter code at most at a class boundary.  The
// first and last cell of an edge contribute only the lines the window needs:
// rows [py0-7, py0+th+7) / [py0-3, py0+th+3) in pass 0, columns [px0-2,
// px0+tw+2) in pass 1.  Within a pass no two edges touch a common sample, so
// the lines run in place in any order.
template <int PASS, int NT>
__device__ __forceinline__ void deblock_filter(const DbCdefArgs& a, int ssx, int ssy, uint16_t* smem,
                                               const uint32_t* s_list, const int* s_count,
                                               const PairStrength* s_str) {
    const int tid = threadIdx.x;
    const PlaneGeom gl = plane_geom(0, ssx, ssy), gc = plane_geom(1, ssx, ssy);
    // The lines, two per lane: lines 2h and 2h+1 of a segment (h = item & 1)
    // as the two halves of every register (filter_pair_class).  In pass 1
    // the first cell of an edge needs only its lines 2 and 3 and the last
    // only 0 and 1; pass 0 skips no pair: the lines the window does not need
    // there (line 0 of the first cell, line 3 of the last) are staged rows
    // that no later step reads, so filtering them changes nothing.
    const int c0 = s_count[0], c1 = s_count[1], c2 = s_count[2], c3 = s_count[3];
    const int pairs = 2 * (c0 + c1 + c2 + c3);
    for (int item = tid; item < pairs; item += NT) {
        int seg = item >> 1, cls = 0;
        const int h = item & 1;
        if (seg >= c0) {
            seg -= c0;
            cls = 1;
            if (seg >= c1) {
                seg -= c1;
                cls = 2;
                if (seg >= c2) {
                    seg -= c2;
                    cls = 3;
                }
            }
        }
        const uint32_t e = s_list[c_list_off[cls] + seg];
        const bool first = (e >> 29) & 1, last = (e >> 30) & 1;
        if (PASS == 1 && ((first && h == 0) || (last && h == 1))) continue;
        const int lvl = e & 63, nq = (e >> 6) & 15, np = (e >> 10) & 15, off = (e >> 14) & 0x1FFF, p = (e >> 27) & 3;
        const int pitch = p ? gc.pitch : gl.pitch;
        uint16_t* q = smem + a.plane_off[p] + off + (PASS == 0 ? 2 * h * pitch : 2 * h);
        const int reach = class_reach(cls);
        if (nq >= reach && np >= reach) {
            filter_pair_class<PASS>(cls, q, pitch, s_str[lvl], a.bit_depth - 8);
        } else {
            // near the plane edge: line by line, with clamped reads and
            // dropped writes
            const Strength s = strength_of(lvl, a.sharpness);
            for (int l = 0; l < 2; ++l) {
                if (PASS == 0)
                    filter_line_class<1>(cls, q + l * pitch, 1, nq, np, s, a.bit_depth);
                else
                    filter_line_class<0>(cls, q + l, pitch, nq, np, s, a.bit_depth);
            }
        }
    }
    __syncthreads();
}

// One 64x64 filter block (tile_x, tile_y) of one frame.  Every thread of the
// CTA calls it; it ends with all threads past their last shared-memory use
// only after the caller's next __syncthreads().
template <int NT, int LAYOUT, bool DIRECT = false>
__device__ __forceinline__ void dbcdef_tile(const DbCdefArgs& a, int tile_x, int tile_y) {
    constexpr int kWarpsNT = NT / 32;
    // chroma subsampling: LAYOUT = ssx | ssy << 1 fixes it at compile time
    // (every plane geometry below becomes a constant); LAYOUT < 0 reads it
    const int ssx = LAYOUT < 0 ? a.ssx : (LAYOUT & 1), ssy = LAYOUT < 0 ? a.ssy : (LAYOUT >> 1);
    extern __shared__ __align__(16) uint16_t smem[];
    __shared__ int s_cost[64][8];
    __shared__ PairBlock s_pair[3][64];
    __shared__ uint8_t s_active[64];
    __shared__ int s_count[8];  // list lengths per size class, pass 0 then pass 1
    __shared__ PairStrength s_str[64];  // per loop-filter level, for this frame's sharpness and depth
    // The deblocking lists and side window are dead once deblocking is done;
    // the CDEF phase reuses their space for the odd-aligned luma pairs.
    __shared__ union {
        struct {
            uint32_t list[2 * kListTotal];  // per pass and size class, see seg_entry()
            SideWindow side;
        } db;
        uint32_t shifted[kShiftRows * (64 + 2 * kHalo) / 2];
    } s_u;
    uint32_t* s_list = s_u.db.list;
    SideWindow& s_side = s_u.db.side;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int mi_r0 = tile_y * 16, mi_c0 = tile_x * 16;
    const int x0 = mi_c0 * 4, y0 = mi_r0 * 4;

    // ---- CDEF block activity (decode.rs:772-779)
    const long slot = (long)(mi_r0 >> 4) * a.cdef_stride + (mi_c0 >> 4);
    const int index = (a.cdef_on && slot < a.cdef_count) ? __ldg(a.cdef_idx + slot) : -1;
    bool act = false;
    if (tid < 64) {
        const int r = mi_r0 + (tid >> 3) * 2, c = mi_c0 + (tid & 7) * 2;
        if (r < a.mi_rows && c < a.mi_cols && index >= 0) {
            auto sk = [&](int rr, int cc) {
                return rr < a.mi_rows && cc < a.mi_cols && a.skip[(long)rr * a.mi_cols + cc] != 0;
            };
            act = !(sk(r, c) && sk(r + 1, c) && sk(r, c + 1) && sk(r + 1, c + 1));
        }
        s_active[tid] = act;
    }

    // the deblocking lists' lengths and strengths, published by the staging
    // barrier below
    if (tid < 8) s_count[tid] = 0;
    if (a.deblock_on && tid < 64) s_str[tid] = pair_strength(strength_of(tid, a.sharpness), a.bit_depth - 8);

    // ---- every plane's tile with an 8-sample halo (edge-clamped).  Whole
    // 16-byte chunks inside the plane go by cp.async, all in flight at once;
    // chunks that straddle the left/right plane edge are gathered sample by
    // sample.  Rows past the top/bottom edge repeat the edge row.  (Staging
    // interior tiles with 2-D tensor copies instead measured 1.4 % slower
    // for the whole chain: the extra path costs more than the copies save.)
    for (int p = 0; p < a.num_planes; ++p) {
        const PlaneGeom g = plane_geom(p, ssx, ssy);
        const DevPlaneC& P = a.src[p];
        uint16_t* t = smem + a.plane_off[p];
        const int px0 = x0 >> g.sx, py0 = y0 >> g.sy;
        const int vpr = g.pitch / 8;
        const unsigned mv = small_div_magic(vpr);
        for (int v = tid; v < g.rows * vpr; v += NT) {
            const int r = small_div(v, mv), cv = v - r * vpr;
            const int y = clampi(py0 - kHalo + r, 0, P.height - 1);
            const int x = px0 - kHalo + cv * 8;
            const uint16_t* row = P.data + (long)y * P.stride;
            uint16_t* d = t + r * g.pitch + cv * 8;
            if (a.vec_ok && x >= 0 && x + 8 <= P.width) {
                const unsigned dst = (unsigned)__cvta_generic_to_shared(d);
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(row + x) : "memory");
            } else {
#pragma unroll
                for (int k = 0; k < 8; ++k) d[k] = __ldg(row + clampi(x + k, 0, P.width - 1));
            }
        }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");

    // ---- the side information the deblocking decisions read, while the
    // copies are in flight (cells the two passes touch; see SideWindow)
    {
        const int crows = (a.mi_rows + ssy) >> ssy, ccols = (a.mi_cols + ssx) >> ssx;
        const int cr0 = (mi_r0 >> ssy) - kWinTop, cc0 = (mi_c0 >> ssx) - kWinLeft;
        for (int i = tid; i < kWinCells; i += NT) {
            const int wr = i / kWinCols, wc = i - wr * kWinCols;
            const int r = mi_r0 - kWinTop + wr, c = mi_c0 - kWinLeft + wc;
            if (r >= 0 && c >= 0 && r < a.mi_rows && c < a.mi_cols) {
                const long cell = (long)r * a.mi_cols + c;
                s_side.tx[0][i] = __ldg(a.tx_luma + cell);
                if (a.lvl_map) s_side.lvl[i] = __ldg(reinterpret_cast<const uint32_t*>(a.lvl_map) + cell);
            }
            if (a.num_planes > 1 && cr0 + wr >= 0 && cc0 + wc >= 0 && cr0 + wr < crows && cc0 + wc < ccols)
                s_side.tx[1][i] = __ldg(a.tx_chroma + (long)(cr0 + wr) * ccols + cc0 + wc);
        }
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    const bool any_active = __syncthreads_or(act);

    // ---- input checks from shared memory: the tile's own cells (transform
    // sizes, levels) and the tile's own samples
    {
        int bad = 0;
        for (int i = tid; i < 256; i += NT) {
            const int r = mi_r0 + (i >> 4), c = mi_c0 + (i & 15);
            if (r < a.mi_rows && c < a.mi_cols) {
                const int w = (i >> 4) + kWinTop, wc = (i & 15) + kWinLeft;
                bad |= s_side.tx[0][w * kWinCols + wc] > 18;
                if (a.lvl_map) {
                    const uint32_t v = s_side.lvl[w * kWinCols + wc];
                    bad |= ((v & 0xFF) > 63) | (((v >> 8) & 0xFF) > 63) | (((v >> 16) & 0xFF) > 63) | ((v >> 24) > 63);
                }
            }
        }
        if (a.num_planes > 1) {
            const int ccols = (a.mi_cols + ssx) >> ssx, crows = (a.mi_rows + ssy) >> ssy;
            const int cw = 16 >> ssx, ch = 16 >> ssy;
            for (int i = tid; i < cw * ch; i += NT) {
                const int dr = i >> (4 - ssx), dc = i - dr * cw;  // cw = 16 >> ssx
                const int r = (mi_r0 >> ssy) + dr, c = (mi_c0 >> ssx) + dc;
                if (r < crows && c < ccols) bad |= s_side.tx[1][(dr + kWinTop) * kWinCols + dc + kWinLeft] > 18;
            }
        }
        if (bad) report_error(a.status, STAGE_DEBLOCK, 0, VACO_AV1_MSG_DB_PARAMS);
    }
    {
        // Every staged sample, halo included: the halo holds samples of the
        // same planes (edge-clamped copies past their borders), so the tiles
        // together check exactly the planes' samples, and a flat pass over
        // the staged vectors needs no per-row indexing.
        const uint32_t hi = ((0xFFFFu << a.bit_depth) & 0xFFFFu) * 0x10001u;  // bits above the depth, per lane
        const uint4* v = reinterpret_cast<const uint4*>(smem);
        uint32_t acc = 0;
        for (int i = tid; i < a.staged_vectors; i += NT) {
            const uint4 w = v[i];
            acc |= w.x | w.y | w.z | w.w;
        }
        if (acc & hi) report_error(a.status, STAGE_DEBLOCK, 1, VACO_AV1_MSG_DB_SAMPLE);
    }

    // ---- deblocking, pass 0 (vertical edges) then pass 1 (horizontal edges)
    if (a.deblock_on) {
        deblock_lists<NT>(a, ssx, ssy, x0, y0, s_side, s_list, s_count);
        __syncthreads();
        deblock_filter<0, NT>(a, ssx, ssy, smem, s_list, s_count, s_str);
        deblock_filter<1, NT>(a, ssx, ssy, smem, s_list + kListTotal, s_count + 4, s_str);
    }

    // ---- stripe-boundary rows of the deblocked picture for restoration:
    // rows y with (y + offset + 2) mod stripe < 4, stored at 4*boundary + that
    // remainder (boundary = (y + offset + 2) / stripe >= 1).
    for (int p = 0; p < a.num_planes; ++p) {
        const DevPlane& R = a.pre_rows[p];
        if (!R.data) continue;
        const PlaneGeom g = plane_geom(p, ssx, ssy);
        const int sh = 64 >> g.sy, off = 8 >> g.sy;
        const int px0 = x0 >> g.sx, py0 = y0 >> g.sy;
        const uint16_t* src = smem + a.plane_off[p];
        const int width = a.dst[p].width, height = a.dst[p].height;
        // the tile (th rows, th a multiple of the stripe height or half of it)
        // holds boundary rows y = k*sh - off - 2 + sub, sub < 4
        const int lsh = 6 - g.sy;  // log2 of the stripe height
        for (int i = warp; i < 4 * ((g.th >> lsh) + 1); i += kWarpsNT) {
            const int kk = i >> 2, sub = i & 3;
            const int kb = ((py0 + off + 2) >> lsh) + kk;
            const int y = kb * sh - off - 2 + sub;
            if (kb < 1 || y < py0 || y >= py0 + g.th || y >= height) continue;
            for (int c = lane; c < g.tw; c += 32)
                if (px0 + c < width)
                    R.data[(long)(4 * kb + sub) * R.stride + px0 + c] = src[(y - py0 + kHalo) * g.pitch + c + kHalo];
        }
    }

    // ---- CDEF on the deblocked tile
    if (!any_active) {
        // Nothing filtered (or CDEF off): the output is the deblocked tile.
        for (int p = 0; p < a.num_planes; ++p) {
            const PlaneGeom g = plane_geom(p, ssx, ssy);
            const DevPlane& d = a.dst[p];
            const int px0 = x0 >> g.sx, py0 = y0 >> g.sy;
            const DirectPlane* D = DIRECT ? &a.direct[p] : nullptr;
            const uint16_t* t = smem + a.plane_off[p];
            for (int r = warp; r < g.th; r += kWarpsNT) {
                const int y = py0 + r;
                if (y >= d.height) break;
                for (int c = lane; c < g.tw; c += 32) {
                    const int x = px0 + c;
                    if (x >= d.width) continue;
                    const uint16_t v = t[(r + kHalo) * g.pitch + c + kHalo];
                    d.data[(long)y * d.stride + x] = v;
                    // the final output too, for a plane without restoration
                    if (D && D->out.data && y < D->out.height && x < D->out.width)
                        D->out.data[(long)y * D->out.stride + x] = v;
                }
            }
        }
        return;
    }
    // Samples outside the plane become the "unavailable" sentinel for CDEF.
    for (int p = 0; p < a.num_planes; ++p) {
        const PlaneGeom g = plane_geom(p, ssx, ssy);
        const DevPlane& d = a.dst[p];
        const int px0 = x0 >> g.sx, py0 = y0 >> g.sy;
        if (px0 + g.tw + 2 <= d.width && py0 + g.th + 2 <= d.height && px0 >= 2 && py0 >= 2) continue;
        uint16_t* t = smem + a.plane_off[p];
        const int wr = g.th + 4, wc = g.tw + 4;
        const unsigned mw = small_div_magic(wc);
        for (int i = tid; i < wr * wc; i += NT) {
            const int r = small_div(i, mw), c = i - r * wc;
            const int y = py0 - 2 + r, x = px0 - 2 + c;
            if (y < 0 || x < 0 || y >= d.height || x >= d.width)
                t[(r + kHalo - 2) * g.pitch + (c + kHalo - 2)] = (uint16_t)kSent;
        }
    }
    __syncthreads();

    // The luma CDEF window's pairs that start on odd samples (rows kHalo-2 ..
    // kHalo+th+1, first samples on columns kHalo-1 .. kHalo+tw-1), as words
    // on the staged row pitch, so the pair filter reads every luma tap with
    // one aligned load.
    {
        constexpr int WP = (64 + 2 * kHalo) / 2, W0 = (kHalo - 1) / 2, NW = 64 / 2 + 1;
        const uint32_t* t32 = reinterpret_cast<const uint32_t*>(smem + a.plane_off[0]);
        for (int i = tid; i < kShiftRows * NW; i += NT) {
            const int r = i / NW, w = W0 + (i - r * NW);
            const int src = (kHalo - 2 + r) * WP + w;
            s_u.shifted[r * WP + w] = __byte_perm(t32[src], t32[src + 1], 0x5432);
        }
    }

    // Direction search: job j (0..7, spread over the warps) handles direction
    // pair (j & 3) for blocks (j >> 2)*32 + lane (warp-uniform branches).
    const int lpitch = 64 + 2 * kHalo;
    for (int job = warp; job < 8; job += kWarpsNT) {
        const int pair = job & 3, b = ((job >> 2) << 5) + lane;
        if (s_active[b]) {
            const uint16_t* blk = smem + a.plane_off[0] + (kHalo + (b >> 3) * 8) * lpitch + kHalo + (b & 7) * 8;
            int lo, hi;
            dir_costs_pair(pair, blk, lpitch, a.shift, lo, hi);
            s_cost[b][pair] = lo;
            s_cost[b][pair + 4] = hi;
        }
    }
    __syncthreads();
    // Per block and plane (one thread each): direction, strengths, checks.
    for (int i = tid; i < 64 * a.num_planes; i += NT) {
        if (!s_active[i & 63]) continue;
        const int b = i & 63, p = i >> 6;
        int dir;
        uint32_t var;
        best_direction(s_cost[b], dir, var);
        const bool chroma = p != 0;
        int sp = 0, ss = 0;
        if (index < 8) {
            sp = chroma ? a.uv_pri[index] : a.y_pri[index];
            ss = chroma ? a.uv_sec[index] : a.y_sec[index];
        }
        int primary = (sp << a.shift) & 0xFFFF;
        const int secondary = (ss << a.shift) & 0xFFFF;
        const int chosen = primary == 0 ? 0 : chroma ? chroma_direction(dir, ssx, ssy) : dir;
        if (!chroma) primary = adjust_strength(primary, var);
        const int damping = (a.damping + a.shift - (chroma ? 1 : 0)) & 0xFF;
        // Each plane reports its own failure; the status word keeps the
        // lowest (block, plane) key, i.e. the first plane vaco would reject.
        if (index >= 8 || damping > 12 || primary > (15 << a.shift) || secondary > (4 << a.shift)) {
            const int r = mi_r0 + (b >> 3) * 2, c = mi_c0 + (b & 7) * 2;
            report_error(a.status, STAGE_CDEF, ((unsigned long long)r * a.mi_cols + c) * 4 + 1 + p,
                         index >= 8 ? VACO_AV1_MSG_CDEF_STRENGTH_INDEX : VACO_AV1_MSG_CDEF_BLOCK_PARAMS);
        }
        const PlaneGeom g = plane_geom(p, ssx, ssy);
        s_pair[p][b] = make_pair_block(chosen, primary, secondary, min(damping, 12), a.shift, g.pitch);
    }
    __syncthreads();

    // Filtering: pixel pairs (two 16-bit lanes per register), one warp per
    // block row, lanes across the tile width.
    for (int p = 0; p < a.num_planes; ++p) {
        const PlaneGeom g = plane_geom(p, ssx, ssy);
        const DevPlane& d = a.dst[p];
        const int px0 = x0 >> g.sx, py0 = y0 >> g.sy;
        const bool edge = px0 < 2 || py0 < 2 || px0 + g.tw + 2 > d.width || py0 + g.th + 2 > d.height;
        const uint16_t* tp = smem + a.plane_off[p];
        // the tile's tap sets, from its preset (uniform over the tile)
        bool pri_on = true, sec_on = true;
        if (index < 8) {
            pri_on = (p ? a.uv_pri[index] : a.y_pri[index]) != 0;
            sec_on = (p ? a.uv_sec[index] : a.y_sec[index]) != 0;
        }
        // tile layouts: 64x64 (luma, 4:4:4 chroma), 32x32 (4:2:0), 32x64 (4:2:2)
        if (p == 0) {
            filter_pairs_edge<64 + 2 * kHalo, 8, 1, true>(edge, tp, s_u.shifted, d, DIRECT ? &a.direct[p] : nullptr, px0, py0, g.tw, s_active,
                                                          s_pair[p], pri_on, sec_on, warp, lane, g.sx, kWarpsNT);
        } else if (g.tw == 64) {
            filter_pairs_edge<64 + 2 * kHalo, 8, 1, false>(edge, tp, nullptr, d, DIRECT ? &a.direct[p] : nullptr, px0, py0, g.tw, s_active, s_pair[p],
                                                           pri_on, sec_on, warp, lane, g.sx, kWarpsNT);
        } else if (g.th == 32) {
            filter_pairs_edge<32 + 2 * kHalo, 4, 2, false>(edge, tp, nullptr, d, DIRECT ? &a.direct[p] : nullptr, px0, py0, g.tw, s_active, s_pair[p],
                                                           pri_on, sec_on, warp, lane, g.sx, kWarpsNT);
        } else {
            filter_pairs_edge<32 + 2 * kHalo, 8, 2, false>(edge, tp, nullptr, d, DIRECT ? &a.direct[p] : nullptr, px0, py0, g.tw, s_active, s_pair[p],
                                                           pri_on, sec_on, warp, lane, g.sx, kWarpsNT);
        }
    }
}

// NT threads per tile, MIN_CTAS CTAs per SM.  The per-frame path runs 256
// threads at 4 CTAs per SM (64 registers a thread), measured at least as fast
// as 3 (80 registers) on 1080p and on 2560-, 2880- and 3840-wide frames
// (1.5-2 % faster on the last two); 128 threads at 5 CTAs
// per SM is the smaller-CTA shape (shorter barriers, about the same warps per
// SM).  The batched form also has the 256 x 3 body (see dbcdef_batch_kernel).
// DIRECT: a body that also writes the output of planes without restoration
// (DirectPlane); the code for it measured 3 % slower on frames that have no
// such plane, so it is a separate body.
template <int NT, int MIN_CTAS, int LAYOUT, bool DIRECT = false>
__global__ void __launch_bounds__(NT, MIN_CTAS) dbcdef_kernel(DbCdefArgs a) {
    overlap_prologue();
    dbcdef_tile<NT, LAYOUT, DIRECT>(a, blockIdx.x, blockIdx.y);
}

// Batched form: one CTA per tile of all frames of a batch, frames laid end to
// end in `tile_prefix` order, so frames of any size share one launch and the
// hardware hands out the tiles in that order.  MIN_CTAS as for dbcdef_kernel.
// (A persistent form, CTAs taking tiles from a device queue, kept its loop
// state and the frame record live across the tile and spilled registers: it
// measured 4 % slower on 4K frames.)  LAYOUT as for dbcdef_tile: a batch
// whose frames share one chroma layout takes the body compiled for it.
template <int NT, int MIN_CTAS, int LAYOUT>
__global__ void __launch_bounds__(NT, MIN_CTAS) dbcdef_batch_kernel(const DbCdefArgs* __restrict__ frames,
                                                                    const int* __restrict__ tile_prefix, int n) {
    const int f = frame_of_tile(tile_prefix, n, blockIdx.x);
    const DbCdefArgs& a = frames[f];
    const int local = blockIdx.x - tile_prefix[f];
    const int tiles_x = (a.mi_cols + 15) / 16;
    dbcdef_tile<NT, LAYOUT>(a, local % tiles_x, local / tiles_x);
}

}  // namespace

size_t dbcdef_args_size() { return sizeof(DbCdefArgs); }

// Kernel arguments of one frame; returns the dynamic shared memory it needs.
size_t build_dbcdef_args(const DbCdefLaunch& L, void* out) {
    DbCdefArgs a;
    memset(&a, 0, sizeof a);
    const int np = L.info.monochrome ? 1 : 3;
    bool vec = true;
    size_t off = 0;
    for (int p = 0; p < 3; ++p) {
        a.src[p] = DevPlaneC{L.src.planes[p], L.src.width[p], L.src.height[p], L.src.stride[p]};
        a.dst[p] = DevPlane{L.dst.planes[p], L.dst.width[p], L.dst.height[p], L.dst.stride[p]};
        a.pre_rows[p] = L.pre_rows[p];
        a.plane_off[p] = off;
        if (p < np) {
            vec = vec && (L.src.stride[p] % 8 == 0) && ((uintptr_t)L.src.planes[p] % 16 == 0);
            const int sx = p ? L.info.subsampling_x : 0, sy = p ? L.info.subsampling_y : 0;
            off += (size_t)((64 >> sx) + 2 * kHalo) * ((64 >> sy) + 2 * kHalo);
        }
    }
    a.num_planes = np;
    a.ssx = np > 1 ? L.info.subsampling_x : 0;
    a.ssy = np > 1 ? L.info.subsampling_y : 0;
    a.bit_depth = L.info.bit_depth;
    a.shift = L.info.bit_depth - 8;
    a.mi_rows = L.info.mi_rows;
    a.mi_cols = L.info.mi_cols;
    a.coded_width = L.info.coded_width;
    a.coded_height = L.info.coded_height;
    a.tx_luma = L.tx_luma;
    a.tx_chroma = L.tx_chroma;
    a.lvl_map = L.lvl_map;
    for (int k = 0; k < 4; ++k) a.levels[k] = L.deblock.levels[k];
    a.sharpness = L.deblock.sharpness;
    a.deblock_on = !(L.deblock.levels[0] == 0 && L.deblock.levels[1] == 0);
    bool all_zero = true;
    for (int k = 0; k < 8; ++k)
        all_zero = all_zero && L.cdef.y_primary[k] == 0 && L.cdef.y_secondary[k] == 0 && L.cdef.uv_primary[k] == 0 &&
                   L.cdef.uv_secondary[k] == 0;
    a.cdef_on = L.cdef.enabled && !all_zero && L.skip != nullptr;
    a.skip = L.skip;
    a.cdef_idx = L.cdef_idx;
    a.cdef_stride = L.cdef_stride;
    a.cdef_count = L.cdef_idx ? L.cdef_count : 0;
    a.damping = L.cdef.damping;
    for (int k = 0; k < 8; ++k) {
        a.y_pri[k] = L.cdef.y_primary[k];
        a.y_sec[k] = L.cdef.y_secondary[k];
        a.uv_pri[k] = L.cdef.uv_primary[k];
        a.uv_sec[k] = L.cdef.uv_secondary[k];
    }
    a.status = L.status;
    a.vec_ok = vec;
    a.staged_vectors = (int)(off / 8);  // each staged plane is a multiple of 8 samples
    for (int p = 0; p < 3; ++p) a.direct[p] = p < np ? L.direct[p] : DirectPlane{};
    memcpy(out, &a, sizeof a);
    return off * sizeof(uint16_t);
}

// Per-device cache, shared by every host thread that launches: an atomic, so
// concurrent first launches on a device only repeat idempotent set-up.
std::atomic<unsigned long long> g_attr_devices{0};

cudaError_t dbcdef_kernel_attributes() {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !(g_attr_devices.load(std::memory_order_acquire) & (1ull << dev))) {
        constexpr int kMaxSmem = 96 * 1024;
        const cudaFuncAttribute attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
        cudaError_t e = cudaSuccess;
        for (auto k : {dbcdef_kernel<256, 4, 0>, dbcdef_kernel<256, 4, 1>, dbcdef_kernel<256, 4, 3>,
                       dbcdef_kernel<256, 4, 0, true>, dbcdef_kernel<256, 4, 1, true>,
                       dbcdef_kernel<256, 4, 3, true>, dbcdef_kernel<128, 5, 0>, dbcdef_kernel<128, 5, 1>,
                       dbcdef_kernel<128, 5, 3>})
            if (e == cudaSuccess) e = cudaFuncSetAttribute(k, attr, kMaxSmem);
        for (auto k : {dbcdef_batch_kernel<256, 3, -1>, dbcdef_batch_kernel<256, 3, 0>, dbcdef_batch_kernel<256, 3, 1>,
                       dbcdef_batch_kernel<256, 3, 3>, dbcdef_batch_kernel<256, 4, -1>, dbcdef_batch_kernel<128, 5, -1>})
            if (e == cudaSuccess) e = cudaFuncSetAttribute(k, attr, kMaxSmem);
        if (e != cudaSuccess) return e;
        g_attr_devices.fetch_or(1ull << dev, std::memory_order_release);
    }
    return cudaSuccess;
}

cudaError_t launch_dbcdef(const DbCdefLaunch& L, cudaStream_t stream) {
    DbCdefArgs a;
    const size_t smem = build_dbcdef_args(L, &a);
    cudaError_t e = dbcdef_kernel_attributes();
    if (e != cudaSuccess) return e;
    dim3 grid(div_up(L.info.mi_cols, 16), div_up(L.info.mi_rows, 16));
    // one kernel per chroma layout (4:4:4 and monochrome, 4:2:2, 4:2:0); a
    // frame with a plane written straight to the output takes the 256-thread
    // body that does so, whatever the threads per tile
    const int layout = a.ssx | a.ssy << 1;
    if (a.direct[0].out.data || a.direct[1].out.data || a.direct[2].out.data) {
        auto k = layout == 3   ? dbcdef_kernel<256, 4, 3, true>
                 : layout == 1 ? dbcdef_kernel<256, 4, 1, true>
                               : dbcdef_kernel<256, 4, 0, true>;
        return launch_overlapped(k, grid, dim3(256), smem, stream, a);
    }
    if (L.threads == 128) {
        auto k = layout == 3 ? dbcdef_kernel<128, 5, 3> : layout == 1 ? dbcdef_kernel<128, 5, 1> : dbcdef_kernel<128, 5, 0>;
        return launch_overlapped(k, grid, dim3(128), smem, stream, a);
    }
    auto k = layout == 3 ? dbcdef_kernel<256, 4, 3> : layout == 1 ? dbcdef_kernel<256, 4, 1> : dbcdef_kernel<256, 4, 0>;
    return launch_overlapped(k, grid, dim3(256), smem, stream, a);
}

cudaError_t launch_dbcdef_batch(const void* dev_args, const int* dev_prefix, int n, int tiles, size_t smem,
                                int ctas_per_sm, int threads, int layout, cudaStream_t stream) {
    if (tiles <= 0) return cudaSuccess;
    cudaError_t e = dbcdef_kernel_attributes();
    if (e != cudaSuccess) return e;
    const DbCdefArgs* args = static_cast<const DbCdefArgs*>(dev_args);
    using K = void (*)(const DbCdefArgs*, const int*, int);
    K k;
    if (threads == 128) {
        k = dbcdef_batch_kernel<128, 5, -1>;
    } else if (ctas_per_sm <= 3) {  // up to 3 resident: the 80-register body
        k = layout == 3 ? dbcdef_batch_kernel<256, 3, 3> : layout == 1 ? dbcdef_batch_kernel<256, 3, 1>
          : layout == 0 ? dbcdef_batch_kernel<256, 3, 0> : dbcdef_batch_kernel<256, 3, -1>;
    } else {  // 64 registers: the layout-specialised bodies would spill
        k = dbcdef_batch_kernel<256, 4, -1>;
    }
    k<<<tiles, threads == 128 ? 128 : 256, smem, stream>>>(args, dev_prefix, n);
    return cudaGetLastError();
}

}  // namespace vaco
