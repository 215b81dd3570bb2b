// batch.cu -- the batched form of the post-filter chain.
//
// vaco filters one frame per decode_frame call (crates/codec/vaco-codec-av1/
// src/decode.rs:553-559).  Here a batch of frames of any sizes and bit depths
// shares one launch set:
//   1. one upload of the per-batch tables (frame argument records, tile
//      prefix sums, initial status words)
//   2. one deblock+CDEF kernel with one CTA per tile of all frames
//      (dbcdef.cu)
//   3. superres launches for the frames that upscale
//   4. one restoration kernel over all frames' tiles (restoration.cu), which
//      also validates every restoration unit and copies planes whose
//      frame-level restoration is off
//   5. one download of the per-frame status words
// With tuning.use_graphs, steps 1-5 are captured once per batch composition as
// a CUDA graph and replayed afterwards; the tables carry every per-batch
// pointer, so a replay only needs the host to refresh the pinned staging copy.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "common.cuh"
#include "ctx.cuh"
#include "kernels.cuh"

using namespace vaco;

namespace {

unsigned long long key_of(unsigned stage, unsigned long long position, unsigned msg) {
    return ((unsigned long long)stage << 60) | ((position & ((1ull << 52) - 1)) << 8) | msg;
}

bool depth_ok(int bd) { return bd == 8 || bd == 10 || bd == 12; }

bool geometry_ok(const vaco_av1_frame_job& j) {
    const vaco_av1_frame_info& i = j.info;
    if (i.mi_rows <= 0 || i.mi_cols <= 0 || i.mi_rows > (1 << 15) || i.mi_cols > (1 << 15)) return false;
    if (!av1_subsampling_ok(i.subsampling_x, i.subsampling_y)) return false;
    if (i.coded_width <= 0 || i.coded_height <= 0) return false;
    if (i.mi_cols != 2 * ((i.coded_width + 7) >> 3) || i.mi_rows != 2 * ((i.coded_height + 7) >> 3)) return false;
    if (i.upscaled_width < i.coded_width) return false;
    const int np = i.monochrome ? 1 : 3;
    if (np > 1 && ((i.subsampling_x && ((i.coded_width | i.upscaled_width) & 1)) ||
                   (i.subsampling_y && (i.coded_height & 1))))
        return false;
    for (int k = 0; k < np; ++k) {
        const int sx = k ? i.subsampling_x : 0, sy = k ? i.subsampling_y : 0;
        if (!j.src.planes[k] || j.src.width[k] != (i.mi_cols * 4) >> sx || j.src.height[k] != (i.mi_rows * 4) >> sy ||
            j.src.stride[k] < j.src.width[k])
            return false;
        if (!j.dst.planes[k] || j.dst.width[k] != (i.upscaled_width >> sx) || j.dst.height[k] != (i.coded_height >> sy) ||
            j.dst.stride[k] < j.dst.width[k])
            return false;
    }
    return true;
}

struct PlaneBuf {
    size_t off;  // arena byte offset
    int w, h, pitch;
};

struct FramePlan {
    int index;
    bool run_db = false, run_lr = false, superres = false, lr_active = false;
    unsigned long long host_key = kNoError;
    PlaneBuf cdef[3], rows[3], ucdef[3], urows[3];
    PlaneBuf deb[3], udeb[3];  // unfused stages: the whole deblocked picture (and its upscaled copy)
    int np = 0, tiles_db = 0;
    long long pixels = 0;
};

struct Arena {
    size_t used = 0;
    PlaneBuf take(int w, int h) {
        PlaneBuf b;
        b.w = w;
        b.h = h;
        b.pitch = (int)align_up((size_t)(w > 0 ? w : 1), 64);
        b.off = used;
        used += align_up((size_t)b.pitch * (size_t)(h > 0 ? h : 1) * 2, 256);
        return b;
    }
};

DevPlane dev_plane(unsigned char* base, const PlaneBuf& b) {
    return DevPlane{reinterpret_cast<uint16_t*>(base + b.off), b.w, b.h, b.pitch};
}
DevPlaneC dev_cplane(unsigned char* base, const PlaneBuf& b) {
    return DevPlaneC{reinterpret_cast<const uint16_t*>(base + b.off), b.w, b.h, b.pitch};
}

int32_t fail(vaco_av1_ctx* ctx, cudaError_t e, int32_t* statuses, int32_t* msgs, int n) {
    ctx->last_cuda_error = (int)e;
    for (int i = 0; i < n; ++i) {
        if (statuses) statuses[i] = VACO_AV1_DEVICE_ERROR;
        if (msgs) msgs[i] = VACO_AV1_MSG_CUDA;
    }
    return VACO_AV1_DEVICE_ERROR;
}

// Deblocking and CDEF of one frame as separate kernels (the unfused stage
// choice): copy with checks into the frame's deblocked picture, both passes
// in place, then CDEF into its CDEF picture (a copy when CDEF is off, as
// apply_cdef leaves the picture alone).
cudaError_t enqueue_unfused(const vaco_av1_frame_job& J, const FramePlan& F, unsigned char* base, DeviceStatus* status,
                            cudaStream_t s) {
    const vaco_av1_frame_info& info = J.info;
    const int ssx = info.subsampling_x, ssy = info.subsampling_y;
    DevPlaneC sp[3];
    DevPlane deb[3];
    for (int k = 0; k < F.np; ++k) {
        sp[k] = DevPlaneC{J.src.planes[k], J.src.width[k], J.src.height[k], J.src.stride[k]};
        deb[k] = dev_plane(base, F.deb[k]);
    }
    const long n_luma = (long)info.mi_rows * info.mi_cols;
    const long n_chroma = F.np > 1 ? (long)((info.mi_rows + ssy) >> ssy) * ((info.mi_cols + ssx) >> ssx) : 0;
    cudaError_t e = launch_deblock_prepare(sp, deb, F.np, info.bit_depth, J.tx_luma, n_luma, J.tx_chroma, n_chroma,
                                           J.lvl_map, status, s);
    if (e != cudaSuccess) return e;
    DeblockLaunch L;
    for (int k = 0; k < 3; ++k) L.pic[k] = k < F.np ? deb[k] : DevPlane{nullptr, 0, 0, 0};
    L.num_planes = F.np;
    L.ssx = ssx;
    L.ssy = ssy;
    L.bit_depth = info.bit_depth;
    L.mi_rows = info.mi_rows;
    L.mi_cols = info.mi_cols;
    L.coded_width = info.coded_width;
    L.coded_height = info.coded_height;
    L.tx_luma = J.tx_luma;
    L.tx_chroma = J.tx_chroma;
    L.lvl_map = J.lvl_map;
    for (int k = 0; k < 4; ++k) L.levels[k] = J.deblock.levels[k];
    L.sharpness = J.deblock.sharpness;
    e = launch_deblock_passes(L, s);
    if (e != cudaSuccess) return e;
    vaco_av1_picture deb_pic{}, cdef_pic{};
    for (int k = 0; k < F.np; ++k) {
        const DevPlane c = dev_plane(base, F.cdef[k]);
        deb_pic.planes[k] = deb[k].data;
        deb_pic.width[k] = deb[k].width;
        deb_pic.height[k] = deb[k].height;
        deb_pic.stride[k] = deb[k].stride;
        cdef_pic.planes[k] = c.data;
        cdef_pic.width[k] = c.width;
        cdef_pic.height[k] = c.height;
        cdef_pic.stride[k] = c.stride;
    }
    bool all_zero = true;
    for (int k = 0; k < 8; ++k)
        all_zero = all_zero && J.cdef.y_primary[k] == 0 && J.cdef.y_secondary[k] == 0 && J.cdef.uv_primary[k] == 0 &&
                   J.cdef.uv_secondary[k] == 0;
    if (!J.cdef.enabled || all_zero) {
        for (int k = 0; k < F.np && e == cudaSuccess; ++k)
            e = cudaMemcpy2DAsync(cdef_pic.planes[k], (size_t)cdef_pic.stride[k] * 2, deb_pic.planes[k],
                                  (size_t)deb_pic.stride[k] * 2, (size_t)deb_pic.width[k] * 2, deb_pic.height[k],
                                  cudaMemcpyDeviceToDevice, s);
        return e;
    }
    CdefLaunch C;
    C.src = deb_pic;
    C.dst = cdef_pic;
    C.info = info;
    C.skip = J.skip;
    C.cdef_idx = J.cdef_idx;
    C.cdef_stride = J.cdef_stride;
    C.cdef_count = J.cdef_idx ? J.cdef_count : 0;
    C.params = J.cdef;
    C.status = status;
    return launch_cdef_frame(C, s);
}

}  // namespace

extern "C" int32_t vaco_av1_ctx_set_tuning(vaco_av1_ctx* ctx, const vaco_av1_tuning* t) {
    if (!ctx || !t) return VACO_AV1_INVALID_DATA;
    if (t->dbcdef_ctas_per_sm < 1 || t->dbcdef_ctas_per_sm > 8 || t->lr_ctas_per_sm < 1 || t->lr_ctas_per_sm > 8 ||
        !(t->dbcdef_threads == 0 || t->dbcdef_threads == 128 || t->dbcdef_threads == 256) ||
        t->stage_fusion < 0 || t->stage_fusion > 1)
        return VACO_AV1_INVALID_DATA;
    ctx->tuning = *t;
    return VACO_AV1_OK;
}

extern "C" int32_t vaco_av1_ctx_get_tuning(const vaco_av1_ctx* ctx, vaco_av1_tuning* t) {
    if (!ctx || !t) return VACO_AV1_INVALID_DATA;
    *t = ctx->tuning;
    return VACO_AV1_OK;
}

// Enqueues the whole batch on `s` without waiting; `pending` keeps what
// batch_collect() needs once the stream has passed the batch.
int32_t vaco::batch_enqueue(vaco_av1_ctx* ctx, cudaStream_t s, const vaco_av1_frame_job* jobs, int n,
                            BatchPending* pending) {
    int32_t* statuses = nullptr;
    int32_t* msgs = nullptr;
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaSuccess;
    if (!ctx->sm_count) {
        e = cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, ctx->device);
        if (e != cudaSuccess) return fail(ctx, e, statuses, msgs, n);
    }

    // Stage fusion (tuning): deblocking and CDEF in the one fused kernel, or
    // as the per-stage kernels, frame by frame, with the whole deblocked
    // picture kept for restoration.
    const bool fused = ctx->tuning.stage_fusion != 0;

    // ---- host pass: checks, scratch layout, tile counts
    std::vector<FramePlan> plan(n);
    Arena arena;
    std::string signature = std::to_string(n) + ":";
    for (int i = 0; i < n; ++i) {
        const vaco_av1_frame_job& J = jobs[i];
        FramePlan& F = plan[i];
        F.index = i;
        if (!geometry_ok(J)) {
            F.host_key = key_of(STAGE_DEBLOCK, 0, VACO_AV1_MSG_FRAME_GEOMETRY);
            signature += "x;";
            continue;
        }
        const vaco_av1_frame_info& info = J.info;
        F.np = info.monochrome ? 1 : 3;
        F.superres = info.upscaled_width != info.coded_width;
        for (int k = 0; k < F.np; ++k) F.lr_active = F.lr_active || J.lr_type[k] != VACO_AV1_FRAME_LR_NONE;
        F.pixels = (long long)info.upscaled_width * info.coded_height;
        // deblocking / CDEF host checks (as postfilter_dev_impl runs them)
        bool params_ok = depth_ok(info.bit_depth) && J.deblock.sharpness <= 7;
        for (int k = 0; k < 4; ++k) params_ok = params_ok && J.deblock.levels[k] <= 63;
        bool all_zero = true;
        for (int k = 0; k < 8; ++k)
            all_zero = all_zero && J.cdef.y_primary[k] == 0 && J.cdef.y_secondary[k] == 0 &&
                       J.cdef.uv_primary[k] == 0 && J.cdef.uv_secondary[k] == 0;
        const bool cdef_on = J.cdef.enabled && !all_zero;
        if (!params_ok || !J.tx_luma || (F.np > 1 && !J.tx_chroma))
            F.host_key = key_of(STAGE_DEBLOCK, 0, params_ok ? VACO_AV1_MSG_NULL_ARGUMENT : VACO_AV1_MSG_DB_PARAMS);
        else if (cdef_on && (!J.skip || (!J.cdef_idx && J.cdef_count > 0)))
            F.host_key = key_of(STAGE_CDEF, 0, VACO_AV1_MSG_NULL_ARGUMENT);
        F.run_db = F.host_key == kNoError;
        if (!F.run_db) {
            signature += "x;";
            continue;
        }
        // restoration host checks, plane by plane (restore_plane's order)
        F.run_lr = true;
        for (int k = 0; k < F.np && F.run_lr; ++k) {
            if (J.lr_type[k] == VACO_AV1_FRAME_LR_NONE) continue;
            const int sx = k ? info.subsampling_x : 0, sy = k ? info.subsampling_y : 0;
            const int w = info.upscaled_width >> sx, h = info.coded_height >> sy, u = J.lr_unit_size[k];
            unsigned long long key = kNoError;
            if (u == 0) {
                key = key_of(STAGE_LR, lr_key_position(k, LRC_NO_UNIT_SIZE, 0), VACO_AV1_MSG_LR_NO_UNIT_SIZE);
            } else if (!(u == 32 || u == 64 || u == 128 || u == 256)) {
                key = key_of(STAGE_LR, lr_key_position(k, LRC_GEOMETRY, 0), VACO_AV1_MSG_LR_GEOMETRY);
            } else {
                const int cols = std::max((w + u / 2) / u, 1), rows = std::max((h + u / 2) / u, 1);
                if ((long)cols * rows != J.lr_unit_count[k] || !J.lr_units[k])
                    key = key_of(STAGE_LR, lr_key_position(k, LRC_COUNT, 0),
                                 J.lr_units[k] ? VACO_AV1_MSG_LR_UNIT_COUNT : VACO_AV1_MSG_NULL_ARGUMENT);
            }
            if (key != kNoError) {
                F.host_key = key;
                F.run_lr = false;
            }
        }
        // scratch: CDEF planes, then (restoration) boundary rows, then superres copies
        for (int k = 0; k < F.np; ++k) F.cdef[k] = arena.take(J.src.width[k], J.src.height[k]);
        if (!fused)
            for (int k = 0; k < F.np; ++k) F.deb[k] = arena.take(J.src.width[k], J.src.height[k]);
        F.tiles_db = dbcdef_tiles(info);
        signature += std::to_string(info.coded_width) + "x" + std::to_string(info.coded_height) + "/" +
                     std::to_string(info.upscaled_width) + "/" + std::to_string(info.bit_depth) +
                     (info.monochrome ? "m" : "c") + std::to_string(info.subsampling_x) +
                     std::to_string(info.subsampling_y) + (F.run_lr ? "L" : "-");
        for (int k = 0; k < F.np; ++k) signature += std::to_string(J.lr_type[k]) + "," + std::to_string(J.lr_unit_size[k]);
        signature += ";";
    }
    // boundary rows (restoration's pre-CDEF source) of every frame
    for (int i = 0; i < n; ++i) {
        FramePlan& F = plan[i];
        if (!F.run_db || !F.lr_active || !fused) continue;
        for (int k = 0; k < F.np; ++k)
            F.rows[k] = arena.take(jobs[i].src.width[k], pre_rows_count(jobs[i].src.height[k], k ? jobs[i].info.subsampling_y : 0));
    }
    for (int i = 0; i < n; ++i) {
        FramePlan& F = plan[i];
        if (!F.run_db || !F.superres) continue;
        const vaco_av1_frame_info& info = jobs[i].info;
        for (int k = 0; k < F.np; ++k) {
            const int sx = k ? info.subsampling_x : 0, sy = k ? info.subsampling_y : 0;
            const int w = (info.upscaled_width + sx) >> sx, h = (info.coded_height + sy) >> sy;
            F.ucdef[k] = arena.take(w, h);
            if (F.lr_active && fused) F.urows[k] = arena.take(w, F.rows[k].h);
            if (F.lr_active && !fused) F.udeb[k] = arena.take(w, h);
        }
    }
    unsigned char* base = static_cast<unsigned char*>(ctx->scratch(S_BATCH_ARENA, arena.used));
    if (!base) return fail(ctx, cudaErrorMemoryAllocation, statuses, msgs, n);

    // ---- tile order: frames that run, largest first when tuned so
    std::vector<int> order;
    for (int i = 0; i < n; ++i)
        if (plan[i].run_db) order.push_back(i);
    if (ctx->tuning.largest_first)
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return plan[a].pixels > plan[b].pixels; });
    std::vector<int> lr_order;
    for (int i : order)
        if (plan[i].run_lr) lr_order.push_back(i);

    // ---- table layout (one buffer, 256-byte aligned sections)
    const size_t db_rec = dbcdef_args_size(), lr_rec = lr_args_size();
    size_t off = 0;
    const size_t off_status = off;
    off = align_up(off + sizeof(DeviceStatus) * n, 256);
    const size_t off_db = off;
    off = align_up(off + db_rec * order.size(), 256);
    const size_t off_db_prefix = off;
    off = align_up(off + sizeof(int) * (order.size() + 1), 256);
    const size_t off_lr = off;
    off = align_up(off + lr_rec * lr_order.size(), 256);
    const size_t off_lr_prefix = off;
    off = align_up(off + sizeof(int) * (lr_order.size() + 1), 256);
    const size_t table_bytes = off;
    unsigned char* dtab = static_cast<unsigned char*>(ctx->scratch(S_BATCH_TABLE, table_bytes));
    if (!dtab) return fail(ctx, cudaErrorMemoryAllocation, statuses, msgs, n);
    if (ctx->batch_table_host_bytes < table_bytes) {
        if (ctx->batch_table_host) cudaFreeHost(ctx->batch_table_host);
        ctx->batch_table_host = nullptr;
        ctx->batch_table_host_bytes = 0;
        e = cudaMallocHost(&ctx->batch_table_host, table_bytes);
        if (e != cudaSuccess) return fail(ctx, e, statuses, msgs, n);
        ctx->batch_table_host_bytes = table_bytes;
        ++ctx->scratch_generation;
    }
    if (ctx->batch_status_host_count < (size_t)n) {
        if (ctx->batch_status_host) cudaFreeHost(ctx->batch_status_host);
        ctx->batch_status_host = nullptr;
        ctx->batch_status_host_count = 0;
        e = cudaMallocHost(&ctx->batch_status_host, sizeof(unsigned long long) * n);
        if (e != cudaSuccess) return fail(ctx, e, statuses, msgs, n);
        ctx->batch_status_host_count = n;
        ++ctx->scratch_generation;
    }
    unsigned char* htab = ctx->batch_table_host;
    DeviceStatus* dstatus = reinterpret_cast<DeviceStatus*>(dtab + off_status);
    memset(htab + off_status, 0xFF, sizeof(DeviceStatus) * n);

    // deblock + CDEF records
    size_t smem_db = 0;
    int* db_prefix = reinterpret_cast<int*>(htab + off_db_prefix);
    db_prefix[0] = 0;
    for (size_t q = 0; q < order.size() && fused; ++q) {
        const int i = order[q];
        const FramePlan& F = plan[i];
        const vaco_av1_frame_job& J = jobs[i];
        DbCdefLaunch L;
        L.src = J.src;
        L.dst = vaco_av1_picture{};
        for (int k = 0; k < F.np; ++k) {
            const DevPlane d = dev_plane(base, F.cdef[k]);
            L.dst.planes[k] = d.data;
            L.dst.width[k] = d.width;
            L.dst.height[k] = d.height;
            L.dst.stride[k] = d.stride;
            L.pre_rows[k] = F.lr_active ? dev_plane(base, F.rows[k]) : DevPlane{nullptr, 0, 0, 0};
        }
        for (int k = F.np; k < 3; ++k) L.pre_rows[k] = DevPlane{nullptr, 0, 0, 0};
        L.info = J.info;
        L.tx_luma = J.tx_luma;
        L.tx_chroma = J.tx_chroma;
        L.lvl_map = J.lvl_map;
        L.deblock = J.deblock;
        bool all_zero = true;
        for (int k = 0; k < 8; ++k)
            all_zero = all_zero && J.cdef.y_primary[k] == 0 && J.cdef.y_secondary[k] == 0 &&
                       J.cdef.uv_primary[k] == 0 && J.cdef.uv_secondary[k] == 0;
        L.skip = (J.cdef.enabled && !all_zero) ? J.skip : nullptr;
        L.cdef_idx = J.cdef_idx;
        L.cdef_stride = J.cdef_stride;
        L.cdef_count = J.cdef_count;
        L.cdef = J.cdef;
        L.status = dstatus + i;
        smem_db = std::max(smem_db, build_dbcdef_args(L, htab + off_db + db_rec * q));
        db_prefix[q + 1] = db_prefix[q] + F.tiles_db;
    }

    // restoration records and unit checks
    int* lr_prefix = reinterpret_cast<int*>(htab + off_lr_prefix);
    lr_prefix[0] = 0;
    for (size_t q = 0; q < lr_order.size(); ++q) {
        const int i = lr_order[q];
        const FramePlan& F = plan[i];
        const vaco_av1_frame_job& J = jobs[i];
        const vaco_av1_frame_info& info = J.info;
        LrPlane lp[3];
        for (int k = 0; k < F.np; ++k) {
            const int sx = k ? info.subsampling_x : 0, sy = k ? info.subsampling_y : 0;
            const int w = info.upscaled_width >> sx, h = info.coded_height >> sy;
            const PlaneBuf& after = F.superres ? F.ucdef[k] : F.cdef[k];
            LrPlane& p = lp[k];
            p.plane_index = k;
            p.unit_status = dstatus + i;  // units are validated by the restoration tiles
            p.before = DevPlaneC{nullptr, 0, 0, 0};
            p.after = dev_cplane(base, after);
            p.out = DevPlane{J.dst.planes[k], w, h, J.dst.stride[k]};
            p.width = w;
            p.height = h;
            p.sub_y = (k && info.subsampling_y) ? 1 : 0;
            if (J.lr_type[k] == VACO_AV1_FRAME_LR_NONE) {
                p.before_rows = DevPlaneC{nullptr, 0, 0, 0};
                p.unit_size = 64;
                p.units = nullptr;
                p.unit_cols = p.unit_rows = 1;
                p.copy_only = 1;
            } else {
                const int u = J.lr_unit_size[k];
                if (fused) {
                    p.before_rows = dev_cplane(base, F.superres ? F.urows[k] : F.rows[k]);
                } else {
                    p.before = dev_cplane(base, F.superres ? F.udeb[k] : F.deb[k]);
                    p.before_rows = DevPlaneC{nullptr, 0, 0, 0};
                }
                p.unit_size = u;
                p.units = J.lr_units[k];
                p.unit_cols = std::max((w + u / 2) / u, 1);
                p.unit_rows = std::max((h + u / 2) / u, 1);
                p.copy_only = 0;

            }
        }
        const int tiles = build_lr_args(lp, F.np, info.bit_depth, htab + off_lr + lr_rec * q);
        lr_prefix[q + 1] = lr_prefix[q] + tiles;
    }

    // ---- the launch sequence (captured once per composition when tuned so)
    // the frames' common chroma layout (monochrome counts as 4:4:4), -1 if mixed
    int layout = -2;
    for (int i : order) {
        const vaco_av1_frame_info& fi = jobs[i].info;
        const int l = fi.monochrome ? 0 : fi.subsampling_x | fi.subsampling_y << 1;
        layout = layout == -2 || layout == l ? l : -1;
    }
    auto enqueue = [&]() -> cudaError_t {
        cudaError_t r = cudaMemcpyAsync(dtab, htab, table_bytes, cudaMemcpyHostToDevice, s);
        for (int i : order) {  // unfused: deblocking then CDEF, frame by frame
            if (r != cudaSuccess || fused) break;
            r = enqueue_unfused(jobs[i], plan[i], base, dstatus + i, s);
        }
        if (r == cudaSuccess && fused && !order.empty() && db_prefix[order.size()] > 0)
            r = launch_dbcdef_batch(dtab + off_db, reinterpret_cast<const int*>(dtab + off_db_prefix), (int)order.size(),
                                    db_prefix[order.size()], smem_db, ctx->tuning.dbcdef_ctas_per_sm,
                                    ctx->tuning.dbcdef_threads, layout, s);
        for (int i : order) {
            const FramePlan& F = plan[i];
            if (r != cudaSuccess || !F.superres) continue;
            const vaco_av1_frame_info& info = jobs[i].info;
            SuperresPlane sp[2 * 3];
            int nsp = F.np;
            for (int k = 0; k < F.np; ++k) {
                const int sx = k ? info.subsampling_x : 0, sy = k ? info.subsampling_y : 0;
                sp[k].in = dev_cplane(base, F.cdef[k]);
                sp[k].out = dev_plane(base, F.ucdef[k]);
                sp[k].visible_width = (info.coded_width + sx) >> sx;
                sp[k].output_width = (info.upscaled_width + sx) >> sx;
                sp[k].height = (info.coded_height + sy) >> sy;
            }
            if (F.lr_active && F.run_lr && !fused) {
                // the whole deblocked picture, in the same launch
                for (int k = 0; k < F.np; ++k) {
                    sp[F.np + k] = sp[k];
                    sp[F.np + k].in = dev_cplane(base, F.deb[k]);
                    sp[F.np + k].out = dev_plane(base, F.udeb[k]);
                }
                nsp = 2 * F.np;
            } else if (F.lr_active && F.run_lr) {
                // only the rows the fused kernel wrote (indices 4 .. 4+n), in the same launch
                for (int k = 0; k < F.np; ++k) {
                    const int n_rows = pre_rows_written(jobs[i].src.height[k], k ? info.subsampling_y : 0);
                    DevPlaneC in = dev_cplane(base, F.rows[k]);
                    DevPlane out = dev_plane(base, F.urows[k]);
                    in.data += 4L * in.stride;
                    out.data += 4L * out.stride;
                    in.height = out.height = n_rows;
                    sp[F.np + k] = sp[k];
                    sp[F.np + k].in = in;
                    sp[F.np + k].out = out;
                    sp[F.np + k].height = n_rows;
                }
                nsp = 2 * F.np;
            }
            r = launch_superres(sp, nsp, info.bit_depth, dstatus + i, STAGE_SUPERRES, s);
        }
        if (r == cudaSuccess && !lr_order.empty() && lr_prefix[lr_order.size()] > 0)
            r = launch_restoration_batch(dtab + off_lr, reinterpret_cast<const int*>(dtab + off_lr_prefix),
                                         (int)lr_order.size(), lr_prefix[lr_order.size()], ctx->tuning.lr_ctas_per_sm,
                                         s);
        if (r == cudaSuccess)
            r = cudaMemcpyAsync(ctx->batch_status_host, dstatus, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost,
                                s);
        return r;
    };
    // kernel launches of this batch: deblock+CDEF, superres, restoration
    size_t launches = (order.empty() || !fused ? 0 : 1) + (lr_order.empty() ? 0 : 1);
    for (int i : order) {
        launches += plan[i].superres ? 1 : 0;
        if (!fused)  // copy + checks (1 + planes), two passes, CDEF
            launches += 1 + plan[i].np + (jobs[i].deblock.levels[0] || jobs[i].deblock.levels[1] ? 2 : 0) + 1;
    }
    ctx->mark(0, s);
    const bool graphs = ctx->tuning.use_graphs && s != nullptr;
    if (graphs) {
        signature += "@" + std::to_string(ctx->scratch_generation) + "/" +
                     std::to_string(ctx->tuning.dbcdef_ctas_per_sm) + "/" + std::to_string(ctx->tuning.lr_ctas_per_sm) +
                     "/" + std::to_string(ctx->tuning.largest_first) + "/" +
                     std::to_string(ctx->tuning.dbcdef_threads) + "/" + std::to_string(ctx->tuning.stage_fusion);
        auto it = ctx->graphs.find(signature);
        if (it == ctx->graphs.end()) {
            // kernel attributes are set outside the capture
            e = kernel_attributes();
            cudaGraph_t graph = nullptr;
            if (e == cudaSuccess) e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                cudaError_t r = enqueue();
                e = cudaStreamEndCapture(s, &graph);
                if (r != cudaSuccess) e = r;
            }
            cudaGraphExec_t exec = nullptr;
            if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
            if (graph) cudaGraphDestroy(graph);
            if (e != cudaSuccess) return fail(ctx, e, statuses, msgs, n);
            if (ctx->graphs.size() > 64) {
                for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.second);
                ctx->graphs.clear();
            }
            it = ctx->graphs.emplace(signature, exec).first;
        }
        e = cudaGraphLaunch(it->second, s);
    } else {
        e = enqueue();
    }
    ctx->launches += launches;
    if (e == cudaSuccess) ctx->mark(1, s), ctx->mark(2, s), ctx->mark(3, s), ctx->mark(4, s);
    if (e != cudaSuccess) return fail(ctx, e, statuses, msgs, n);
    pending->n = n;
    pending->host_keys.resize(n);
    pending->queued.resize(n);
    for (int i = 0; i < n; ++i) {
        pending->host_keys[i] = plan[i].host_key;
        pending->queued[i] = plan[i].run_db ? 1 : 0;
    }
    return VACO_AV1_OK;
}

// Per-frame results of a batch whose stream work has completed.
int32_t vaco::batch_collect(vaco_av1_ctx* ctx, const BatchPending& pending, int32_t* statuses, int32_t* msgs) {
    ctx->collect_marks();
    int32_t first = VACO_AV1_OK;
    for (int i = 0; i < pending.n; ++i) {
        unsigned long long key = pending.queued[i] ? ctx->batch_status_host[i] : kNoError;
        if (pending.host_keys[i] < key) key = pending.host_keys[i];
        const int32_t st = key == kNoError ? VACO_AV1_OK : VACO_AV1_INVALID_DATA;
        if (statuses) statuses[i] = st;
        if (msgs) msgs[i] = key == kNoError ? 0 : (int32_t)(key & 0xFF);
        if (first == VACO_AV1_OK && st != VACO_AV1_OK) first = st;
    }
    return first;
}

extern "C" int32_t vaco_av1_postfilter_batch_dev(vaco_av1_ctx* ctx, void* stream, const vaco_av1_frame_job* jobs,
                                                 int32_t n, int32_t* statuses, int32_t* msgs) {
    if (!ctx || (n > 0 && !jobs)) return VACO_AV1_INVALID_DATA;
    if (n <= 0) return VACO_AV1_OK;
    cudaStream_t s = (cudaStream_t)stream;
    BatchPending pending;
    int32_t st = batch_enqueue(ctx, s, jobs, n, &pending);
    if (st != VACO_AV1_OK) {
        for (int i = 0; i < n; ++i) {
            if (statuses) statuses[i] = st;
            if (msgs) msgs[i] = VACO_AV1_MSG_CUDA;
        }
        return st;
    }
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(ctx, e, statuses, msgs, n);
    return batch_collect(ctx, pending, statuses, msgs);
}
