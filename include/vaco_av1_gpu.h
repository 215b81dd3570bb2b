/*
 * vaco_av1_gpu.h -- C ABI of the B200 (sm_100a) AV1 post-decode filter library.
 *
 * The library replaces the scalar AV1 post-filter functions of vaco's
 * `vaco-codec-av1` crate (paths below are relative to the vaco repository):
 *
 *   deblocking (AV1 spec 7.14; vaco has none, see crates/codec/vaco-codec-av1/src/lib.rs:16-18)
 *   -> CDEF      (src/cdef.rs, driver src/decode.rs:739-896)
 *   -> superres  (src/superres.rs:163-274, driver src/decode.rs:865-890)
 *   -> loop restoration (src/restoration.rs:178-384, driver src/decode.rs:683-737)
 *
 * Conventions
 *   - Samples are uint16_t for every bit depth, like vaco's `framebuf::Plane`
 *     (src/framebuf.rs:16-20).  A plane is (pointer, width, height, stride);
 *     stride is the row pitch in samples and must be >= width.
 *   - Inputs are borrowed and never written.  Outputs are caller-allocated.
 *   - `*_host` entry points take host pointers and are synchronous: they copy
 *     inputs to the device, run the kernels and copy results back before
 *     returning.  `*_dev` entry points take device pointers and only enqueue
 *     work on `stream` (a cudaStream_t, NULL = the legacy default stream); the
 *     status they return covers argument checks, launch errors and the data
 *     checks, which need one small device-to-host read of a status word, so a
 *     `*_dev` call synchronizes `stream` once before returning.
 *   - Every entry point returns a status (vaco_av1_status) and, when `msg` is
 *     non-NULL, stores a message id (vaco_av1_msg) naming the failed check;
 *     vaco_av1_message() maps it to the same text vaco's
 *     `vaco_core::Error::InvalidData(&'static str)` carries.  On any error the
 *     output contents are unspecified, matching vaco's all-or-nothing
 *     `Result<Plane>`.
 *   - A context is used by one host thread at a time.  Contexts on the same
 *     device are independent.
 *
 * Budget/fuel accounting (vaco-limits::Budget) stays with the caller, which
 * allocates the outputs through its Budget before the call, so vaco's
 * Error::LimitExceeded keeps its meaning (crates/hw/vaco-hw-cuda-av1 is the
 * Rust shim that does it).
 */
#ifndef VACO_AV1_GPU_H
#define VACO_AV1_GPU_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define VACO_AV1_API __attribute__((visibility("default")))
#else
#define VACO_AV1_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */

/* Mirrors the vaco_core::Error variants a filter can return
 * (crates/core/vaco-core/src/error.rs:14-54). */
typedef enum vaco_av1_status {
    VACO_AV1_OK = 0,
    VACO_AV1_INVALID_DATA = 1,   /* Error::InvalidData(msg)            */
    VACO_AV1_UNSUPPORTED = 2,    /* Error::Unsupported(msg)            */
    VACO_AV1_LIMIT_EXCEEDED = 3, /* Error::LimitExceeded               */
    VACO_AV1_DEVICE_ERROR = 4,   /* CUDA runtime or launch failure     */
    VACO_AV1_TIMEOUT = 5         /* a bounded device wait ran out      */
} vaco_av1_status;

/* Message ids.  The text of each is vaco's own error string where vaco has
 * one (file:line of the string in crates/codec/vaco-codec-av1/). */
typedef enum vaco_av1_msg {
    VACO_AV1_MSG_NONE = 0,
    VACO_AV1_MSG_CDEF_BIT_DEPTH = 1,      /* src/cdef.rs:71  */
    VACO_AV1_MSG_CDEF_SAMPLE = 2,         /* src/cdef.rs:85  */
    VACO_AV1_MSG_CDEF_BLOCK_PARAMS = 3,   /* src/cdef.rs:153 */
    VACO_AV1_MSG_CDEF_STRENGTH_INDEX = 4, /* src/decode.rs:808 */
    VACO_AV1_MSG_SR_BIT_DEPTH = 5,        /* src/superres.rs:130-132 */
    VACO_AV1_MSG_SR_GEOMETRY = 6,         /* src/superres.rs:140 */
    VACO_AV1_MSG_SR_SAMPLE = 7,           /* src/superres.rs:202 */
    VACO_AV1_MSG_LR_GEOMETRY = 8,         /* src/restoration.rs:147-149 */
    VACO_AV1_MSG_LR_UNIT_COUNT = 9,       /* src/restoration.rs:153 */
    VACO_AV1_MSG_LR_COEFFICIENT = 10,     /* src/restoration.rs:85-87 */
    VACO_AV1_MSG_LR_SAMPLE = 11,          /* src/restoration.rs:163-165 */
    VACO_AV1_MSG_LR_NO_UNIT_SIZE = 12,    /* src/decode.rs:599-601 */
    VACO_AV1_MSG_DB_PARAMS = 13,          /* deblocking (no vaco counterpart) */
    VACO_AV1_MSG_DB_SAMPLE = 14,          /* deblocking (no vaco counterpart) */
    VACO_AV1_MSG_FRAME_GEOMETRY = 15,     /* frame/picture descriptor mismatch */
    VACO_AV1_MSG_NULL_ARGUMENT = 16,
    VACO_AV1_MSG_CUDA = 17,               /* see vaco_av1_ctx_last_cuda_error() */
    VACO_AV1_MSG_SCRATCH_LIMIT = 18,      /* request exceeds a fixed scratch size */
    VACO_AV1_MSG_QUEUE_FULL = 19,         /* job admission refused */
    VACO_AV1_MSG_TIMEOUT = 20,
    VACO_AV1_MSG_PIXEL_FORMAT = 21,       /* src/decode.rs:3819 */
    VACO_AV1_MSG_FG_PARAMS = 22,          /* film grain (no vaco counterpart) */
    VACO_AV1_MSG_FG_SAMPLE = 23,          /* film grain (no vaco counterpart) */
    VACO_AV1_MSG_SR_MISSING_U = 24,       /* src/superres.rs:257 */
    VACO_AV1_MSG_SR_MISSING_V = 25,       /* src/superres.rs:265 */
    VACO_AV1_MSG_COUNT = 26
} vaco_av1_msg;

/* Static, NUL-terminated text for a message id ("" for unknown ids). */
VACO_AV1_API const char* vaco_av1_message(int32_t msg);

/* ---------------------------------------------------------------- context */

typedef struct vaco_av1_ctx vaco_av1_ctx;

/* Creates a context on CUDA device `device`.  The context owns the device
 * scratch buffers the multi-stage entry points use and a staging area for the
 * `*_host` entry points; both grow on demand. */
VACO_AV1_API int32_t vaco_av1_ctx_create(int32_t device, vaco_av1_ctx** out);
VACO_AV1_API void vaco_av1_ctx_destroy(vaco_av1_ctx* ctx);
/* cudaError_t of the last VACO_AV1_DEVICE_ERROR on this context (0 if none). */
VACO_AV1_API int32_t vaco_av1_ctx_last_cuda_error(const vaco_av1_ctx* ctx);
/* Number of kernel launches this context has issued (for launch accounting). */
VACO_AV1_API uint64_t vaco_av1_ctx_launch_count(const vaco_av1_ctx* ctx);

/* Deferred status (no counterpart in vaco, whose calls are synchronous).  By
 * default vaco_av1_postfilter_frame_dev (and vaco_av1_film_grain_dev)
 * synchronizes its stream before it returns, to report the first error the
 * device found in that frame, as vaco's Result does.  With deferred status
 * enabled it enqueues the chain (or the grain) and
 * returns after the host-side checks only, so a decoder can keep frames
 * flowing with no host round trip between them.  Device-side errors then
 * accumulate in the context: vaco_av1_ctx_flush() synchronizes `stream`,
 * returns the earliest error (lowest stage, then raster position, then
 * check) of every frame since the previous flush, and clears it.  Output
 * planes of a frame are valid once the stream has passed it.  Enabling or
 * disabling synchronizes the device.  Every other entry point stays
 * synchronous and starts from a clear word, so flush before calling one. */
VACO_AV1_API int32_t vaco_av1_ctx_set_deferred_status(vaco_av1_ctx* ctx, int32_t enable);
VACO_AV1_API int32_t vaco_av1_ctx_flush(vaco_av1_ctx* ctx, void* stream, int32_t* msg);

/* Per-stage device timing (no counterpart in vaco, whose profiling is
 * perf-based: crates/tool/vaco-bench/src/perf_stat.rs).  While enabled, the
 * chain and batch entry points record a CUDA event pair around each stage on
 * the stream the stage runs on; vaco_av1_ctx_stage_ms() returns the summed
 * milliseconds per stage (0 deblocking + CDEF, which the chain runs as one
 * fused kernel; 1 empty in the chain; 2 superres; 3 restoration) and the
 * number of timed frames since timing was (re)enabled.  `enable` > 1 times
 * one frame in `enable` (each timed frame records five events, which take
 * stream time of their own).  Frames enqueued under deferred status are
 * timed too; their events are read at the flush. */
VACO_AV1_API int32_t vaco_av1_ctx_set_stage_timing(vaco_av1_ctx* ctx, int32_t enable);
VACO_AV1_API int32_t vaco_av1_ctx_stage_ms(const vaco_av1_ctx* ctx, double* ms4, uint64_t* frames);

/* ---------------------------------------------------------------- pictures */

/* One reconstruction picture: vaco's `framebuf::Picture` (src/framebuf.rs:79-86).
 * planes[1], planes[2] are NULL for a monochrome picture. */
typedef struct vaco_av1_picture {
    uint16_t* planes[3];
    int32_t width[3];
    int32_t height[3];
    int32_t stride[3];
} vaco_av1_picture;

/* Frame geometry shared by the picture-level entry points.
 * mi_rows/mi_cols count 4x4 luma mode-info cells; the reconstruction planes
 * are Mi-padded (luma mi_cols*4 x mi_rows*4), as vaco allocates them
 * (src/decode.rs:516-526). */
typedef struct vaco_av1_frame_info {
    int32_t bit_depth;      /* 8, 10 or 12 */
    int32_t subsampling_x;  /* 0/1 */
    int32_t subsampling_y;  /* 0/1 */
    int32_t monochrome;     /* 0/1 */
    int32_t mi_rows;
    int32_t mi_cols;
    int32_t coded_width;    /* visible luma width before superres */
    int32_t coded_height;   /* visible luma height */
    int32_t upscaled_width; /* == coded_width when superres is off */
} vaco_av1_frame_info;

/* ---------------------------------------------------------------- CDEF */

/* src/cdef.rs:24-33 CdefParams (strength pairs unscaled, 8-bit units). */
typedef struct vaco_av1_cdef_params {
    uint8_t enabled;
    uint8_t damping;          /* CdefDamping, 3..6 from the syntax */
    uint8_t y_primary[8];
    uint8_t y_secondary[8];
    uint8_t uv_primary[8];
    uint8_t uv_secondary[8];
} vaco_av1_cdef_params;

/* src/cdef.rs:37-54 FilterParams. */
typedef struct vaco_av1_cdef_filter_params {
    uint8_t width;      /* 4 or 8 */
    uint8_t height;     /* 4 or 8 */
    uint8_t edges;      /* left=1 right=2 top=4 bottom=8 */
    uint8_t bit_depth;
    uint8_t direction;  /* 0..7 */
    uint8_t damping;
    uint16_t primary;   /* after variance adjustment and bit-depth scaling */
    uint16_t secondary; /* after bit-depth scaling */
} vaco_av1_cdef_filter_params;

/* cdef::find_direction (src/cdef.rs:79-124) over `n` 8x8 blocks of 64
 * samples each: directions[i], variances[i] for block i. */
VACO_AV1_API int32_t vaco_av1_cdef_find_direction_dev(vaco_av1_ctx* ctx, void* stream,
                                         const uint16_t* blocks, int32_t n,
                                         int32_t bit_depth, uint8_t* directions,
                                         uint32_t* variances, int32_t* msg);
VACO_AV1_API int32_t vaco_av1_cdef_find_direction_host(vaco_av1_ctx* ctx, const uint16_t* blocks,
                                          int32_t n, int32_t bit_depth,
                                          uint8_t* directions, uint32_t* variances,
                                          int32_t* msg);

/* cdef::filter_block (src/cdef.rs:142-205) over `n` 12x12 neighborhoods
 * (144 samples each, block origin at (2,2)); outputs are 8x8 with stride 8
 * and zeroes outside the active width x height. */
VACO_AV1_API int32_t vaco_av1_cdef_filter_block_dev(vaco_av1_ctx* ctx, void* stream,
                                       const uint16_t* inputs,
                                       const vaco_av1_cdef_filter_params* params,
                                       int32_t n, uint16_t* outputs, int32_t* msg);
VACO_AV1_API int32_t vaco_av1_cdef_filter_block_host(vaco_av1_ctx* ctx, const uint16_t* inputs,
                                        const vaco_av1_cdef_filter_params* params,
                                        int32_t n, uint16_t* outputs, int32_t* msg);

/* The frame pass of decode.rs:739-862 (apply_cdef) with its inputs explicit:
 *   skip      mi_rows*mi_cols bytes, 1 = the 4x4 cell's skip flag (MiCell.skip)
 *   cdef_idx  per-64x64 strength index, -1 = absent; entry (r>>4)*cdef_stride+(c>>4)
 * `dst` receives the whole filtered picture (same extents as `src`); src and
 * dst must not overlap.  When CDEF is disabled or every strength is zero the
 * output is a copy of the input, as apply_cdef leaves the picture untouched. */
VACO_AV1_API int32_t vaco_av1_cdef_picture_dev(vaco_av1_ctx* ctx, void* stream,
                                  const vaco_av1_picture* src, const vaco_av1_picture* dst,
                                  const vaco_av1_frame_info* info, const uint8_t* skip,
                                  const int32_t* cdef_idx, int32_t cdef_stride,
                                  int32_t cdef_count, const vaco_av1_cdef_params* params,
                                  int32_t* msg);
VACO_AV1_API int32_t vaco_av1_cdef_picture_host(vaco_av1_ctx* ctx, const vaco_av1_picture* src,
                                   const vaco_av1_picture* dst,
                                   const vaco_av1_frame_info* info, const uint8_t* skip,
                                   const int32_t* cdef_idx, int32_t cdef_stride,
                                   int32_t cdef_count, const vaco_av1_cdef_params* params,
                                   int32_t* msg);

/* ---------------------------------------------------------------- superres */

/* superres::upscale_plane (src/superres.rs:163-216).  `input` is the Mi-padded
 * plane (in_width x in_height); the output is output_width x height. */
VACO_AV1_API int32_t vaco_av1_superres_upscale_plane_dev(vaco_av1_ctx* ctx, void* stream,
                                            const uint16_t* input, int32_t in_width,
                                            int32_t in_height, int32_t in_stride,
                                            int32_t visible_width, int32_t output_width,
                                            int32_t height, int32_t bit_depth,
                                            uint16_t* output, int32_t out_stride,
                                            int32_t* msg);
VACO_AV1_API int32_t vaco_av1_superres_upscale_plane_host(vaco_av1_ctx* ctx, const uint16_t* input,
                                             int32_t in_width, int32_t in_height,
                                             int32_t visible_width, int32_t output_width,
                                             int32_t height, int32_t bit_depth,
                                             uint16_t* output, int32_t* msg);

/* superres::PictureConfig (src/superres.rs:107-122): luma geometry and
 * colour layout of a reconstructed picture. */
typedef struct vaco_av1_superres_picture_config {
    int32_t coded_width;     /* luma width before superres */
    int32_t upscaled_width;  /* luma width after superres */
    int32_t coded_height;    /* visible luma height */
    int32_t subsampling_x;   /* 0/1 */
    int32_t subsampling_y;   /* 0/1 */
    int32_t monochrome;      /* 0/1: U and V absent */
    int32_t bit_depth;       /* 8, 10 or 12 */
} vaco_av1_superres_picture_config;

/* superres::upscale_picture (src/superres.rs:226-274): upscale_plane on luma
 * (coded_width -> upscaled_width, coded_height rows), then on U and V with
 * the ceil-divided chroma geometry, in that order; the first plane that
 * fails decides the error, as in vaco.  `in` holds the Mi-padded planes
 * (width[k] is each plane's padded width, the edge-extension limit); `out`
 * holds caller-allocated planes of exactly the output extents (luma
 * upscaled_width x coded_height, chroma ceil-divided).  A NULL U or V input
 * plane of a non-monochrome picture fails with VACO_AV1_MSG_SR_MISSING_U /
 * _V once luma has succeeded.  All planes run in one launch. */
VACO_AV1_API int32_t vaco_av1_superres_upscale_picture_dev(vaco_av1_ctx* ctx, void* stream,
                                              const vaco_av1_picture* in, const vaco_av1_picture* out,
                                              const vaco_av1_superres_picture_config* config,
                                              int32_t* msg);
VACO_AV1_API int32_t vaco_av1_superres_upscale_picture_host(vaco_av1_ctx* ctx, const vaco_av1_picture* in,
                                               const vaco_av1_picture* out,
                                               const vaco_av1_superres_picture_config* config,
                                               int32_t* msg);

/* ---------------------------------------------------------------- restoration */

enum {
    VACO_AV1_LR_NONE = 0,
    VACO_AV1_LR_WIENER = 1,
    VACO_AV1_LR_SGRPROJ = 2
};

/* src/restoration.rs:48-65 RestorationUnit. */
typedef struct vaco_av1_lr_unit {
    int16_t type;          /* VACO_AV1_LR_* */
    int16_t set;           /* self-guided parameter set, 0..15 */
    int16_t vertical[3];   /* Wiener taps, outermost first */
    int16_t horizontal[3];
    int16_t xqd[2];        /* self-guided projection coefficients */
} vaco_av1_lr_unit;

/* src/restoration.rs:95-106 PlaneConfig. */
typedef struct vaco_av1_lr_plane_config {
    int32_t width;
    int32_t height;
    int32_t bit_depth;
    int32_t unit_size;     /* 32, 64, 128 or 256 */
    int32_t subsampling_y; /* 0/1 */
} vaco_av1_lr_plane_config;

/* restoration::restore_plane (src/restoration.rs:178-207).  before/after are
 * the already-upscaled pre- and post-CDEF planes; output is width x height. */
VACO_AV1_API int32_t vaco_av1_restore_plane_dev(vaco_av1_ctx* ctx, void* stream,
                                   const uint16_t* before, int32_t before_width,
                                   int32_t before_height, int32_t before_stride,
                                   const uint16_t* after, int32_t after_width,
                                   int32_t after_height, int32_t after_stride,
                                   const vaco_av1_lr_plane_config* config,
                                   const vaco_av1_lr_unit* units, int32_t unit_count,
                                   uint16_t* output, int32_t out_stride, int32_t* msg);
VACO_AV1_API int32_t vaco_av1_restore_plane_host(vaco_av1_ctx* ctx, const uint16_t* before,
                                    int32_t before_width, int32_t before_height,
                                    const uint16_t* after, int32_t after_width,
                                    int32_t after_height,
                                    const vaco_av1_lr_plane_config* config,
                                    const vaco_av1_lr_unit* units, int32_t unit_count,
                                    uint16_t* output, int32_t* msg);

/* ---------------------------------------------------------------- deblocking */

/* Frame-level loop-filter syntax kept by vaco's LoopFilterParams
 * (src/frame_header.rs:980-983) plus loop_filter_sharpness, which vaco parses
 * and drops (src/frame_header.rs:1013). */
typedef struct vaco_av1_deblock_params {
    uint8_t levels[4];  /* Y vertical, Y horizontal, U, V */
    uint8_t sharpness;  /* 0..7 */
    uint8_t reserved[3];
} vaco_av1_deblock_params;

/* AV1 spec 7.14 loop filter over an intra frame (vaco decodes intra frames
 * only, src/decode.rs:511-515), in place semantics with src copied to dst:
 *   tx_luma    mi_rows*mi_cols TX_SIZE values (AV1 TX_SIZE enum, 0..18)
 *   tx_chroma  ((mi_rows+ssy)>>ssy)*((mi_cols+ssx)>>ssx) chroma TX_SIZE values
 *   lvl_map    NULL for frame-uniform levels, else 4 bytes per luma Mi cell
 *              holding the final filter level for (Y vertical, Y horizontal,
 *              U, V) after segment and delta adjustments.
 * The tx maps must tile each plane with transform blocks aligned to their own
 * size, as a decoder produces them. */
VACO_AV1_API int32_t vaco_av1_deblock_picture_dev(vaco_av1_ctx* ctx, void* stream,
                                     const vaco_av1_picture* src, const vaco_av1_picture* dst,
                                     const vaco_av1_frame_info* info, const uint8_t* tx_luma,
                                     const uint8_t* tx_chroma, const uint8_t* lvl_map,
                                     const vaco_av1_deblock_params* params, int32_t* msg);
VACO_AV1_API int32_t vaco_av1_deblock_picture_host(vaco_av1_ctx* ctx, const vaco_av1_picture* src,
                                      const vaco_av1_picture* dst,
                                      const vaco_av1_frame_info* info, const uint8_t* tx_luma,
                                      const uint8_t* tx_chroma, const uint8_t* lvl_map,
                                      const vaco_av1_deblock_params* params, int32_t* msg);

/* ---------------------------------------------------------------- whole chain */

/* Frame-level restoration mode, src/restoration.rs:17-27 RestorationType. */
enum {
    VACO_AV1_FRAME_LR_NONE = 0,
    VACO_AV1_FRAME_LR_SWITCHABLE = 1,
    VACO_AV1_FRAME_LR_WIENER = 2,
    VACO_AV1_FRAME_LR_SGRPROJ = 3
};

/* Everything decode_frame (src/decode.rs:553-559) hands the post-filters,
 * with deblocking in front.  Pointers are device pointers for the `_dev`
 * entry points and host pointers for the `_host` ones. */
typedef struct vaco_av1_frame_job {
    vaco_av1_frame_info info;
    vaco_av1_picture src;            /* reconstruction, Mi-padded */
    vaco_av1_picture dst;            /* visible output: upscaled_width x coded_height */
    const uint8_t* tx_luma;
    const uint8_t* tx_chroma;
    const uint8_t* lvl_map;          /* may be NULL */
    const uint8_t* skip;
    const int32_t* cdef_idx;
    int32_t cdef_stride;
    int32_t cdef_count;
    vaco_av1_deblock_params deblock;
    vaco_av1_cdef_params cdef;
    int32_t lr_type[3];              /* VACO_AV1_FRAME_LR_* per plane */
    int32_t lr_unit_size[3];
    const vaco_av1_lr_unit* lr_units[3];
    int32_t lr_unit_count[3];
} vaco_av1_frame_job;

/* deblock -> CDEF -> superres (when upscaled_width != coded_width) -> loop
 * restoration for one frame.  The output is the picture vaco's decode_frame
 * would hand to pic_to_frame, cropped to the visible size; subsampled frames
 * need even coded/upscaled widths and heights. */
VACO_AV1_API int32_t vaco_av1_postfilter_frame_dev(vaco_av1_ctx* ctx, void* stream,
                                      const vaco_av1_frame_job* job, int32_t* msg);
VACO_AV1_API int32_t vaco_av1_postfilter_frame_host(vaco_av1_ctx* ctx, const vaco_av1_frame_job* job,
                                       int32_t* msg);

/* ---------------------------------------------------------------- batched form */

/* Launch-shape knobs for the batched form (no counterpart in vaco).  The
 * values in tuned/ are picked by vaco_b200.autotune on the target GPU. */
typedef struct vaco_av1_tuning {
    int32_t dbcdef_ctas_per_sm;  /* resident CTAs per SM the batched deblock+CDEF kernel
                                    is compiled for, i.e. its register budget (1..8):
                                    up to 3 -> 80 registers a thread, 4 and more -> 64
                                    (256-thread tiles; 128-thread tiles have one body) */
    int32_t lr_ctas_per_sm;      /* the same for the batched restoration kernel (1..8):
                                    up to 3 -> 80 registers, 4 and more -> 64 */
    int32_t use_graphs;          /* capture each batch composition once as a CUDA graph */
    int32_t largest_first;       /* lay the largest frames' tiles first in the launch */
    int32_t dbcdef_threads;      /* threads per 64x64 tile of the deblock+CDEF kernel, in the
                                    batched form and vaco_av1_postfilter_frame_dev: 256 or
                                    128 (0 = 256) */
    int32_t stage_fusion;        /* batched form: 1 = deblocking and CDEF in one fused
                                    kernel; 0 = as separate per-stage kernels, frame by
                                    frame */
} vaco_av1_tuning;

VACO_AV1_API int32_t vaco_av1_ctx_set_tuning(vaco_av1_ctx* ctx, const vaco_av1_tuning* tuning);
VACO_AV1_API int32_t vaco_av1_ctx_get_tuning(const vaco_av1_ctx* ctx, vaco_av1_tuning* tuning);

/* The chain over `n` frames of any sizes and bit depths in one launch set
 * (no counterpart in vaco, which filters one frame per decode_frame call,
 * src/decode.rs:553-559).  Pointers in `jobs` are device pointers.
 * Deblock+CDEF and restoration each run as one kernel launch with one CTA
 * per tile of all frames, the frames' tiles laid end to end; every frame
 * keeps its own status word.  statuses[i] / msgs[i] (both optional) receive
 * frame i's result; the return value is VACO_AV1_OK when every frame
 * succeeded, else the status of the first failing frame.  Synchronizes
 * `stream` once for the whole batch. */
VACO_AV1_API int32_t vaco_av1_postfilter_batch_dev(vaco_av1_ctx* ctx, void* stream, const vaco_av1_frame_job* jobs,
                                                   int32_t n, int32_t* statuses, int32_t* msgs);

/* ---------------------------------------------------------------- served form */

/* A request server (no counterpart in vaco): many decoder streams submit
 * frames as they are reconstructed; a worker thread packs every pending frame
 * into the next batched launch set as soon as one of its in-flight slots is
 * free (continuous batching), so frames that arrive while others are on the
 * GPU are admitted as slots free up and their work overlaps on the device.
 * Each stream's frame buffers live in device memory for the stream's
 * lifetime, admitted against a device-memory budget. */
typedef struct vaco_av1_server vaco_av1_server;

typedef struct vaco_av1_server_config {
    int32_t device;
    int32_t max_batch_frames;     /* frames packed into one launch set */
    int32_t inflight_batches;     /* launch sets in flight (one CUDA stream each) */
    int32_t host_wait_ms;         /* bound of the host waits in submit (backpressure)
                                     and close_stream; 0 = 10000 */
    int64_t memory_budget_bytes;  /* stream buffers + batch scratch */
} vaco_av1_server_config;

typedef struct vaco_av1_server_stats {
    uint64_t submitted;
    uint64_t completed;
    uint64_t failed;
    uint64_t batches;
    uint64_t max_batch;           /* largest launch set so far */
    int64_t resident_bytes;       /* stream buffers currently admitted */
    int64_t scratch_bytes;        /* batch scratch reserved per in-flight slot x slots */
} vaco_av1_server_stats;

VACO_AV1_API int32_t vaco_av1_server_create(const vaco_av1_server_config* config, vaco_av1_server** out);
VACO_AV1_API void vaco_av1_server_destroy(vaco_av1_server* server);

/* Admits a stream of frames with geometry `info` (4:2:0 or any layout the
 * chain accepts) and restoration unit sizes lr_unit_size[3] (0 = no
 * restoration for that plane), holding `buffers` frame slots resident on the
 * device.  Fails with VACO_AV1_LIMIT_EXCEEDED / VACO_AV1_MSG_QUEUE_FULL when
 * the budget cannot hold the stream's buffers. */
VACO_AV1_API int32_t vaco_av1_server_open_stream(vaco_av1_server* server, const vaco_av1_frame_info* info,
                                                 const int32_t* lr_unit_size, int32_t buffers, int32_t* stream_id,
                                                 int32_t* msg);
/* Closes a stream and frees its buffers once none of its frames is in flight.
 * Waits at most host_wait_ms (10 s by default) for them; then returns
 * VACO_AV1_TIMEOUT and leaves the stream open (its frames still complete, and
 * a later close succeeds). */
VACO_AV1_API int32_t vaco_av1_server_close_stream(vaco_av1_server* server, int32_t stream_id);

/* Device pointers of slot `slot` of a stream, filled into `job` (src and dst
 * pictures, side-information arrays, unit arrays): the decoder writes the
 * reconstruction and side information there before submitting the slot. */
VACO_AV1_API int32_t vaco_av1_server_slot(vaco_av1_server* server, int32_t stream_id, int32_t slot,
                                          vaco_av1_frame_job* job);

/* Queues slot `slot` of a stream with the frame-level parameters of `params`
 * (deblock, cdef, lr_type; its pointers and geometry are ignored) and returns
 * a ticket.  Does not wait for the GPU, except that a slot whose previous
 * frame is still being filtered is waited for first (backpressure, at most
 * host_wait_ms, 10 s by default, then VACO_AV1_TIMEOUT). */
VACO_AV1_API int32_t vaco_av1_server_submit(vaco_av1_server* server, int32_t stream_id, int32_t slot,
                                            const vaco_av1_frame_job* params, uint64_t* ticket);

/* Like vaco_av1_server_submit, with the frame's inputs in HOST memory: `host`
 * carries host pointers to the reconstruction, side information and
 * restoration units (extents as the stream's, as for
 * vaco_av1_server_upload) together with the frame-level parameters.  The
 * copies into the slot are enqueued on the server's own copy streams and the
 * launch that takes the frame waits for them on the device, so one frame's
 * upload overlaps other frames' filtering and the ticket's latency includes
 * the upload.  Host buffers must stay valid until the ticket's wait returns;
 * page-locked buffers let the copies run asynchronously.  Backpressure and
 * TIMEOUT as for vaco_av1_server_submit; VACO_AV1_INVALID_DATA when the host
 * frame does not match the stream. */
VACO_AV1_API int32_t vaco_av1_server_submit_host(vaco_av1_server* server, int32_t stream_id, int32_t slot,
                                                 const vaco_av1_frame_job* host, uint64_t* ticket);

/* Waits up to timeout_ms (< 0: forever) for a ticket.  Returns VACO_AV1_TIMEOUT
 * if it has not completed; otherwise the frame's status, with the message and
 * the submit-to-completion latency in milliseconds.  A completed ticket is
 * released by this call. */
VACO_AV1_API int32_t vaco_av1_server_wait(vaco_av1_server* server, uint64_t ticket, int32_t timeout_ms,
                                          int32_t* msg, double* latency_ms);

VACO_AV1_API int32_t vaco_av1_server_get_stats(vaco_av1_server* server, vaco_av1_server_stats* stats);

/* Bulk forms of submit / wait for clients that feed many streams from one
 * thread: entry i is (stream_ids[i], slots[i], params[i]) -> tickets[i]. */
VACO_AV1_API int32_t vaco_av1_server_submit_many(vaco_av1_server* server, int32_t n, const int32_t* stream_ids,
                                                 const int32_t* slots, const vaco_av1_frame_job* params,
                                                 uint64_t* tickets);
VACO_AV1_API int32_t vaco_av1_server_wait_many(vaco_av1_server* server, int32_t n, const uint64_t* tickets,
                                               int32_t timeout_ms, int32_t* statuses, int32_t* msgs,
                                               double* latency_ms);

/* Host-memory conveniences around vaco_av1_server_slot(): copy a frame's
 * reconstruction, side information and restoration units from host arrays
 * (`host` uses host pointers; extents must match the stream) into a slot, and
 * copy a completed slot's output planes back.  Both are synchronous. */
VACO_AV1_API int32_t vaco_av1_server_upload(vaco_av1_server* server, int32_t stream_id, int32_t slot,
                                            const vaco_av1_frame_job* host);
VACO_AV1_API int32_t vaco_av1_server_download(vaco_av1_server* server, int32_t stream_id, int32_t slot,
                                              const vaco_av1_picture* host);

/* Pipelined form of vaco_av1_postfilter_frame_host (no counterpart in vaco,
 * whose decode_frame filters one frame at a time).  submit validates the
 * job, enqueues the copy of its inputs to the device, the chain and the copy
 * of the output planes back to job->dst, and returns a ticket at once; up to
 * three frames are in flight, each in its own device buffers, so one
 * frame's copies overlap another's filtering.  A fourth submit before any
 * wait returns VACO_AV1_LIMIT_EXCEEDED / VACO_AV1_MSG_QUEUE_FULL.  wait
 * blocks until the frame's output planes are in host memory and returns its
 * status as vaco_av1_postfilter_frame_host would.  The job's host buffers
 * must stay valid until its wait returns; page-locked buffers let the
 * copies run asynchronously.  Host-side check failures are returned by
 * submit itself. */
VACO_AV1_API int32_t vaco_av1_postfilter_frame_host_submit(vaco_av1_ctx* ctx, const vaco_av1_frame_job* job,
                                                           uint64_t* ticket, int32_t* msg);
VACO_AV1_API int32_t vaco_av1_postfilter_frame_host_wait(vaco_av1_ctx* ctx, uint64_t ticket, int32_t* msg);

/* ---------------------------------------------------------------- frame emission */

/* Destination planes of an emitted frame (Y, U, V; U and V unused for
 * monochrome), in the layout vaco's Frame::alloc_video gives them
 * (crates/model/vaco-frame/src/alloc.rs:58-90): each row `linesize` bytes. */
typedef struct vaco_av1_frame_buffer {
    void* planes[3];
    int64_t linesize[3];
} vaco_av1_frame_buffer;

/* Replaces pic_to_frame / blit (src/decode.rs:3795-3891): packs `pic` into
 * `out` as the frame's pixel format -- gray / yuv4xxp for 8 bits (one byte
 * per sample; a sample above 255 becomes 0, as blit's u8 conversion does) or
 * gray / yuv4xxp{10,12}le (little-endian u16).  Copies
 * upscaled_width x coded_height luma samples and the chroma extents rounded
 * up, each cut to its source plane's size; the rest of every row is left
 * untouched.  8-bit 4:4:0 has no pixel format in vaco and fails with
 * VACO_AV1_MSG_PIXEL_FORMAT.  _dev: device pointers (pic and out); no sample
 * can fail, so it returns once the kernel is enqueued on `stream` and the
 * frame is complete when the stream passes it.  _host: host pointers,
 * synchronous. */
VACO_AV1_API int32_t vaco_av1_emit_frame_dev(vaco_av1_ctx* ctx, void* stream, const vaco_av1_picture* pic,
                                             const vaco_av1_frame_info* info, const vaco_av1_frame_buffer* out,
                                             int32_t* msg);
VACO_AV1_API int32_t vaco_av1_emit_frame_host(vaco_av1_ctx* ctx, const vaco_av1_picture* pic,
                                              const vaco_av1_frame_info* info, const vaco_av1_frame_buffer* out,
                                              int32_t* msg);

/* decode_frame's filter tail followed by pic_to_frame (src/decode.rs:553-559,
 * :3795-3891), host memory in and out: the chain's u16 output stays on the
 * device and only the packed frame (half the bytes at 8 bits) comes back.
 * job->dst is ignored. */
VACO_AV1_API int32_t vaco_av1_postfilter_frame_emit_host(vaco_av1_ctx* ctx, const vaco_av1_frame_job* job,
                                                         const vaco_av1_frame_buffer* out, int32_t* msg);

/* ---------------------------------------------------------------- film grain */

/* film_grain_params() (AV1 spec 5.9.30): the fields vaco's parser reads and
 * discards (src/frame_header.rs:1125-1210; vaco has no grain synthesis,
 * src/lib.rs:16-18), plus mc_identity (matrix_coefficients == MC_IDENTITY,
 * from the sequence header).  Coefficients keep their coded "+128" form. */
typedef struct vaco_av1_film_grain_params {
    uint8_t apply_grain;
    uint8_t num_y_points;             /* 0..14, point values increasing */
    uint16_t grain_seed;
    uint8_t point_y_value[14];
    uint8_t point_y_scaling[14];
    uint8_t chroma_scaling_from_luma;
    uint8_t num_cb_points;            /* 0..10 */
    uint8_t point_cb_value[10];
    uint8_t point_cb_scaling[10];
    uint8_t num_cr_points;            /* 0..10 */
    uint8_t point_cr_value[10];
    uint8_t point_cr_scaling[10];
    uint8_t grain_scaling_minus_8;    /* 0..3 */
    uint8_t ar_coeff_lag;             /* 0..3 */
    uint8_t ar_coeffs_y_plus_128[24];
    uint8_t ar_coeffs_cb_plus_128[25];
    uint8_t ar_coeffs_cr_plus_128[25];
    uint8_t ar_coeff_shift_minus_6;   /* 0..3 */
    uint8_t grain_scale_shift;        /* 0..3 */
    uint8_t cb_mult, cb_luma_mult;
    uint16_t cb_offset;               /* 0..511 */
    uint8_t cr_mult, cr_luma_mult;
    uint16_t cr_offset;               /* 0..511 */
    uint8_t overlap_flag;
    uint8_t clip_to_restricted_range;
    uint8_t mc_identity;
} vaco_av1_film_grain_params;

/* Film grain synthesis (AV1 spec 7.18.3; the step after the post-filters
 * that vaco parses but does not implement): `out` = `in` with the grain of
 * `params` added, for the frame of info->upscaled_width x
 * info->coded_height (chroma extents rounded up).  `gaussian_sequence` is
 * the spec's 2048-entry Gaussian_Sequence table in HOST memory, supplied by
 * the caller (the decoder holds the normative table); the call reads it
 * before returning.  Fails with VACO_AV1_MSG_FG_PARAMS for parameters
 * outside the ranges above (point values must increase), with
 * VACO_AV1_MSG_FRAME_GEOMETRY for planes smaller than the frame, and with
 * VACO_AV1_MSG_FG_SAMPLE when a sample of `in` exceeds the bit depth.
 * apply_grain == 0 copies `in` to `out`.  `in` and `out` may not overlap.
 * The grain templates depend only on `params`; they are built on one of the
 * context's internal streams (one per workspace set, eight sets used in
 * turn), ordered against `stream` by events, so consecutive frames' template
 * builds overlap each other and the frames' other work.
 * _dev: device pointers, runs on `stream` and synchronizes it for the
 * status, unless the context has deferred status enabled (then it only
 * enqueues; vaco_av1_ctx_flush reports).  _host: host pointers,
 * synchronous. */
VACO_AV1_API int32_t vaco_av1_film_grain_dev(vaco_av1_ctx* ctx, void* stream, const vaco_av1_picture* in,
                                             const vaco_av1_picture* out, const vaco_av1_frame_info* info,
                                             const vaco_av1_film_grain_params* params,
                                             const int16_t* gaussian_sequence, int32_t* msg);
VACO_AV1_API int32_t vaco_av1_film_grain_host(vaco_av1_ctx* ctx, const vaco_av1_picture* in,
                                              const vaco_av1_picture* out, const vaco_av1_frame_info* info,
                                              const vaco_av1_film_grain_params* params,
                                              const int16_t* gaussian_sequence, int32_t* msg);

/* The whole chain for callers that cannot call cudaMalloc.  No counterpart in
 * vaco (vaco allocates every intermediate picture through its Budget).
 *
 * Examples of such callers: a decoder plugin in a host application that owns
 * all device memory through its own pool and forbids plugins from
 * allocating, or a real-time path where an allocation's implicit device-wide
 * synchronization would stall unrelated streams.
 *
 * The caller passes device pointers for every input and output in `job`.
 * The call needs no context and allocates nothing.  Intermediate pictures
 * and the status word live in one fixed device array of 16 MiB (plus 256 B)
 * in the library; every GPU that loads the library holds it until exit.
 * Frames whose intermediates do not fit fail with VACO_AV1_LIMIT_EXCEEDED /
 * VACO_AV1_MSG_SCRATCH_LIMIT before any work.  A 1920-wide 4:2:0 frame fits
 * up to 1456 rows without superres (so 1920x1088 fits); with superres and
 * restoration, 1024x720 -> 1280x720 fits and 1440x1080 -> 1920x1080 does
 * not.  The chain runs as per-stage kernels (not the fused deblock+CDEF
 * kernel of vaco_av1_postfilter_frame_dev), with identical output.
 * All calls share the array.  Calls whose GPU work overlaps race and produce
 * undefined output.
 * The first call on a device does a one-time set-up there: it looks up the
 * array's device address (cudaGetSymbolAddress) and caches it.  Make that
 * first call before any stream capture begins on the device.
 * Works on the current device and synchronizes `stream` once. */
VACO_AV1_API int32_t vaco_av1_postfilter_frame_noalloc(void* stream, const vaco_av1_frame_job* job,
                                                       int32_t* msg);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* VACO_AV1_GPU_H */
