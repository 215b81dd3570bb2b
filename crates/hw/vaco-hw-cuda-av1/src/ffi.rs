//! Raw C ABI of the B200 AV1 post-filter library (`include/vaco_av1_gpu.h`
//! of the library's repository): `#[repr(C)]` mirrors of its structs, its
//! status and message codes, and one declaration per entry point.
//!
//! Everything here is `unsafe` to call; `crate` wraps the calls vaco's
//! decoder makes in safe functions with vaco's own signatures.

#![allow(missing_docs, reason = "field-for-field mirror of the C header, documented there")]

use core::ffi::{c_char, c_void};

/// `vaco_av1_status`: mirrors `vaco_core::Error` (crates/core/vaco-core/src/error.rs:14-54).
pub const OK: i32 = 0;
pub const INVALID_DATA: i32 = 1;
pub const UNSUPPORTED: i32 = 2;
pub const LIMIT_EXCEEDED: i32 = 3;
pub const DEVICE_ERROR: i32 = 4;
pub const TIMEOUT: i32 = 5;

/// `vaco_av1_msg` texts, index = message id.  The same `&'static str` vaco
/// returns where vaco has the check; `tests::message_table_matches_library`
/// compares this table with the library's `vaco_av1_message`.
pub const MESSAGES: [&str; 26] = [
    "",
    "CDEF bit depth must be 8, 10, or 12",
    "CDEF sample exceeds bit depth",
    "invalid CDEF block parameters",
    "CDEF strength index exceeds table",
    "AV1 superres bit depth must be 8, 10, or 12",
    "invalid AV1 superres plane geometry",
    "AV1 superres sample exceeds bit depth",
    "AV1 restoration plane geometry or bit depth",
    "AV1 restoration unit count",
    "AV1 restoration coefficient out of range",
    "AV1 restoration sample exceeds bit depth",
    "AV1 active restoration has no unit size",
    "invalid AV1 deblocking parameters",
    "AV1 deblocking sample exceeds bit depth",
    "AV1 frame geometry does not match its pictures",
    "required argument is NULL",
    "CUDA runtime error",
    "request exceeds the fixed scratch size",
    "job admission refused: queue or memory budget full",
    "bounded device wait timed out",
    "vaco-codec-av1: unsupported pixel format",
    "invalid AV1 film grain parameters",
    "AV1 film grain sample exceeds bit depth",
    "AV1 superres missing U plane",
    "AV1 superres missing V plane",
];

/// `vaco_av1_ctx` (opaque).
#[repr(C)]
#[derive(Debug)]
pub struct Ctx {
    _opaque: [u8; 0],
}

/// `vaco_av1_server` (opaque).
#[repr(C)]
#[derive(Debug)]
pub struct Server {
    _opaque: [u8; 0],
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct Picture {
    pub planes: [*mut u16; 3],
    pub width: [i32; 3],
    pub height: [i32; 3],
    pub stride: [i32; 3],
}

impl Default for Picture {
    fn default() -> Self {
        Self {
            planes: [core::ptr::null_mut(); 3],
            width: [0; 3],
            height: [0; 3],
            stride: [0; 3],
        }
    }
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct FrameInfo {
    pub bit_depth: i32,
    pub subsampling_x: i32,
    pub subsampling_y: i32,
    pub monochrome: i32,
    pub mi_rows: i32,
    pub mi_cols: i32,
    pub coded_width: i32,
    pub coded_height: i32,
    pub upscaled_width: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct CdefParams {
    pub enabled: u8,
    pub damping: u8,
    pub y_primary: [u8; 8],
    pub y_secondary: [u8; 8],
    pub uv_primary: [u8; 8],
    pub uv_secondary: [u8; 8],
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct CdefFilterParams {
    pub width: u8,
    pub height: u8,
    pub edges: u8,
    pub bit_depth: u8,
    pub direction: u8,
    pub damping: u8,
    pub primary: u16,
    pub secondary: u16,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct SuperresPictureConfig {
    pub coded_width: i32,
    pub upscaled_width: i32,
    pub coded_height: i32,
    pub subsampling_x: i32,
    pub subsampling_y: i32,
    pub monochrome: i32,
    pub bit_depth: i32,
}

/// `VACO_AV1_LR_*` unit kinds.
pub const LR_NONE: i16 = 0;
pub const LR_WIENER: i16 = 1;
pub const LR_SGRPROJ: i16 = 2;

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct LrUnit {
    /// `type` in the header.
    pub kind: i16,
    pub set: i16,
    pub vertical: [i16; 3],
    pub horizontal: [i16; 3],
    pub xqd: [i16; 2],
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct LrPlaneConfig {
    pub width: i32,
    pub height: i32,
    pub bit_depth: i32,
    pub unit_size: i32,
    pub subsampling_y: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct DeblockParams {
    pub levels: [u8; 4],
    pub sharpness: u8,
    pub reserved: [u8; 3],
}

/// `VACO_AV1_FRAME_LR_*` frame-level restoration modes.
pub const FRAME_LR_NONE: i32 = 0;
pub const FRAME_LR_SWITCHABLE: i32 = 1;
pub const FRAME_LR_WIENER: i32 = 2;
pub const FRAME_LR_SGRPROJ: i32 = 3;

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct FrameJob {
    pub info: FrameInfo,
    pub src: Picture,
    pub dst: Picture,
    pub tx_luma: *const u8,
    pub tx_chroma: *const u8,
    pub lvl_map: *const u8,
    pub skip: *const u8,
    pub cdef_idx: *const i32,
    pub cdef_stride: i32,
    pub cdef_count: i32,
    pub deblock: DeblockParams,
    pub cdef: CdefParams,
    pub lr_type: [i32; 3],
    pub lr_unit_size: [i32; 3],
    pub lr_units: [*const LrUnit; 3],
    pub lr_unit_count: [i32; 3],
}

impl Default for FrameJob {
    fn default() -> Self {
        Self {
            info: FrameInfo::default(),
            src: Picture::default(),
            dst: Picture::default(),
            tx_luma: core::ptr::null(),
            tx_chroma: core::ptr::null(),
            lvl_map: core::ptr::null(),
            skip: core::ptr::null(),
            cdef_idx: core::ptr::null(),
            cdef_stride: 0,
            cdef_count: 0,
            deblock: DeblockParams::default(),
            cdef: CdefParams::default(),
            lr_type: [0; 3],
            lr_unit_size: [0; 3],
            lr_units: [core::ptr::null(); 3],
            lr_unit_count: [0; 3],
        }
    }
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct Tuning {
    pub dbcdef_ctas_per_sm: i32,
    pub lr_ctas_per_sm: i32,
    pub use_graphs: i32,
    pub largest_first: i32,
    pub dbcdef_threads: i32,
    pub stage_fusion: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ServerConfig {
    pub device: i32,
    pub max_batch_frames: i32,
    pub inflight_batches: i32,
    pub host_wait_ms: i32,
    pub memory_budget_bytes: i64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ServerStats {
    pub submitted: u64,
    pub completed: u64,
    pub failed: u64,
    pub batches: u64,
    pub max_batch: u64,
    pub resident_bytes: i64,
    pub scratch_bytes: i64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct FrameBuffer {
    pub planes: [*mut c_void; 3],
    pub linesize: [i64; 3],
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct FilmGrainParams {
    pub apply_grain: u8,
    pub num_y_points: u8,
    pub grain_seed: u16,
    pub point_y_value: [u8; 14],
    pub point_y_scaling: [u8; 14],
    pub chroma_scaling_from_luma: u8,
    pub num_cb_points: u8,
    pub point_cb_value: [u8; 10],
    pub point_cb_scaling: [u8; 10],
    pub num_cr_points: u8,
    pub point_cr_value: [u8; 10],
    pub point_cr_scaling: [u8; 10],
    pub grain_scaling_minus_8: u8,
    pub ar_coeff_lag: u8,
    pub ar_coeffs_y_plus_128: [u8; 24],
    pub ar_coeffs_cb_plus_128: [u8; 25],
    pub ar_coeffs_cr_plus_128: [u8; 25],
    pub ar_coeff_shift_minus_6: u8,
    pub grain_scale_shift: u8,
    pub cb_mult: u8,
    pub cb_luma_mult: u8,
    pub cb_offset: u16,
    pub cr_mult: u8,
    pub cr_luma_mult: u8,
    pub cr_offset: u16,
    pub overlap_flag: u8,
    pub clip_to_restricted_range: u8,
    pub mc_identity: u8,
}

// One declaration per entry point of include/vaco_av1_gpu.h, in header order.
#[link(name = "vaco_av1_gpu")]
unsafe extern "C" {
    pub fn vaco_av1_message(msg: i32) -> *const c_char;
    pub fn vaco_av1_ctx_create(device: i32, out: *mut *mut Ctx) -> i32;
    pub fn vaco_av1_ctx_destroy(ctx: *mut Ctx);
    pub fn vaco_av1_ctx_last_cuda_error(ctx: *const Ctx) -> i32;
    pub fn vaco_av1_ctx_launch_count(ctx: *const Ctx) -> u64;
    pub fn vaco_av1_ctx_set_deferred_status(ctx: *mut Ctx, enable: i32) -> i32;
    pub fn vaco_av1_ctx_flush(ctx: *mut Ctx, stream: *mut c_void, msg: *mut i32) -> i32;
    pub fn vaco_av1_ctx_set_stage_timing(ctx: *mut Ctx, enable: i32) -> i32;
    pub fn vaco_av1_ctx_stage_ms(ctx: *const Ctx, ms4: *mut f64, frames: *mut u64) -> i32;
    pub fn vaco_av1_cdef_find_direction_dev(ctx: *mut Ctx, stream: *mut c_void, blocks: *const u16, n: i32, bit_depth: i32, directions: *mut u8, variances: *mut u32, msg: *mut i32) -> i32;
    pub fn vaco_av1_cdef_find_direction_host(ctx: *mut Ctx, blocks: *const u16, n: i32, bit_depth: i32, directions: *mut u8, variances: *mut u32, msg: *mut i32) -> i32;
    pub fn vaco_av1_cdef_filter_block_dev(ctx: *mut Ctx, stream: *mut c_void, inputs: *const u16, params: *const CdefFilterParams, n: i32, outputs: *mut u16, msg: *mut i32) -> i32;
    pub fn vaco_av1_cdef_filter_block_host(ctx: *mut Ctx, inputs: *const u16, params: *const CdefFilterParams, n: i32, outputs: *mut u16, msg: *mut i32) -> i32;
    pub fn vaco_av1_cdef_picture_dev(ctx: *mut Ctx, stream: *mut c_void, src: *const Picture, dst: *const Picture, info: *const FrameInfo, skip: *const u8, cdef_idx: *const i32, cdef_stride: i32, cdef_count: i32, params: *const CdefParams, msg: *mut i32) -> i32;
    pub fn vaco_av1_cdef_picture_host(ctx: *mut Ctx, src: *const Picture, dst: *const Picture, info: *const FrameInfo, skip: *const u8, cdef_idx: *const i32, cdef_stride: i32, cdef_count: i32, params: *const CdefParams, msg: *mut i32) -> i32;
    pub fn vaco_av1_superres_upscale_plane_dev(ctx: *mut Ctx, stream: *mut c_void, input: *const u16, in_width: i32, in_height: i32, in_stride: i32, visible_width: i32, output_width: i32, height: i32, bit_depth: i32, output: *mut u16, out_stride: i32, msg: *mut i32) -> i32;
    pub fn vaco_av1_superres_upscale_plane_host(ctx: *mut Ctx, input: *const u16, in_width: i32, in_height: i32, visible_width: i32, output_width: i32, height: i32, bit_depth: i32, output: *mut u16, msg: *mut i32) -> i32;
    pub fn vaco_av1_superres_upscale_picture_dev(ctx: *mut Ctx, stream: *mut c_void, in_: *const Picture, out: *const Picture, config: *const SuperresPictureConfig, msg: *mut i32) -> i32;
    pub fn vaco_av1_superres_upscale_picture_host(ctx: *mut Ctx, in_: *const Picture, out: *const Picture, config: *const SuperresPictureConfig, msg: *mut i32) -> i32;
    pub fn vaco_av1_restore_plane_dev(ctx: *mut Ctx, stream: *mut c_void, before: *const u16, before_width: i32, before_height: i32, before_stride: i32, after: *const u16, after_width: i32, after_height: i32, after_stride: i32, config: *const LrPlaneConfig, units: *const LrUnit, unit_count: i32, output: *mut u16, out_stride: i32, msg: *mut i32) -> i32;
    pub fn vaco_av1_restore_plane_host(ctx: *mut Ctx, before: *const u16, before_width: i32, before_height: i32, after: *const u16, after_width: i32, after_height: i32, config: *const LrPlaneConfig, units: *const LrUnit, unit_count: i32, output: *mut u16, msg: *mut i32) -> i32;
    pub fn vaco_av1_deblock_picture_dev(ctx: *mut Ctx, stream: *mut c_void, src: *const Picture, dst: *const Picture, info: *const FrameInfo, tx_luma: *const u8, tx_chroma: *const u8, lvl_map: *const u8, params: *const DeblockParams, msg: *mut i32) -> i32;
    pub fn vaco_av1_deblock_picture_host(ctx: *mut Ctx, src: *const Picture, dst: *const Picture, info: *const FrameInfo, tx_luma: *const u8, tx_chroma: *const u8, lvl_map: *const u8, params: *const DeblockParams, msg: *mut i32) -> i32;
    pub fn vaco_av1_postfilter_frame_dev(ctx: *mut Ctx, stream: *mut c_void, job: *const FrameJob, msg: *mut i32) -> i32;
    pub fn vaco_av1_postfilter_frame_host(ctx: *mut Ctx, job: *const FrameJob, msg: *mut i32) -> i32;
    pub fn vaco_av1_ctx_set_tuning(ctx: *mut Ctx, tuning: *const Tuning) -> i32;
    pub fn vaco_av1_ctx_get_tuning(ctx: *const Ctx, tuning: *mut Tuning) -> i32;
    pub fn vaco_av1_postfilter_batch_dev(ctx: *mut Ctx, stream: *mut c_void, jobs: *const FrameJob, n: i32, statuses: *mut i32, msgs: *mut i32) -> i32;
    pub fn vaco_av1_server_create(config: *const ServerConfig, out: *mut *mut Server) -> i32;
    pub fn vaco_av1_server_destroy(server: *mut Server);
    pub fn vaco_av1_server_open_stream(server: *mut Server, info: *const FrameInfo, lr_unit_size: *const i32, buffers: i32, stream_id: *mut i32, msg: *mut i32) -> i32;
    pub fn vaco_av1_server_close_stream(server: *mut Server, stream_id: i32) -> i32;
    pub fn vaco_av1_server_slot(server: *mut Server, stream_id: i32, slot: i32, job: *mut FrameJob) -> i32;
    pub fn vaco_av1_server_submit(server: *mut Server, stream_id: i32, slot: i32, params: *const FrameJob, ticket: *mut u64) -> i32;
    pub fn vaco_av1_server_submit_host(server: *mut Server, stream_id: i32, slot: i32, host: *const FrameJob, ticket: *mut u64) -> i32;
    pub fn vaco_av1_server_wait(server: *mut Server, ticket: u64, timeout_ms: i32, msg: *mut i32, latency_ms: *mut f64) -> i32;
    pub fn vaco_av1_server_get_stats(server: *mut Server, stats: *mut ServerStats) -> i32;
    pub fn vaco_av1_server_submit_many(server: *mut Server, n: i32, stream_ids: *const i32, slots: *const i32, params: *const FrameJob, tickets: *mut u64) -> i32;
    pub fn vaco_av1_server_wait_many(server: *mut Server, n: i32, tickets: *const u64, timeout_ms: i32, statuses: *mut i32, msgs: *mut i32, latency_ms: *mut f64) -> i32;
    pub fn vaco_av1_server_upload(server: *mut Server, stream_id: i32, slot: i32, host: *const FrameJob) -> i32;
    pub fn vaco_av1_server_download(server: *mut Server, stream_id: i32, slot: i32, host: *const Picture) -> i32;
    pub fn vaco_av1_postfilter_frame_host_submit(ctx: *mut Ctx, job: *const FrameJob, ticket: *mut u64, msg: *mut i32) -> i32;
    pub fn vaco_av1_postfilter_frame_host_wait(ctx: *mut Ctx, ticket: u64, msg: *mut i32) -> i32;
    pub fn vaco_av1_emit_frame_dev(ctx: *mut Ctx, stream: *mut c_void, pic: *const Picture, info: *const FrameInfo, out: *const FrameBuffer, msg: *mut i32) -> i32;
    pub fn vaco_av1_emit_frame_host(ctx: *mut Ctx, pic: *const Picture, info: *const FrameInfo, out: *const FrameBuffer, msg: *mut i32) -> i32;
    pub fn vaco_av1_postfilter_frame_emit_host(ctx: *mut Ctx, job: *const FrameJob, out: *const FrameBuffer, msg: *mut i32) -> i32;
    pub fn vaco_av1_film_grain_dev(ctx: *mut Ctx, stream: *mut c_void, in_: *const Picture, out: *const Picture, info: *const FrameInfo, params: *const FilmGrainParams, gaussian_sequence: *const i16, msg: *mut i32) -> i32;
    pub fn vaco_av1_film_grain_host(ctx: *mut Ctx, in_: *const Picture, out: *const Picture, info: *const FrameInfo, params: *const FilmGrainParams, gaussian_sequence: *const i16, msg: *mut i32) -> i32;
    pub fn vaco_av1_postfilter_frame_noalloc(stream: *mut c_void, job: *const FrameJob, msg: *mut i32) -> i32;
}
