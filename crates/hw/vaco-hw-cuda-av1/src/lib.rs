//! vaco's AV1 post-decode filters on an NVIDIA B200 (sm_100a), behind the
//! filter functions' own signatures.
//!
//! Each wrapper below is a drop-in for one function of `vaco-codec-av1`:
//!
//! | wrapper | replaces |
//! |---|---|
//! | [`restore_plane`] | `restoration::restore_plane` (src/restoration.rs:178) |
//! | [`upscale_plane`] | `superres::upscale_plane` (src/superres.rs:163) |
//! | [`upscale_picture`] | `superres::upscale_picture` (src/superres.rs:226) |
//! | [`find_direction`] | `cdef::find_direction` (src/cdef.rs:79), many blocks per call |
//! | [`filter_block`] | `cdef::filter_block` (src/cdef.rs:142), many blocks per call |
//! | [`cdef_picture`] | the frame pass of `apply_cdef` (src/decode.rs:739-862) |
//! | [`deblock_picture`] | AV1 §7.14 deblocking, which vaco does not implement |
//! | [`postfilter_frame`] | `decode_frame`'s filter tail (src/decode.rs:553-559) with deblocking in front |
//!
//! Ownership follows vaco: inputs are borrowed, outputs are allocated
//! through the caller's [`Budget`] before the library runs, so
//! `Error::LimitExceeded` keeps its meaning, and fuel is charged as the
//! scalar code charges it.  A library status maps back to
//! [`vaco_core::Error`] with vaco's own `&'static str` ([`to_error`]).
//!
//! This is the only crate of the decoder path that uses `unsafe` (D13 allows
//! it in the `vaco-hw-*` family); every block states why the call is sound.

pub mod ffi;

use core::ptr::NonNull;

use vaco_codec_av1::cdef::{CdefParams, FilterParams};
use vaco_codec_av1::framebuf::{Picture, Plane};
use vaco_codec_av1::restoration::{PlaneConfig, RestorationUnit};
use vaco_codec_av1::superres;
use vaco_core::{Error, Result};
use vaco_limits::Budget;

/// The message text of a library message id: vaco's own string where vaco
/// has the check, else the library's.
#[must_use]
pub fn message(msg: i32) -> &'static str {
    usize::try_from(msg).ok().and_then(|i| ffi::MESSAGES.get(i)).copied().unwrap_or("")
}

/// The `vaco_core::Error` of a library status.
///
/// - `INVALID_DATA` and `UNSUPPORTED` carry vaco's message, so a caller
///   matching on them sees exactly what the scalar path returns.
/// - `LIMIT_EXCEEDED` (a fixed scratch size, a full in-flight queue, or a
///   server's memory budget) is `Error::LimitExceeded`, its `limit` naming
///   which; the library does not report sizes, so `requested` and `cap` are 0.
/// - `DEVICE_ERROR` and `TIMEOUT` are failures of the device, not of the
///   input: `Error::Io`, which vaco's decode loop treats as unrecoverable.
#[must_use]
pub fn to_error(status: i32, msg: i32) -> Error {
    match status {
        ffi::INVALID_DATA => Error::InvalidData(message(msg)),
        ffi::UNSUPPORTED => Error::Unsupported(message(msg)),
        ffi::LIMIT_EXCEEDED => Error::LimitExceeded { limit: message(msg), requested: 0, cap: 0 },
        ffi::TIMEOUT => Error::Io(std::io::Error::new(std::io::ErrorKind::TimedOut, message(msg))),
        _ => Error::Io(std::io::Error::other(message(msg))),
    }
}

fn check(status: i32, msg: i32) -> Result<()> {
    if status == ffi::OK { Ok(()) } else { Err(to_error(status, msg)) }
}

fn dim(v: usize) -> Result<i32> {
    i32::try_from(v).map_err(|_| Error::InvalidData("AV1 GPU post-filter dimension exceeds i32"))
}

/// One library context on one CUDA device.  A context is used by one thread
/// at a time (`Send`, not `Sync`).
#[derive(Debug)]
pub struct Gpu {
    ctx: NonNull<ffi::Ctx>,
}

// SAFETY: a vaco_av1_ctx may move between threads; the library only requires
// that one thread uses it at a time, which `&mut self` on every call ensures.
unsafe impl Send for Gpu {}

impl Gpu {
    /// Creates a context on CUDA device `device`.
    ///
    /// # Errors
    /// `Error::Io` when the device cannot be used (no device, no driver).
    pub fn new(device: i32) -> Result<Self> {
        let mut raw = core::ptr::null_mut();
        // SAFETY: `raw` is a valid out-pointer for the duration of the call.
        let status = unsafe { ffi::vaco_av1_ctx_create(device, &mut raw) };
        check(status, 17)?;
        NonNull::new(raw).map(|ctx| Self { ctx }).ok_or_else(|| to_error(ffi::DEVICE_ERROR, 17))
    }

    fn raw(&mut self) -> *mut ffi::Ctx {
        self.ctx.as_ptr()
    }
}

impl Drop for Gpu {
    fn drop(&mut self) {
        // SAFETY: the context was created by vaco_av1_ctx_create and is
        // destroyed exactly once.
        unsafe { ffi::vaco_av1_ctx_destroy(self.ctx.as_ptr()) }
    }
}

/// Allocates a `width x height` plane through `budget` and fills it from the
/// library: `fill` receives a host buffer of `width * height` samples with
/// row pitch `width`.  `framebuf::Plane` exposes no mutable slice, so the
/// samples go through a transient staging buffer (charged to `budget` and
/// released) and `Plane::set`.
fn plane_from_library(
    budget: &mut Budget,
    width: usize,
    height: usize,
    fill: impl FnOnce(*mut u16) -> Result<()>,
) -> Result<Plane> {
    let mut out = Plane::new(budget, width, height)?;
    let n = width.saturating_mul(height);
    let mut staging: Vec<u16> = budget.alloc(n)?;
    let filled = fill(staging.as_mut_ptr());
    if filled.is_ok() && width > 0 {
        for (y, row) in staging.chunks(width).enumerate() {
            for (x, &v) in row.iter().enumerate() {
                out.set(x, y, v);
            }
        }
    }
    drop(staging);
    budget.release(u64::try_from(n.saturating_mul(2)).unwrap_or(u64::MAX));
    filled.map(|()| out)
}

fn lr_unit(u: &RestorationUnit) -> ffi::LrUnit {
    match *u {
        RestorationUnit::None => ffi::LrUnit::default(),
        RestorationUnit::Wiener { vertical, horizontal } => {
            ffi::LrUnit { kind: ffi::LR_WIENER, vertical, horizontal, ..ffi::LrUnit::default() }
        }
        RestorationUnit::SelfGuided { set, xqd } => {
            ffi::LrUnit { kind: ffi::LR_SGRPROJ, set: i16::from(set), xqd, ..ffi::LrUnit::default() }
        }
    }
}

/// Drop-in for `restoration::restore_plane` (src/restoration.rs:178-207).
///
/// # Errors
/// As vaco: `InvalidData` with vaco's message for bad geometry, depth, unit
/// count, coefficients or samples; `LimitExceeded` from `budget`.
pub fn restore_plane(
    gpu: &mut Gpu,
    before: &Plane,
    after: &Plane,
    config: PlaneConfig,
    units: &[RestorationUnit],
    budget: &mut Budget,
) -> Result<Plane> {
    let cfg = ffi::LrPlaneConfig {
        width: dim(config.width)?,
        height: dim(config.height)?,
        bit_depth: i32::from(config.bit_depth),
        unit_size: dim(config.unit_size)?,
        subsampling_y: i32::from(config.subsampling_y),
    };
    let c_units: Vec<ffi::LrUnit> = units.iter().map(lr_unit).collect();
    let (bw, bh, aw, ah) = (dim(before.width())?, dim(before.height())?, dim(after.width())?, dim(after.height())?);
    let n_units = dim(c_units.len())?;
    let ctx = gpu.raw();
    plane_from_library(budget, config.width, config.height, |out| {
        let mut msg = 0;
        // SAFETY: the planes' slices hold width x height samples each (Plane
        // has no padding); `c_units` holds `n_units` entries; `out` holds
        // config.width x config.height samples; the call is synchronous and
        // keeps no pointer.
        let status = unsafe {
            ffi::vaco_av1_restore_plane_host(
                ctx,
                before.as_slice().as_ptr(),
                bw,
                bh,
                after.as_slice().as_ptr(),
                aw,
                ah,
                &cfg,
                c_units.as_ptr(),
                n_units,
                out,
                &mut msg,
            )
        };
        check(status, msg)
    })
}

/// Drop-in for `superres::upscale_plane` (src/superres.rs:163-216).  Fuel:
/// `output_width` per row, as vaco charges it (:174), before the call.
///
/// # Errors
/// As vaco: `InvalidData` for bad depth, geometry or samples; budget errors.
pub fn upscale_plane(
    gpu: &mut Gpu,
    input: &Plane,
    config: superres::PlaneConfig,
    budget: &mut Budget,
) -> Result<Plane> {
    let (w, h) = (dim(input.width())?, dim(input.height())?);
    let (vis, out_w, rows) = (dim(config.visible_width)?, dim(config.output_width)?, dim(config.height)?);
    budget.consume_fuel(u64::try_from(config.output_width.saturating_mul(config.height)).unwrap_or(u64::MAX))?;
    let ctx = gpu.raw();
    plane_from_library(budget, config.output_width, config.height, |out| {
        let mut msg = 0;
        // SAFETY: `input` holds w x h samples; `out` holds output_width x
        // height samples; synchronous call, no pointer kept.
        let status = unsafe {
            ffi::vaco_av1_superres_upscale_plane_host(
                ctx,
                input.as_slice().as_ptr(),
                w,
                h,
                vis,
                out_w,
                rows,
                i32::from(config.bit_depth),
                out,
                &mut msg,
            )
        };
        check(status, msg)
    })
}

/// Drop-in for `superres::upscale_picture` (src/superres.rs:226-274): luma,
/// then U and V at the ceil-divided chroma geometry, in one launch; the
/// first plane that fails decides the error, as in vaco.
///
/// # Errors
/// As vaco, including "AV1 superres missing U/V plane".
pub fn upscale_picture(
    gpu: &mut Gpu,
    input: &Picture,
    config: superres::PictureConfig,
    budget: &mut Budget,
) -> Result<Picture> {
    let sx = usize::from(config.subsampling_x);
    let sy = usize::from(config.subsampling_y);
    let (cw, ch) = (config.upscaled_width.div_ceil(1 << sx), config.coded_height.div_ceil(1 << sy));
    let planes = if config.monochrome { 1 } else { 3 };
    let fuel = config.upscaled_width.saturating_mul(config.coded_height)
        + (planes - 1) * cw.saturating_mul(ch);
    budget.consume_fuel(u64::try_from(fuel).unwrap_or(u64::MAX))?;
    let mut out = Picture::new(budget, config.upscaled_width, config.coded_height, cw, ch, config.monochrome)?;
    let mut staging: Vec<Vec<u16>> = Vec::new();
    let mut pin = ffi::Picture::default();
    let mut pout = ffi::Picture::default();
    for k in 0..planes {
        let (w, h) = if k == 0 { (config.upscaled_width, config.coded_height) } else { (cw, ch) };
        let buf: Vec<u16> = budget.alloc(w.saturating_mul(h))?;
        staging.push(buf);
        if let (Some(p), Some(slot_in), Some(slot_out)) = (input.plane(k), pin.planes.get_mut(k), pout.planes.get_mut(k))
        {
            *slot_in = p.as_slice().as_ptr().cast_mut();
            *slot_out = staging.last_mut().map_or(core::ptr::null_mut(), Vec::as_mut_ptr);
            if let (Some(iw), Some(ih), Some(is)) = (pin.width.get_mut(k), pin.height.get_mut(k), pin.stride.get_mut(k)) {
                (*iw, *ih, *is) = (dim(p.width())?, dim(p.height())?, dim(p.width())?);
            }
            if let (Some(ow), Some(oh), Some(os)) = (pout.width.get_mut(k), pout.height.get_mut(k), pout.stride.get_mut(k))
            {
                (*ow, *oh, *os) = (dim(w)?, dim(h)?, dim(w.max(1))?);
            }
        }
    }
    let cfg = ffi::SuperresPictureConfig {
        coded_width: dim(config.coded_width)?,
        upscaled_width: dim(config.upscaled_width)?,
        coded_height: dim(config.coded_height)?,
        subsampling_x: i32::from(config.subsampling_x),
        subsampling_y: i32::from(config.subsampling_y),
        monochrome: i32::from(config.monochrome),
        bit_depth: i32::from(config.bit_depth),
    };
    let mut msg = 0;
    // SAFETY: every non-null plane pointer in `pin` is a live plane slice of
    // the stated width x height (pitch = width); every plane in `pout` is a
    // staging buffer of exactly the output extent; a missing input plane is
    // NULL, which the library reports as vaco does; synchronous call.
    let status = unsafe { ffi::vaco_av1_superres_upscale_picture_host(gpu.raw(), &pin, &pout, &cfg, &mut msg) };
    let result = check(status, msg);
    for (k, buf) in staging.iter().enumerate() {
        if let (Ok(()), Some(plane)) = (&result, out.plane_mut(k)) {
            let w = plane.width();
            if w > 0 {
                for (y, row) in buf.chunks(w).enumerate() {
                    for (x, &v) in row.iter().enumerate() {
                        plane.set(x, y, v);
                    }
                }
            }
        }
        budget.release(u64::try_from(buf.len().saturating_mul(2)).unwrap_or(u64::MAX));
    }
    result.map(|()| out)
}

/// `cdef::find_direction` (src/cdef.rs:79-124) over many 8x8 blocks in one
/// call: `(direction, variance)` per block.
///
/// # Errors
/// As vaco: `InvalidData` for a bad depth or a sample above it.
pub fn find_direction(gpu: &mut Gpu, blocks: &[[u16; 64]], bit_depth: u8) -> Result<Vec<(u8, u32)>> {
    let n = dim(blocks.len())?;
    let mut dirs = vec![0u8; blocks.len()];
    let mut vars = vec![0u32; blocks.len()];
    let mut msg = 0;
    // SAFETY: `blocks` is n x 64 contiguous samples; `dirs` and `vars` hold n
    // entries each; synchronous call.
    let status = unsafe {
        ffi::vaco_av1_cdef_find_direction_host(
            gpu.raw(),
            blocks.as_ptr().cast(),
            n,
            i32::from(bit_depth),
            dirs.as_mut_ptr(),
            vars.as_mut_ptr(),
            &mut msg,
        )
    };
    check(status, msg)?;
    Ok(dirs.into_iter().zip(vars).collect())
}

/// `cdef::filter_block` (src/cdef.rs:142-205) over many 12x12 neighbourhoods
/// in one call.
///
/// # Errors
/// As vaco: `InvalidData` ("invalid CDEF block parameters", samples).
pub fn filter_block(gpu: &mut Gpu, inputs: &[[u16; 144]], params: &[FilterParams]) -> Result<Vec<[u16; 64]>> {
    if inputs.len() != params.len() {
        return Err(Error::InvalidData("invalid CDEF block parameters"));
    }
    let c_params: Vec<ffi::CdefFilterParams> = params
        .iter()
        .map(|p| ffi::CdefFilterParams {
            width: u8::try_from(p.width).unwrap_or(u8::MAX),
            height: u8::try_from(p.height).unwrap_or(u8::MAX),
            edges: p.edges,
            bit_depth: p.bit_depth,
            direction: p.direction,
            damping: p.damping,
            primary: p.primary,
            secondary: p.secondary,
        })
        .collect();
    let mut out = vec![[0u16; 64]; inputs.len()];
    let mut msg = 0;
    // SAFETY: `inputs` is n x 144 contiguous samples, `c_params` n entries,
    // `out` n x 64 samples; synchronous call.
    let status = unsafe {
        ffi::vaco_av1_cdef_filter_block_host(
            gpu.raw(),
            inputs.as_ptr().cast(),
            c_params.as_ptr(),
            dim(inputs.len())?,
            out.as_mut_ptr().cast(),
            &mut msg,
        )
    };
    check(status, msg)?;
    Ok(out)
}

/// Frame geometry of the picture-level calls: the header's
/// `vaco_av1_frame_info` (luma Mi grid, visible and upscaled sizes).
pub use ffi::FrameInfo;

fn c_cdef_params(p: &CdefParams) -> ffi::CdefParams {
    let mut c = ffi::CdefParams { enabled: u8::from(p.enabled), damping: p.damping, ..ffi::CdefParams::default() };
    for (i, (y, uv)) in p.y.iter().zip(p.uv.iter()).enumerate() {
        if let (Some(yp), Some(ys), Some(up), Some(us)) = (
            c.y_primary.get_mut(i),
            c.y_secondary.get_mut(i),
            c.uv_primary.get_mut(i),
            c.uv_secondary.get_mut(i),
        ) {
            (*yp, *ys, *up, *us) = (y.primary, y.secondary, uv.primary, uv.secondary);
        }
    }
    c
}

/// A host picture as the library's descriptor (pitch = width: `Plane` has no
/// padding).
fn c_picture(p: &Picture) -> Result<ffi::Picture> {
    let mut c = ffi::Picture::default();
    for k in 0..3 {
        if let (Some(plane), Some(ptr), Some(w), Some(h), Some(s)) =
            (p.plane(k), c.planes.get_mut(k), c.width.get_mut(k), c.height.get_mut(k), c.stride.get_mut(k))
        {
            *ptr = plane.as_slice().as_ptr().cast_mut();
            (*w, *h, *s) = (dim(plane.width())?, dim(plane.height())?, dim(plane.width())?);
        }
    }
    Ok(c)
}

/// A picture shaped like `like`, allocated through `budget`, with host
/// staging buffers the library writes; `finish` copies them in (or drops
/// them on error) and releases the staging bytes.
struct Staged {
    bufs: Vec<Vec<u16>>,
    desc: ffi::Picture,
}

impl Staged {
    fn like(like: &Picture, budget: &mut Budget) -> Result<Self> {
        let mut bufs = Vec::new();
        let mut desc = ffi::Picture::default();
        for k in 0..3 {
            if let Some(plane) = like.plane(k) {
                let mut buf: Vec<u16> = budget.alloc(plane.width().saturating_mul(plane.height()))?;
                if let (Some(ptr), Some(w), Some(h), Some(s)) =
                    (desc.planes.get_mut(k), desc.width.get_mut(k), desc.height.get_mut(k), desc.stride.get_mut(k))
                {
                    *ptr = buf.as_mut_ptr();
                    (*w, *h, *s) = (dim(plane.width())?, dim(plane.height())?, dim(plane.width())?);
                }
                bufs.push(buf);
            }
        }
        Ok(Self { bufs, desc })
    }

    fn finish(self, result: Result<()>, mut out: Picture, budget: &mut Budget) -> Result<Picture> {
        for (k, buf) in self.bufs.iter().enumerate() {
            if let (Ok(()), Some(plane)) = (&result, out.plane_mut(k)) {
                let w = plane.width();
                if w > 0 {
                    for (y, row) in buf.chunks(w).enumerate() {
                        for (x, &v) in row.iter().enumerate() {
                            plane.set(x, y, v);
                        }
                    }
                }
            }
            budget.release(u64::try_from(buf.len().saturating_mul(2)).unwrap_or(u64::MAX));
        }
        result.map(|()| out)
    }
}

fn new_like(like: &Picture, budget: &mut Budget) -> Result<Picture> {
    let (cw, ch) = like.u.as_ref().map_or((0, 0), |u| (u.width(), u.height()));
    Picture::new(budget, like.y.width(), like.y.height(), cw, ch, like.u.is_none())
}

/// The frame pass of `apply_cdef` (src/decode.rs:739-862) with its inputs
/// explicit: `skip` holds one flag per 4x4 luma cell (`MiCell.skip`),
/// `cdef_idx` one strength index per 64x64 (-1 = none), row stride
/// `cdef_stride`.  Fuel: 1 per filtered 8x8 block, as decode.rs:788.
///
/// # Errors
/// As vaco's CDEF: `InvalidData` with vaco's messages.
pub fn cdef_picture(
    gpu: &mut Gpu,
    pic: &Picture,
    info: &FrameInfo,
    skip: &[u8],
    cdef_idx: &[i32],
    cdef_stride: usize,
    params: &CdefParams,
    budget: &mut Budget,
) -> Result<Picture> {
    budget.consume_fuel(filtered_blocks(info, skip, cdef_idx, cdef_stride, params))?;
    let src = c_picture(pic)?;
    let out = new_like(pic, budget)?;
    let staged = Staged::like(pic, budget)?;
    let c_params = c_cdef_params(params);
    let mut msg = 0;
    // SAFETY: `src` describes live planes of `pic`, `staged.desc` live
    // staging buffers of the same extents; `skip` and `cdef_idx` are live
    // slices the library reads within the frame's Mi grid; synchronous call.
    let status = unsafe {
        ffi::vaco_av1_cdef_picture_host(
            gpu.raw(),
            &src,
            &staged.desc,
            info,
            skip.as_ptr(),
            cdef_idx.as_ptr(),
            dim(cdef_stride)?,
            dim(cdef_idx.len())?,
            &c_params,
            &mut msg,
        )
    };
    staged.finish(check(status, msg), out, budget)
}

/// 8x8 blocks `apply_cdef` filters (and charges one fuel unit for): not all
/// four 4x4 cells skipped, index present (src/decode.rs:772-788).
fn filtered_blocks(info: &FrameInfo, skip: &[u8], cdef_idx: &[i32], cdef_stride: usize, params: &CdefParams) -> u64 {
    if !params.enabled {
        return 0;
    }
    let rows = usize::try_from(info.mi_rows).unwrap_or(0);
    let cols = usize::try_from(info.mi_cols).unwrap_or(0);
    let skipped = |r: usize, c: usize| r >= rows || c >= cols || skip.get(r * cols + c).is_some_and(|&s| s != 0);
    let mut n = 0u64;
    for r in (0..rows).step_by(2) {
        for c in (0..cols).step_by(2) {
            let idx = cdef_idx.get((r >> 4) * cdef_stride + (c >> 4)).copied().unwrap_or(-1);
            let all_skip = skipped(r, c) && skipped(r + 1, c) && skipped(r, c + 1) && skipped(r + 1, c + 1);
            if idx >= 0 && !all_skip {
                n += 1;
            }
        }
    }
    n
}

/// AV1 §7.14 deblocking of an intra frame (vaco has none): `tx_luma` /
/// `tx_chroma` hold one TX_SIZE per 4x4 cell, `lvl_map` optionally four
/// final levels (Y vertical, Y horizontal, U, V) per luma cell.
///
/// # Errors
/// `InvalidData` for bad levels, transform sizes or samples.
pub fn deblock_picture(
    gpu: &mut Gpu,
    pic: &Picture,
    info: &FrameInfo,
    tx_luma: &[u8],
    tx_chroma: &[u8],
    lvl_map: Option<&[[u8; 4]]>,
    levels: [u8; 4],
    sharpness: u8,
    budget: &mut Budget,
) -> Result<Picture> {
    let src = c_picture(pic)?;
    let out = new_like(pic, budget)?;
    let staged = Staged::like(pic, budget)?;
    let params = ffi::DeblockParams { levels, sharpness, reserved: [0; 3] };
    let mut msg = 0;
    // SAFETY: as cdef_picture; `lvl_map`, when given, holds 4 bytes per luma
    // cell; synchronous call.
    let status = unsafe {
        ffi::vaco_av1_deblock_picture_host(
            gpu.raw(),
            &src,
            &staged.desc,
            info,
            tx_luma.as_ptr(),
            tx_chroma.as_ptr(),
            lvl_map.map_or(core::ptr::null(), |m| m.as_ptr().cast()),
            &params,
            &mut msg,
        )
    };
    staged.finish(check(status, msg), out, budget)
}

/// Everything `decode_frame` hands the post-filters (src/decode.rs:553-559),
/// with deblocking's inputs in front.
#[derive(Debug)]
pub struct FrameSide<'a> {
    pub info: FrameInfo,
    pub tx_luma: &'a [u8],
    pub tx_chroma: &'a [u8],
    pub lvl_map: Option<&'a [[u8; 4]]>,
    pub levels: [u8; 4],
    pub sharpness: u8,
    pub skip: &'a [u8],
    pub cdef_idx: &'a [i32],
    pub cdef_stride: usize,
    pub cdef: CdefParams,
    /// Per plane: frame restoration type (`ffi::FRAME_LR_*`), unit size, units.
    pub restoration: [(i32, usize, &'a [RestorationUnit]); 3],
}

/// Deblocking -> CDEF -> superres -> loop restoration of one frame; the
/// result is the visible picture vaco's `decode_frame` hands `pic_to_frame`
/// (upscaled_width x coded_height, chroma by the subsampling).
///
/// # Errors
/// The first error vaco's stages would meet, in stage order.
pub fn postfilter_frame(gpu: &mut Gpu, pic: &Picture, side: &FrameSide<'_>, budget: &mut Budget) -> Result<Picture> {
    budget.consume_fuel(filtered_blocks(&side.info, side.skip, side.cdef_idx, side.cdef_stride, &side.cdef))?;
    let i = side.info;
    let (sx, sy) = (usize::try_from(i.subsampling_x).unwrap_or(0), usize::try_from(i.subsampling_y).unwrap_or(0));
    let (w, h) = (usize::try_from(i.upscaled_width).unwrap_or(0), usize::try_from(i.coded_height).unwrap_or(0));
    let out = Picture::new(budget, w, h, w >> sx, h >> sy, i.monochrome != 0)?;
    let staged = Staged::like(&out, budget)?;
    let units: Vec<Vec<ffi::LrUnit>> =
        side.restoration.iter().map(|(_, _, u)| u.iter().map(lr_unit).collect()).collect();
    let mut job = ffi::FrameJob {
        info: i,
        src: c_picture(pic)?,
        dst: staged.desc,
        tx_luma: side.tx_luma.as_ptr(),
        tx_chroma: side.tx_chroma.as_ptr(),
        lvl_map: side.lvl_map.map_or(core::ptr::null(), |m| m.as_ptr().cast()),
        skip: side.skip.as_ptr(),
        cdef_idx: side.cdef_idx.as_ptr(),
        cdef_stride: dim(side.cdef_stride)?,
        cdef_count: dim(side.cdef_idx.len())?,
        deblock: ffi::DeblockParams { levels: side.levels, sharpness: side.sharpness, reserved: [0; 3] },
        cdef: c_cdef_params(&side.cdef),
        ..ffi::FrameJob::default()
    };
    for (k, ((kind, size, _), u)) in side.restoration.iter().zip(units.iter()).enumerate() {
        if let (Some(t), Some(s), Some(p), Some(n)) =
            (job.lr_type.get_mut(k), job.lr_unit_size.get_mut(k), job.lr_units.get_mut(k), job.lr_unit_count.get_mut(k))
        {
            (*t, *s, *p, *n) = (*kind, dim(*size)?, u.as_ptr(), dim(u.len())?);
        }
    }
    let mut msg = 0;
    // SAFETY: every pointer in `job` is a live host slice or plane of the
    // extents the job states (the library checks the geometry first), the
    // destination planes are the staging buffers; synchronous call.
    let status = unsafe { ffi::vaco_av1_postfilter_frame_host(gpu.raw(), &job, &mut msg) };
    staged.finish(check(status, msg), out, budget)
}

#[cfg(test)]
mod tests {
    use super::ffi;

    #[test]
    fn message_table_matches_library() {
        for (id, text) in ffi::MESSAGES.iter().enumerate() {
            let id = i32::try_from(id).unwrap_or(i32::MAX);
            // SAFETY: vaco_av1_message returns a static NUL-terminated string.
            let lib = unsafe { core::ffi::CStr::from_ptr(ffi::vaco_av1_message(id)) };
            assert_eq!(lib.to_str().ok(), Some(*text));
        }
    }

    #[test]
    fn limit_exceeded_keeps_its_variant() {
        assert!(matches!(super::to_error(ffi::LIMIT_EXCEEDED, 18), vaco_core::Error::LimitExceeded { .. }));
        assert!(matches!(super::to_error(ffi::INVALID_DATA, 7), vaco_core::Error::InvalidData(m) if Some(&m) == ffi::MESSAGES.get(7)));
    }
}
