//! Raw bindings of `liboxpt.so` (`include/oxpt.h`) and a thin owning
//! wrapper. This is the only crate of the drop-in with `unsafe` code: the
//! path tracer crate on top of it forbids it, as the reference's crate does
//! (`src/lib.rs:72`). Not compiled here (no Rust toolchain on these
//! machines); the C side is what the repository builds and tests.
#![allow(non_camel_case_types)]

use std::ffi::CStr;
use std::os::raw::{c_char, c_int, c_void};

/// Opaque context: one CUDA stream and the scene's device buffers.
#[repr(C)]
pub struct oxpt_ctx {
    _p: [u8; 0],
}

/// The reference's `Params` uniform (`src/pathtrace.rs:100-114`), 176 bytes.
#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct oxpt_params {
    pub eye: [f32; 4],
    pub forward: [f32; 4],
    pub side: [f32; 4],
    pub up: [f32; 4],
    pub dims: [u32; 4],
    pub cfg: [u32; 4],
    pub env: [u32; 4],
    pub offs0: [u32; 4],
    pub offs1: [u32; 4],
    pub offs2: [u32; 4],
    pub fparams: [f32; 4],
}

/// `FrameParams` (`src/pathtrace.rs:116-123`).
#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct oxpt_frame {
    pub first: u32,
    pub count: u32,
    pub y0: u32,
    pub rows: u32,
}

/// `ResolveParams` (`src/pathtrace.rs:125-131`).
#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct oxpt_resolve_params {
    pub cfg: [u32; 4],
    pub exposure: [f32; 4],
    pub background: [f32; 4],
}

/// Flat scene buffers in the layouts `upload` writes (`src/pathtrace.rs:970-1239`).
#[repr(C)]
pub struct oxpt_scene_desc {
    pub geom: *const u32,
    pub geom_words: usize,
    pub attrs: *const f32,
    pub attr_floats: usize,
    pub atlas: *const u16,
    pub atlas_side: u32,
    pub atlas_layers: u32,
    pub node_count: u32,
    pub slot_count: u32,
}

/// A headless device image: what `draw_texture` returns in place of a
/// `wgpu::Texture`.
#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct oxpt_devimage {
    pub data: *mut c_void,
    pub width: u32,
    pub height: u32,
    pub pitch_bytes: u32,
    pub format: u32,
}

pub const OXPT_OK: c_int = 0;
pub const OXPT_E_NODEV: c_int = 1;
pub const OXPT_E_NOMEM: c_int = 2;
pub const OXPT_E_LIMIT: c_int = 3;
pub const OXPT_E_INVALID: c_int = 4;
pub const OXPT_E_TIMEOUT: c_int = 5;
pub const OXPT_E_CUDA: c_int = 6;
pub const OXPT_FORMAT_RGBA8: u32 = 0;
pub const OXPT_FORMAT_RGBA32F: u32 = 1;
pub const OXPT_ABI_VERSION: u32 = 2;

#[link(name = "oxpt")]
extern "C" {
    pub fn oxpt_abi_version() -> u32;
    pub fn oxpt_create(device: c_int, out: *mut *mut oxpt_ctx) -> c_int;
    pub fn oxpt_destroy(ctx: *mut oxpt_ctx) -> c_int;
    pub fn oxpt_last_error(ctx: *const oxpt_ctx) -> *const c_char;
    pub fn oxpt_device_summary(ctx: *const oxpt_ctx, buf: *mut c_char, len: usize) -> c_int;
    pub fn oxpt_upload_scene(ctx: *mut oxpt_ctx, scene: *const oxpt_scene_desc) -> c_int;
    pub fn oxpt_set_tables(ctx: *mut oxpt_ctx, words: *const u32, count: usize) -> c_int;
    pub fn oxpt_stage_scene(ctx: *mut oxpt_ctx, scene: *const oxpt_scene_desc, tables: *const u32,
                            table_words: usize) -> c_int;
    pub fn oxpt_set_params(ctx: *mut oxpt_ctx, params: *const oxpt_params) -> c_int;
    pub fn oxpt_resize(ctx: *mut oxpt_ctx, width: u32, height: u32) -> c_int;
    pub fn oxpt_reset(ctx: *mut oxpt_ctx) -> c_int;
    pub fn oxpt_dispatch(ctx: *mut oxpt_ctx, frame: *const oxpt_frame) -> c_int;
    pub fn oxpt_refine(ctx: *mut oxpt_ctx, first_sample: u32, count: u32) -> c_int;
    pub fn oxpt_finish(ctx: *mut oxpt_ctx) -> c_int;
    pub fn oxpt_resolve(ctx: *mut oxpt_ctx, params: *const oxpt_resolve_params, hdr: c_int,
                        host_out: *mut c_void, dev_out: *mut oxpt_devimage) -> c_int;
    pub fn oxpt_resolve_async(ctx: *mut oxpt_ctx, params: *const oxpt_resolve_params, hdr: c_int,
                              host_out: *mut c_void) -> c_int;
    pub fn oxpt_resolve_wait(ctx: *mut oxpt_ctx) -> c_int;
    pub fn oxpt_host_alloc(bytes: usize) -> *mut c_void;
    pub fn oxpt_host_free(p: *mut c_void);
    pub fn oxpt_read_accum(ctx: *mut oxpt_ctx, host_out: *mut f32) -> c_int;
}

/// A failed call: the status code and the context's last error message.
#[derive(Debug, Clone)]
pub struct Failure {
    pub status: c_int,
    pub message: String,
}

impl Failure {
    /// Whether the reference would report this as `Error::InvalidOptions`
    /// (bad arguments) rather than `Error::Backend`.
    pub fn is_invalid_options(&self) -> bool {
        self.status == OXPT_E_INVALID
    }
}

pub type Result<T> = std::result::Result<T, Failure>;

/// Flat scene words, borrowed for one upload.
pub struct SceneWords<'a> {
    pub geom: &'a [u32],
    pub attrs: &'a [f32],
    pub atlas: &'a [u16],
    pub atlas_side: u32,
    pub atlas_layers: u32,
    pub node_count: u32,
    pub slot_count: u32,
}

impl SceneWords<'_> {
    fn desc(&self) -> oxpt_scene_desc {
        oxpt_scene_desc {
            geom: self.geom.as_ptr(),
            geom_words: self.geom.len(),
            attrs: self.attrs.as_ptr(),
            attr_floats: self.attrs.len(),
            atlas: self.atlas.as_ptr(),
            atlas_side: self.atlas_side,
            atlas_layers: self.atlas_layers,
            node_count: self.node_count,
            slot_count: self.slot_count,
        }
    }
}

/// An owned context. Used from one thread at a time (`&mut self`), as the
/// reference's tracer is; distinct contexts on distinct threads are safe.
pub struct Ctx(*mut oxpt_ctx);

// The context is a handle to device state; moving it between threads is
// fine, sharing it is not (no `Sync`).
unsafe impl Send for Ctx {}

impl Ctx {
    /// `oxpt_create` on CUDA device `device`.
    pub fn new(device: i32) -> Result<Self> {
        let mut p = std::ptr::null_mut();
        let st = unsafe { oxpt_create(device, &mut p) };
        if st == OXPT_OK {
            Ok(Ctx(p))
        } else {
            Err(Failure { status: st, message: "no usable CUDA device".into() })
        }
    }

    fn check(&self, st: c_int) -> Result<()> {
        if st == OXPT_OK {
            return Ok(());
        }
        let msg = unsafe { CStr::from_ptr(oxpt_last_error(self.0)) };
        Err(Failure { status: st, message: msg.to_string_lossy().into_owned() })
    }

    pub fn device_summary(&self) -> String {
        let mut buf = [0 as c_char; 256];
        unsafe { oxpt_device_summary(self.0, buf.as_mut_ptr(), buf.len()) };
        unsafe { CStr::from_ptr(buf.as_ptr()) }.to_string_lossy().into_owned()
    }

    /// `upload` + `ensure_binding`'s table write: the library copies both;
    /// the slices may be dropped afterwards.
    pub fn upload(&mut self, scene: &SceneWords<'_>, tables: &[u32]) -> Result<()> {
        let d = scene.desc();
        self.check(unsafe { oxpt_upload_scene(self.0, &d) })?;
        self.check(unsafe { oxpt_set_tables(self.0, tables.as_ptr(), tables.len()) })
    }

    /// The next scene, uploaded while queued work keeps tracing the current
    /// one; the next refine traces it.
    pub fn stage(&mut self, scene: &SceneWords<'_>, tables: &[u32]) -> Result<()> {
        let d = scene.desc();
        self.check(unsafe { oxpt_stage_scene(self.0, &d, tables.as_ptr(), tables.len()) })
    }

    pub fn set_params(&mut self, p: &oxpt_params) -> Result<()> {
        self.check(unsafe { oxpt_set_params(self.0, p) })
    }

    pub fn resize(&mut self, width: u32, height: u32) -> Result<()> {
        self.check(unsafe { oxpt_resize(self.0, width, height) })
    }

    pub fn reset(&mut self) -> Result<()> {
        self.check(unsafe { oxpt_reset(self.0) })
    }

    pub fn dispatch(&mut self, f: &oxpt_frame) -> Result<()> {
        self.check(unsafe { oxpt_dispatch(self.0, f) })
    }

    pub fn refine(&mut self, first: u32, count: u32) -> Result<()> {
        self.check(unsafe { oxpt_refine(self.0, first, count) })
    }

    pub fn finish(&mut self) -> Result<()> {
        self.check(unsafe { oxpt_finish(self.0) })
    }

    /// RGBA8 (4 bytes a pixel) or RGBA32F (16) into `out`, blocking.
    pub fn resolve_into(&mut self, p: &oxpt_resolve_params, hdr: bool, out: &mut [u8]) -> Result<()> {
        let st = unsafe {
            oxpt_resolve(self.0, p, hdr as c_int, out.as_mut_ptr() as *mut c_void, std::ptr::null_mut())
        };
        self.check(st)
    }

    /// The resolved image left on the device (`draw_texture`).
    pub fn resolve_device(&mut self, p: &oxpt_resolve_params) -> Result<oxpt_devimage> {
        let mut d = oxpt_devimage { data: std::ptr::null_mut(), width: 0, height: 0, pitch_bytes: 0, format: 0 };
        self.check(unsafe { oxpt_resolve(self.0, p, 0, std::ptr::null_mut(), &mut d) })?;
        Ok(d)
    }

    pub fn read_accum(&mut self, out: &mut [f32]) -> Result<()> {
        self.check(unsafe { oxpt_read_accum(self.0, out.as_mut_ptr()) })
    }
}

impl Drop for Ctx {
    fn drop(&mut self) {
        unsafe {
            oxpt_destroy(self.0);
        }
    }
}
