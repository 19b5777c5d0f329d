//! `"gpu-pathtrace"` on a B200: the reference's progressive path-tracer API
//! (`GpuPathTracer`, `src/pathtrace.rs:309-725`; `Renderer`, `:1241-1264`;
//! `register_into`, `src/lib.rs:329-338`) over `liboxpt` instead of wgpu.
//! Not compiled here (no Rust toolchain on these machines).
//!
//! What stays the reference's: scene preparation (`PreparedScene`,
//! `TraceScene`, `EmissiveLights`, the camera and `radiance_key`) and the
//! word layouts `upload` writes (`src/pathtrace.rs:526-565, 970-1239`). They
//! are reached through [`ScenePreparer`], the one seam of this crate: the
//! reference's `upload` body, minus its `create_buffer_init` calls, is that
//! trait's implementation. What changes: buffers, dispatches and readback go
//! through `oxideav-render-cuda-sys`, and `draw_texture` hands out a
//! headless device image rather than a `wgpu::Texture`.
#![forbid(unsafe_code)]

use std::sync::Arc;

use oxideav_mesh3d::Scene3D;
use oxideav_render::pathtrace::EnvironmentMap;
use oxideav_render::{Error, HdrImage, RenderOptions, RenderRegistry, Renderer, Result, RgbaImage, TextureResolver};
use oxideav_render_cuda_sys as sys;

/// Registry name, as the reference's `PATHTRACE_BACKEND_NAME`.
pub const PATHTRACE_BACKEND_NAME: &str = "gpu-pathtrace";

/// Flat buffers of one prepared scene (the layouts of `include/oxpt.h`).
pub struct FlatScene {
    pub geom: Vec<u32>,
    pub attrs: Vec<f32>,
    pub atlas: Vec<u16>,
    pub atlas_side: u32,
    pub atlas_layers: u32,
    pub node_count: u32,
    pub slot_count: u32,
    /// Scene tables with the environment words appended.
    pub tables: Vec<u32>,
    /// `Params` for `opts` (size, camera, seed, bounces, offsets).
    pub params: sys::oxpt_params,
    /// The reference's `radiance_key`: options that change the estimate.
    pub radiance_key: u64,
}

/// The reference's scene preparation and `upload` word builders.
pub trait ScenePreparer: Send {
    fn prepare(&mut self, scene: &Scene3D, opts: &RenderOptions, env: Option<&Arc<EnvironmentMap>>,
               resolver: Option<&Arc<dyn TextureResolver>>) -> Result<FlatScene>;
}

/// A headless device image (device pointer as an integer, size, format):
/// what `draw_texture` returns without wgpu. Valid until the next call that
/// resizes or resolves.
#[derive(Clone, Copy, Debug)]
pub struct DeviceImage {
    pub address: usize,
    pub width: u32,
    pub height: u32,
    pub pitch_bytes: u32,
    pub hdr: bool,
}

fn backend(f: sys::Failure) -> Error {
    if f.is_invalid_options() {
        Error::InvalidOptions(f.message)
    } else {
        Error::Backend(f.message)
    }
}

/// Progressive path tracer on one CUDA device.
pub struct GpuPathTracer {
    ctx: sys::Ctx,
    prep: Box<dyn ScenePreparer>,
    env: Option<Arc<EnvironmentMap>>,
    resolver: Option<Arc<dyn TextureResolver>>,
    opts: Option<RenderOptions>,
    key: Option<u64>,
    dirty: bool,
    size: (u32, u32),
    samples: u32,
    target: u32,
    params: sys::oxpt_params,
}

impl GpuPathTracer {
    /// A tracer on CUDA device 0 with the given preparation.
    pub fn new(prep: Box<dyn ScenePreparer>) -> Result<Self> {
        Self::on_device(0, prep)
    }

    pub fn on_device(device: i32, prep: Box<dyn ScenePreparer>) -> Result<Self> {
        let ctx = sys::Ctx::new(device).map_err(backend)?;
        Ok(GpuPathTracer {
            ctx,
            prep,
            env: None,
            resolver: None,
            opts: None,
            key: None,
            dirty: true,
            size: (1, 1),
            samples: 0,
            target: 0,
            params: sys::oxpt_params::default(),
        })
    }

    pub fn adapter_summary(&self) -> String {
        self.ctx.device_summary()
    }

    /// `set_environment` (`:482`): the estimate changes, so the scene is
    /// prepared again and accumulation restarts.
    pub fn set_environment(&mut self, env: Option<Arc<EnvironmentMap>>) {
        self.env = env;
        self.invalidate_scene();
    }

    pub fn set_texture_resolver(&mut self, resolver: Arc<dyn TextureResolver>) {
        self.resolver = Some(resolver);
        self.invalidate_scene();
    }

    /// `invalidate_scene` (`:490`).
    pub fn invalidate_scene(&mut self) {
        self.dirty = true;
        self.samples = 0;
    }

    /// `reset` (`:495`): zero the accumulator, keep the scene.
    pub fn reset(&mut self) {
        self.samples = 0;
        let _ = self.ctx.reset();
    }

    pub fn samples(&self) -> u32 {
        self.samples
    }

    pub fn is_converged(&self) -> bool {
        self.target > 0 && self.samples >= self.target
    }

    pub fn size(&self) -> (u32, u32) {
        self.size
    }

    /// `sync` (`:526-565`): prepare and upload when the scene is dirty;
    /// restart accumulation when the radiance key changed; display-only
    /// options (tone map, exposure, background, spp target) never reset.
    /// Returns whether accumulation restarted.
    pub fn sync(&mut self, scene: &Scene3D, opts: &RenderOptions) -> Result<bool> {
        let mut restarted = false;
        if self.dirty {
            let flat = self.prep.prepare(scene, opts, self.env.as_ref(), self.resolver.as_ref())?;
            let words = sys::SceneWords {
                geom: &flat.geom,
                attrs: &flat.attrs,
                atlas: &flat.atlas,
                atlas_side: flat.atlas_side,
                atlas_layers: flat.atlas_layers,
                node_count: flat.node_count,
                slot_count: flat.slot_count,
            };
            self.ctx.upload(&words, &flat.tables).map_err(backend)?;
            self.params = flat.params;
            self.key = Some(flat.radiance_key);
            self.dirty = false;
            restarted = true;
        } else {
            let flat_key = self.prep.prepare(scene, opts, self.env.as_ref(), self.resolver.as_ref())?;
            if self.key != Some(flat_key.radiance_key) {
                self.params = flat_key.params;
                self.key = Some(flat_key.radiance_key);
                restarted = true;
            }
        }
        let size = (opts.width, opts.height);
        if size != self.size || restarted {
            self.ctx.resize(size.0, size.1).map_err(backend)?;
            self.ctx.set_params(&self.params).map_err(backend)?;
            self.ctx.reset().map_err(backend)?;
            self.size = size;
            self.samples = 0;
            restarted = true;
        }
        self.target = opts.path_trace.samples_per_pixel;
        self.opts = Some(opts.clone());
        Ok(restarted)
    }

    /// `refine` (`:584-671`): `samples` more samples of every pixel,
    /// queued (the call does not wait for the device).
    pub fn refine(&mut self, samples: u32) -> Result<()> {
        if self.opts.is_none() || samples == 0 {
            return Ok(());
        }
        let n = samples.min(u32::MAX - self.samples);
        self.ctx.refine(self.samples, n).map_err(backend)?;
        self.samples += n;
        Ok(())
    }

    /// `finish` (`:674`): wait for queued work; device-side errors surface here.
    pub fn finish(&mut self) -> Result<()> {
        self.ctx.finish().map_err(backend)
    }

    fn resolve_params(&self, hdr: bool) -> sys::oxpt_resolve_params {
        let o = self.opts.as_ref();
        let exposure = o.map(|o| o.exposure.max(0.0)).unwrap_or(1.0);
        let tone = o.map(|o| tone_map_code(o.tone_map)).unwrap_or(0);
        let bg = o.map(|o| o.background).unwrap_or([0, 0, 0, 255]);
        sys::oxpt_resolve_params {
            cfg: [1, 3, tone, hdr as u32],
            exposure: [exposure, self.samples as f32, self.size.0 as f32, 0.0],
            background: [bg[0] as f32 / 255.0, bg[1] as f32 / 255.0, bg[2] as f32 / 255.0, bg[3] as f32 / 255.0],
        }
    }

    /// `image` (`:695`): the tone-mapped RGBA8 frame (sRGB bytes).
    pub fn image(&mut self) -> Result<RgbaImage> {
        let (w, h) = self.size;
        let mut buf = vec![0u8; (w * h * 4) as usize];
        let p = self.resolve_params(false);
        self.ctx.resolve_into(&p, false, &mut buf).map_err(backend)?;
        RgbaImage::from_raw(w, h, buf).ok_or_else(|| Error::Backend("image size".into()))
    }

    /// `hdr` (`:710`): the linear mean radiance, RGBA32F.
    pub fn hdr(&mut self) -> Result<HdrImage> {
        let (w, h) = self.size;
        let mut buf = vec![0u8; (w * h * 16) as usize];
        let p = self.resolve_params(true);
        self.ctx.resolve_into(&p, true, &mut buf).map_err(backend)?;
        let px: Vec<f32> = buf.chunks_exact(4).map(|b| f32::from_le_bytes([b[0], b[1], b[2], b[3]])).collect();
        HdrImage::from_raw(w, h, px).ok_or_else(|| Error::Backend("image size".into()))
    }

    /// `draw_texture` (`:687`): the resolved RGBA8 frame left on the device.
    pub fn draw_texture(&mut self) -> Result<DeviceImage> {
        let p = self.resolve_params(false);
        let d = self.ctx.resolve_device(&p).map_err(backend)?;
        Ok(DeviceImage { address: d.data as usize, width: d.width, height: d.height, pitch_bytes: d.pitch_bytes,
                         hdr: d.format == sys::OXPT_FORMAT_RGBA32F })
    }

    /// Full render: re-prepare, take the target samples, resolve.
    fn run(&mut self, scene: &Scene3D, opts: &RenderOptions) -> Result<()> {
        self.invalidate_scene();
        self.sync(scene, opts)?;
        self.refine(opts.path_trace.samples_per_pixel.max(1))
    }
}

fn tone_map_code(t: oxideav_render::ToneMap) -> u32 {
    match t {
        oxideav_render::ToneMap::Reinhard => 1,
        oxideav_render::ToneMap::AcesFitted => 2,
        _ => 0,
    }
}

impl Renderer for GpuPathTracer {
    fn render(&mut self, scene: &Scene3D, opts: &RenderOptions) -> Result<RgbaImage> {
        self.run(scene, opts)?;
        self.image()
    }

    fn render_hdr(&mut self, scene: &Scene3D, opts: &RenderOptions) -> Result<HdrImage> {
        self.run(scene, opts)?;
        self.hdr()
    }

    fn set_texture_resolver(&mut self, resolver: Arc<dyn TextureResolver>) {
        GpuPathTracer::set_texture_resolver(self, resolver);
    }
}

/// Registers the path tracer under [`PATHTRACE_BACKEND_NAME`]; the factory
/// opens the device on each `make`, so registration never touches the GPU.
pub fn register_into(registry: &mut RenderRegistry, prep: fn() -> Box<dyn ScenePreparer>) {
    registry.register(
        PATHTRACE_BACKEND_NAME,
        Box::new(move || Ok(Box::new(GpuPathTracer::new(prep())?) as Box<dyn Renderer>)),
    );
}
