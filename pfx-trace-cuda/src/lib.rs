//! The B200 path tracer behind pfx's `Trace` (crates/trace/src/gpu.rs), as a
//! Rust crate over libpfxtrace's C ABI (include/pfxt.h).
//!
//! `crates/trace` keeps its `SceneBuffers::build` or hands the scene to
//! `SceneBuffers::build` here; `Trace` mirrors the reference's methods with
//! the same argument meaning and the same error split (`TraceError::Refused`
//! for a device that cannot take the work, `TraceError::Setup` for invalid
//! input).  One `Trace` per thread: the methods take `&mut self`, as the
//! reference's do.
//!
//! This image has no Rust toolchain: the crate is written against the header
//! and has not been compiled here.

pub mod ffi;

use std::ffi::{CStr, CString};
use std::os::raw::{c_int, c_void};
use std::ptr;

/// TraceError (gpu.rs:269-307).
#[derive(Debug, Clone, PartialEq)]
pub enum TraceError {
    /// The device refused: no CUDA device, out of memory.
    Refused(String),
    /// Invalid scene, settings or arguments, or a failed device call.
    Setup(String),
}

impl std::fmt::Display for TraceError {
    fn fmt(&self, f: &mut std::fmt::Formatter<'_>) -> std::fmt::Result {
        match self {
            TraceError::Refused(m) => write!(f, "the GPU refused the trace: {m}"),
            TraceError::Setup(m) => write!(f, "{m}"),
        }
    }
}

impl std::error::Error for TraceError {}

fn last_error() -> String {
    // SAFETY: pfxt_last_error returns a NUL-terminated thread-local string.
    unsafe { CStr::from_ptr(ffi::pfxt_last_error()) }.to_string_lossy().into_owned()
}

fn check(code: c_int) -> Result<(), TraceError> {
    match code {
        ffi::PFXT_OK => Ok(()),
        ffi::PFXT_ERR_REFUSED => Err(TraceError::Refused(last_error())),
        _ => Err(TraceError::Setup(last_error())),
    }
}

/// Adaptive (adaptive.rs:10-26).
#[derive(Clone, Copy, Debug, PartialEq)]
pub struct Adaptive {
    pub threshold: f32,
    pub min_samples: u32,
    pub max_samples: u32,
    pub growth: f32,
}

impl Adaptive {
    fn raw(&self) -> ffi::PfxtAdaptive {
        ffi::PfxtAdaptive {
            threshold: self.threshold,
            min_samples: self.min_samples,
            max_samples: self.max_samples,
            growth: self.growth,
        }
    }

    /// Adaptive::rounds (adaptive.rs:46-63).
    pub fn rounds(&self) -> Result<Vec<u32>, TraceError> {
        let mut out = vec![0u32; 4096];
        let mut n = 0u32;
        // SAFETY: `out` holds `cap` entries.
        check(unsafe { ffi::pfxt_adaptive_rounds(&self.raw(), out.as_mut_ptr(), out.len() as u32, &mut n) })?;
        out.truncate(n as usize);
        Ok(out)
    }
}

/// Round (adaptive.rs:73-77).
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub struct Round {
    pub samples: u32,
    pub active: u64,
}

/// Converged (adaptive.rs:66-102).
#[derive(Clone, Debug, PartialEq)]
pub struct Converged {
    pub rounds: Vec<Round>,
    pub pixels: u64,
}

impl Converged {
    pub fn mean_samples(&self) -> f64 {
        if self.pixels == 0 {
            return 0.0;
        }
        let (mut total, mut before, mut running) = (0.0f64, 0u32, self.pixels);
        for r in &self.rounds {
            total += f64::from(r.samples - before) * running as f64;
            before = r.samples;
            running = r.active;
        }
        total / self.pixels as f64
    }

    pub fn converged(&self) -> bool {
        self.rounds.last().is_some_and(|r| r.active == 0)
    }
}

/// Output (gpu.rs:406-410): raw little-endian RGBA32F bytes of each film.
#[derive(Clone, Debug, PartialEq)]
pub struct Output {
    pub color: Vec<u8>,
    pub albedo: Vec<u8>,
    pub normal: Vec<u8>,
}

/// Stats (crates/gpu/src/pace.rs:66-70) of a paced call.
#[derive(Clone, Debug, PartialEq)]
pub struct Stats {
    pub milliseconds: Vec<f64>,
    pub wall_ms: f64,
}

/// SceneBuffers::build (gpu.rs:566-1061) on the host: the packed blobs of a
/// scene, kept for moving its instances later.
pub struct SceneBuffers {
    raw: *mut ffi::PfxtSceneBlobs,
    buffers: ffi::PfxtBuffers,
}

impl SceneBuffers {
    pub fn build(scene: &ffi::PfxtScene, settings: &ffi::PfxtSettings) -> Result<Self, TraceError> {
        let mut raw = ptr::null_mut();
        // SAFETY: the scene's arrays are read during the call only.
        check(unsafe { ffi::pfxt_scene_build(scene, settings, &mut raw) })?;
        let mut buffers = std::mem::MaybeUninit::<ffi::PfxtBuffers>::zeroed();
        // SAFETY: `raw` is a live handle; pfxt_scene_buffers fills every field.
        let buffers = unsafe {
            check(ffi::pfxt_scene_buffers(raw, buffers.as_mut_ptr())).inspect_err(|_| ffi::pfxt_scene_free(raw))?;
            buffers.assume_init()
        };
        Ok(Self { raw, buffers })
    }

    pub fn buffers(&self) -> &ffi::PfxtBuffers {
        &self.buffers
    }

    /// Trace::builds (gpu.rs:2356): (bottom-level BVHs built, top-level laid).
    pub fn builds(&self) -> Result<(u32, u32), TraceError> {
        let (mut bottom, mut top) = (0u32, 0u32);
        // SAFETY: live handle.
        check(unsafe { ffi::pfxt_scene_builds(self.raw, &mut bottom, &mut top) })?;
        Ok((bottom, top))
    }
}

impl Drop for SceneBuffers {
    fn drop(&mut self) {
        // SAFETY: the handle is owned and freed once.
        unsafe { ffi::pfxt_scene_free(self.raw) }
    }
}

/// The tracer (Trace, gpu.rs:309-342).
pub struct Trace {
    raw: *mut ffi::PfxtTrace,
    width: u32,
    height: u32,
}

impl Trace {
    /// Trace::new_detailed (gpu.rs:1926): uploads the packed scene and
    /// allocates the accumulation and the films.
    pub fn new(
        buffers: &SceneBuffers,
        scene: &ffi::PfxtScene,
        settings: &ffi::PfxtSettings,
        width: u32,
        height: u32,
    ) -> Result<Self, TraceError> {
        let mut raw = ptr::null_mut();
        // SAFETY: the blobs stay alive for the call; the library copies them.
        check(unsafe { ffi::pfxt_create(&buffers.buffers, scene, settings, width, height, &mut raw) })?;
        Ok(Self { raw, width, height })
    }

    fn pixels(&self) -> usize {
        self.width as usize * self.height as usize
    }

    /// Trace::sample (gpu.rs:2942).
    pub fn sample(&mut self, count: u32, seed: u32) -> Result<(), TraceError> {
        // SAFETY: live handle.
        check(unsafe { ffi::pfxt_sample(self.raw, count, seed) })
    }

    /// Trace::sample_paced (gpu.rs:2951): `between` gets each pass's device
    /// milliseconds.
    pub fn sample_paced<F: FnMut(f64)>(&mut self, count: u32, seed: u32, mut between: F) -> Result<Stats, TraceError> {
        unsafe extern "C" fn hook<F: FnMut(f64)>(user: *mut c_void, ms: f64) {
            // SAFETY: `user` is the &mut (F, Vec<f64>) passed below, alive for the call.
            let (f, seen) = unsafe { &mut *(user as *mut (&mut F, Vec<f64>)) };
            seen.push(ms);
            f(ms);
        }
        let mut state: (&mut F, Vec<f64>) = (&mut between, Vec::new());
        let mut wall = 0.0f64;
        // SAFETY: the trampoline and its state outlive the call.
        check(unsafe {
            ffi::pfxt_sample_paced(
                self.raw,
                count,
                seed,
                Some(hook::<F>),
                &mut state as *mut _ as *mut c_void,
                &mut wall,
            )
        })?;
        Ok(Stats { milliseconds: state.1, wall_ms: wall })
    }

    /// Trace::samples (gpu.rs:3233).
    pub fn samples(&self) -> u32 {
        // SAFETY: live handle.
        unsafe { ffi::pfxt_samples(self.raw) }
    }

    /// Trace::sample_adaptive (adaptive.rs:112-325).
    pub fn sample_adaptive(&mut self, adaptive: Adaptive, seed: u32) -> Result<Converged, TraceError> {
        let mut rounds = vec![ffi::PfxtRound::default(); 4096];
        let mut n = 0u32;
        // SAFETY: `rounds` holds `cap` entries.
        check(unsafe {
            ffi::pfxt_sample_adaptive(self.raw, &adaptive.raw(), seed, rounds.as_mut_ptr(), rounds.len() as u32, &mut n)
        })?;
        Ok(Converged {
            rounds: rounds[..n as usize].iter().map(|r| Round { samples: r.samples, active: r.active }).collect(),
            pixels: self.pixels() as u64,
        })
    }

    /// Trace::readback (gpu.rs:3240).
    pub fn readback(&mut self) -> Result<Output, TraceError> {
        let n = self.pixels() * 4;
        let (mut c, mut a, mut m) = (vec![0f32; n], vec![0f32; n], vec![0f32; n]);
        // SAFETY: each film holds width * height * 4 floats.
        check(unsafe { ffi::pfxt_readback(self.raw, c.as_mut_ptr(), a.as_mut_ptr(), m.as_mut_ptr()) })?;
        let bytes = |v: Vec<f32>| v.iter().flat_map(|x| x.to_le_bytes()).collect::<Vec<u8>>();
        Ok(Output { color: bytes(c), albedo: bytes(a), normal: bytes(m) })
    }

    /// sample_counts (adaptive.rs:328).
    pub fn sample_counts(&mut self) -> Result<Vec<u32>, TraceError> {
        let mut out = vec![0u32; self.pixels()];
        // SAFETY: `out` holds width * height entries.
        check(unsafe { ffi::pfxt_sample_counts(self.raw, out.as_mut_ptr()) })?;
        Ok(out)
    }

    /// Trace::set_camera (gpu.rs:2817); restarts the accumulation.
    pub fn set_camera(&mut self, camera: &ffi::PfxtCamera) -> Result<(), TraceError> {
        // SAFETY: live handle.
        check(unsafe { ffi::pfxt_set_camera(self.raw, camera) })
    }

    /// Trace::set_window (gpu.rs:2834).
    pub fn set_window(&mut self, full: [u32; 2], origin: [u32; 2]) -> Result<(), TraceError> {
        // SAFETY: two-element arrays, as the header asks.
        check(unsafe { ffi::pfxt_set_window(self.raw, full.as_ptr(), origin.as_ptr()) })
    }

    /// Trace::set_instance_transforms (gpu.rs:2422): column-major 4x4s for the
    /// first transforms.len() instances; returns whether any moved.
    pub fn set_instance_transforms(
        &mut self,
        buffers: &mut SceneBuffers,
        transforms: &[[[f32; 4]; 4]],
    ) -> Result<bool, TraceError> {
        let mut moved = 0u32;
        // SAFETY: [[f32; 4]; 4] is 16 contiguous f32 per instance.
        check(unsafe {
            ffi::pfxt_set_instance_transforms(
                self.raw,
                buffers.raw,
                transforms.as_ptr() as *const f32,
                transforms.len() as u32,
                &mut moved,
            )
        })?;
        Ok(moved != 0)
    }

    /// Trace::save + Saved::write_to (checkpoint.rs:82-158): the checkpoint
    /// bytes under `key`.
    pub fn save(&mut self, key: &str) -> Result<Vec<u8>, TraceError> {
        let key = CString::new(key).map_err(|_| TraceError::Setup("checkpoint key holds a NUL".into()))?;
        let mut need = 0usize;
        // SAFETY: a null buffer with capacity 0 asks for the size only.
        check(unsafe { ffi::pfxt_save(self.raw, key.as_ptr(), ptr::null_mut(), 0, &mut need) })?;
        let mut out = vec![0u8; need];
        // SAFETY: `out` holds `need` bytes.
        check(unsafe { ffi::pfxt_save(self.raw, key.as_ptr(), out.as_mut_ptr() as *mut c_void, need, &mut need) })?;
        out.truncate(need);
        Ok(out)
    }

    /// Saved::read_from + Trace::restore (checkpoint.rs:160-203).
    pub fn restore(&mut self, key: &str, bytes: &[u8]) -> Result<(), TraceError> {
        let key = CString::new(key).map_err(|_| TraceError::Setup("checkpoint key holds a NUL".into()))?;
        // SAFETY: `bytes` is read during the call only.
        check(unsafe { ffi::pfxt_restore(self.raw, key.as_ptr(), bytes.as_ptr() as *const c_void, bytes.len()) })
    }

    /// The colour, albedo and normal films in device memory, for a denoiser
    /// that reads them without a readback (gpu.rs:328-330).
    pub fn films_device(&mut self) -> Result<[*mut f32; 3], TraceError> {
        let mut f = [ptr::null_mut(); 3];
        // SAFETY: three out-pointers.
        check(unsafe { ffi::pfxt_films_device(self.raw, &mut f[0], &mut f[1], &mut f[2]) })?;
        Ok(f)
    }

    pub fn raw(&mut self) -> *mut ffi::PfxtTrace {
        self.raw
    }
}

impl Drop for Trace {
    fn drop(&mut self) {
        // SAFETY: the handle is owned and destroyed once.
        unsafe { ffi::pfxt_destroy(self.raw) }
    }
}

/// `pfx_denoise::Denoiser` (crates/denoise/src/lib.rs:58-361) on the GPU:
/// OIDN's RT filter with the weights the caller hands it (the reference
/// embeds `rt_hdr_alb_nrm.tza`).
pub struct Denoiser {
    raw: *mut ffi::PfxtDenoiser,
}

impl Denoiser {
    /// Denoiser::new (lib.rs:81-110).
    pub fn new(weights: &[u8]) -> Result<Self, TraceError> {
        let mut raw = ptr::null_mut();
        // SAFETY: the blob is read during the call only.
        check(unsafe { ffi::pfxt_denoiser_create(weights.as_ptr() as *const c_void, weights.len(), &mut raw) })?;
        Ok(Self { raw })
    }

    /// Denoiser::denoise (lib.rs:112-140): row-major RGBA pixels in and out.
    pub fn denoise(
        &mut self,
        width: u32,
        height: u32,
        color: &[[f32; 4]],
        albedo: &[[f32; 4]],
        normal: &[[f32; 4]],
    ) -> Result<Vec<[f32; 4]>, TraceError> {
        let pixels = width as usize * height as usize;
        if color.len() != pixels || albedo.len() != pixels || normal.len() != pixels {
            return Err(TraceError::Setup("image size mismatch".into()));
        }
        let mut out = vec![[0f32; 4]; pixels];
        // SAFETY: every image holds width * height RGBA pixels.
        check(unsafe {
            ffi::pfxt_denoise(
                self.raw,
                width,
                height,
                color.as_ptr() as *const f32,
                albedo.as_ptr() as *const f32,
                normal.as_ptr() as *const f32,
                out.as_mut_ptr() as *mut f32,
            )
        })?;
        Ok(out)
    }

    /// Denoiser::denoise_textures_into (lib.rs:157-183) with a trace's films:
    /// `out` is device memory of width * height RGBA32F, written on the
    /// trace's stream.
    pub fn denoise_trace_into(&mut self, trace: &mut Trace, out: *mut f32) -> Result<(), TraceError> {
        // SAFETY: `out` is the caller's device buffer of the trace's size.
        check(unsafe { ffi::pfxt_denoise_trace(self.raw, trace.raw(), out) })
    }

    /// Denoiser::tiles (lib.rs:112-116).
    pub fn tiles(&self) -> Option<(u32, u32, usize)> {
        let (mut w, mut h, mut n) = (0u32, 0u32, 0u32);
        // SAFETY: plain out-parameters.
        let ok = unsafe { ffi::pfxt_denoiser_tiles(self.raw, &mut w, &mut h, &mut n) } == 0;
        (ok && n > 0).then_some((w, h, n as usize))
    }
}

impl Drop for Denoiser {
    fn drop(&mut self) {
        // SAFETY: the handle is owned and destroyed once.
        unsafe { ffi::pfxt_denoiser_destroy(self.raw) }
    }
}
