//! # vxl-phys-gpu-b200
//!
//! The WCSPH fluid step of `vxl-phys-fluid` on an NVIDIA B200 (sm_100a), behind the traits
//! the facade already drives: [`FluidStepper`] (crates/vxl-phys-core/src/interop.rs:293-316)
//! and [`PhysGpuBackend`] (crates/vxl-phys-gpu/src/lib.rs:20-29). The work runs in
//! libvxl_sph (CUDA), reached through its C ABI ([`ffi`]); this crate converts the trait's
//! slices and tuples to the ABI's arrays and checks every status.
//!
//! Registration follows the GPU tier's own probe (crates/vxl-phys-gpu/examples/
//! gpu_facade_probe.rs:120-130):
//!
//! ```ignore
//! let f = &world.fluids()[fi].0;
//! let (pos, vel, pmass, nf) = f.raw_particles();
//! let st = B200FluidStepper::new(f.config(), f.particle_mass(), nf, pos, vel, pmass, 0)
//!     .expect("B200 fluid stepper");
//! world.set_fluid_stepper(fi, Box::new(st));
//! ```
//!
//! Errors: a length mismatch in `step` panics, as `GpuFluidStepper::step` asserts
//! (crates/vxl-phys-gpu/src/pipeline/stepper.rs:80-96, coupling.rs:22-33); any other
//! non-OK status of the library panics with its message from `vxl_sph_last_error`, since
//! the trait has no error channel and a failed tick must not hand stale reactions to the
//! facade. Fallible construction returns [`B200Error`].

pub mod ffi;

use std::ffi::CStr;
use std::ptr::NonNull;

use vxl_phys_core::interop::{FluidStepper, InteropContact, ProviderColliders};
use vxl_phys_core::Vec3;
use vxl_phys_fluid::FluidConfig;
use vxl_phys_gpu::PhysGpuBackend;

/// A non-OK status of libvxl_sph with its message.
#[derive(Debug, Clone)]
pub struct B200Error {
    pub status: u32,
    pub message: String,
}

impl std::fmt::Display for B200Error {
    fn fmt(&self, f: &mut std::fmt::Formatter<'_>) -> std::fmt::Result {
        write!(f, "libvxl_sph status {}: {}", self.status, self.message)
    }
}

impl std::error::Error for B200Error {}

fn last_error() -> String {
    // SAFETY: the library returns a NUL-terminated string it owns (thread-local), or NULL.
    unsafe {
        let p = ffi::vxl_sph_last_error();
        if p.is_null() {
            String::new()
        } else {
            CStr::from_ptr(p).to_string_lossy().into_owned()
        }
    }
}

/// Ok for status 0, the status and the library's message otherwise.
pub fn check(status: u32) -> Result<(), B200Error> {
    if status == ffi::OK {
        Ok(())
    } else {
        Err(B200Error { status, message: last_error() })
    }
}

fn must(status: u32, what: &str) {
    if let Err(e) = check(status) {
        panic!("{what}: {e}");
    }
}

fn flat(v: &[Vec3]) -> *const f32 {
    // Vec3 is #[repr(C)] {x, y, z: f32} (crates/vxl-phys-core/src/math.rs:8-14)
    v.as_ptr() as *const f32
}

/// The library's parameters for a fluid of this configuration and particle mass
/// (`FluidSystem::mass`, fluid_access.rs:27-42); field meanings are FluidConfig's.
pub fn params_of(cfg: &FluidConfig, mass: f32) -> ffi::Params {
    ffi::Params {
        hdr: ffi::BlockHeader::of::<ffi::Params>(),
        rest_density: cfg.rest_density,
        smoothing_radius: cfg.smoothing_radius,
        xsph_viscosity: cfg.xsph_viscosity,
        tensile_instability_suppression: cfg.tensile_instability_suppression as u32,
        sound_speed: cfg.sound_speed,
        gamma_tait: cfg.gamma_tait,
        substeps: cfg.substeps,
        boundary_layers: cfg.boundary_layers,
        gravity: [cfg.gravity.x, cfg.gravity.y, cfg.gravity.z],
        max_speed_frac: cfg.max_speed_frac,
        artificial_viscosity: cfg.artificial_viscosity,
        particle_mass: mass,
        max_bins: 0,
    }
}

/// `FluidStepper` on a B200: the resident scene owns the fluid state (the host copy is
/// scaffolding, interop.rs:290-292); each `step` uploads the boundary segment and steps
/// one tick; `gather_walls` feeds provider walls of any kind as contact tables.
pub struct B200FluidStepper {
    h: NonNull<ffi::Handle>,
    n_fluid: usize,
    nb: usize,
    boundaries: Vec<u32>,
    spans: Vec<ffi::Span>,
    raw: Vec<ffi::Reaction>,
    out: Vec<(u32, Vec3, Vec3)>,
    scratch: Vec<InteropContact>,
}

impl B200FluidStepper {
    /// Build once from the full particle set (fluid prefix + boundary segment), as
    /// `GpuFluidStepper::new` does (stepper.rs:36-61), on CUDA device `device`.
    pub fn new(cfg: &FluidConfig, mass: f32, n_fluid: usize, pos: &[Vec3], vel: &[Vec3], pmass: &[f32],
               device: i32) -> Result<Self, B200Error> {
        assert_eq!(pos.len(), vel.len(), "pos and vel lengths differ");
        assert_eq!(pos.len(), pmass.len(), "pos and pmass lengths differ");
        assert!(n_fluid <= pos.len(), "fluid prefix longer than the particle set");
        let desc = ffi::Desc {
            hdr: ffi::BlockHeader::of::<ffi::Desc>(),
            params: params_of(cfg, mass),
            n_fluid: n_fluid as u64,
            n_boundary: (pos.len() - n_fluid) as u64,
            pos_xyz: flat(pos),
            vel_xyz: flat(vel),
            pmass: pmass.as_ptr(),
            device,
        };
        let mut h: *mut ffi::Handle = std::ptr::null_mut();
        // SAFETY: desc points at slices that outlive the call; the library copies them.
        check(unsafe { ffi::vxl_sph_create(&desc, &mut h) })?;
        let h = NonNull::new(h).ok_or(B200Error { status: ffi::NULL_POINTER, message: "no handle".into() })?;
        Ok(Self {
            h,
            n_fluid,
            nb: pos.len() - n_fluid,
            boundaries: Vec::new(),
            spans: Vec::new(),
            raw: Vec::new(),
            out: Vec::new(),
            scratch: Vec::new(),
        })
    }

    /// The provider ids of the fluid's walls (`FluidSystem::set_boundaries`), queried by
    /// `gather_walls` (the `boundaries` of GpuFluidStepper, stepper.rs:27, 42).
    pub fn with_boundaries(mut self, boundaries: Vec<u32>) -> Self {
        self.boundaries = boundaries;
        self
    }

    /// Raw handle for the rest of the C ABI (batched/served forms, exports, tuning).
    pub fn handle(&self) -> *mut ffi::Handle {
        self.h.as_ptr()
    }

    /// One side of the contact tables for positions `ps` (gather_in,
    /// crates/vxl-phys-gpu/src/pipeline/walls.rs:164-215): per fluid particle the planes of
    /// every provider within bounds + h, mirror 0 < sdf < h / projection sdf < h, <= 8.
    fn gather(&mut self, h: f32, ps: &[Vec3], providers: &dyn ProviderColliders, side: u32)
              -> (Vec<u32>, Vec<u32>, Vec<f32>) {
        let (mut ids, mut start, mut planes) = (Vec::new(), vec![0u32], Vec::new());
        for (i, &p) in ps.iter().enumerate() {
            let mut np = 0usize;
            for &bid in &self.boundaries {
                if let Some(bb) = providers.bounds(bid) {
                    if p.x < bb.min.x - h || p.x > bb.max.x + h || p.y < bb.min.y - h || p.y > bb.max.y + h
                        || p.z < bb.min.z - h || p.z > bb.max.z + h
                    {
                        continue;
                    }
                }
                self.scratch.clear();
                let hit = if side == ffi::WALLS_MIRROR {
                    providers.contacts_point(bid, p, h, &mut self.scratch)
                } else {
                    providers.contacts_point_boundary(bid, p, h, &mut self.scratch)
                };
                if !hit {
                    continue;
                }
                for c in &self.scratch {
                    let sdf = (p - c.point).dot(c.normal);
                    let keep = if side == ffi::WALLS_MIRROR { sdf > 0.0 && sdf < h } else { sdf < h };
                    if keep && np < 8 {
                        planes.extend_from_slice(&[c.point.x, c.point.y, c.point.z, c.normal.x, c.normal.y,
                                                   c.normal.z]);
                        np += 1;
                    }
                }
            }
            if np > 0 {
                ids.push(i as u32);
                start.push((planes.len() / 6) as u32);
            }
        }
        (ids, start, planes)
    }
}

impl Drop for B200FluidStepper {
    fn drop(&mut self) {
        // SAFETY: the handle came from vxl_sph_create and is destroyed once.
        unsafe {
            ffi::vxl_sph_destroy(self.h.as_ptr());
        }
    }
}

impl FluidStepper for B200FluidStepper {
    fn step(&mut self, dt_tick: f32, n_fluid: usize, pos: &[Vec3], vel: &[Vec3], pmass: &[f32],
            spans: &[(u32, Vec3, u32, u32)]) {
        // length checks of GpuFluidStepper::step (stepper.rs:84-96): errors, not truncation
        assert_eq!(n_fluid, self.n_fluid, "fluid prefix changed since the stepper was built");
        assert_eq!(pos.len(), n_fluid + self.nb, "particle count differs from the stepper's");
        assert_eq!(vel.len(), pos.len(), "vel length differs from pos");
        assert_eq!(pmass.len(), pos.len(), "pmass length differs from pos");
        if self.nb > 0 {
            // SAFETY: the boundary slices hold nb Vec3 each.
            must(unsafe {
                ffi::vxl_sph_upload_boundary(self.h.as_ptr(), n_fluid as u64, flat(&pos[n_fluid..]),
                                             flat(&vel[n_fluid..]), self.nb as u64)
            }, "vxl_sph_upload_boundary");
        }
        self.spans.clear();
        self.spans.extend(spans.iter().map(|s| ffi::Span { body: s.0, origin: [s.1.x, s.1.y, s.1.z], start: s.2,
                                                           end: s.3 }));
        self.raw.clear();
        self.raw.resize(self.spans.len(), ffi::Reaction::default());
        // SAFETY: spans and raw hold nspans entries each.
        must(unsafe {
            ffi::vxl_sph_step_tick(self.h.as_ptr(), dt_tick, self.spans.as_ptr(), self.spans.len() as u32,
                                   self.raw.as_mut_ptr())
        }, "vxl_sph_step_tick");
        self.out.clear();
        self.out.extend(self.raw.iter().map(|r| {
            (r.body, Vec3::new(r.force[0], r.force[1], r.force[2]), Vec3::new(r.torque[0], r.torque[1], r.torque[2]))
        }));
    }

    fn reactions(&self) -> &[(u32, Vec3, Vec3)] {
        &self.out
    }

    fn bounds(&self) -> Option<(Vec3, Vec3)> {
        let (mut lo, mut hi) = ([0f32; 3], [0f32; 3]);
        // SAFETY: lo and hi hold three floats each.
        let st = unsafe { ffi::vxl_sph_bounds(self.h.as_ptr(), lo.as_mut_ptr(), hi.as_mut_ptr()) };
        if st == ffi::NOT_READY {
            return None; // no fluid bounds yet: the caller falls back to its host copy
        }
        must(st, "vxl_sph_bounds");
        Some((Vec3::new(lo[0], lo[1], lo[2]), Vec3::new(hi[0], hi[1], hi[2])))
    }

    /// Provider walls of any kind (GpuFluidStepper::gather_walls, stepper.rs:118-137):
    /// positions from the device (the host copy is stale), both contact tables gathered on
    /// the host and uploaded for this tick's substeps. No registered boundaries: no work.
    fn gather_walls(&mut self, h: f32, providers: &dyn ProviderColliders) {
        if self.boundaries.is_empty() {
            return;
        }
        let mut buf = vec![0f32; 3 * (self.n_fluid + self.nb)];
        // SAFETY: buf holds 3 floats per particle; velocities are not requested.
        must(unsafe { ffi::vxl_sph_read_state(self.h.as_ptr(), buf.as_mut_ptr(), std::ptr::null_mut()) },
             "vxl_sph_read_state");
        let ps: Vec<Vec3> = buf[..3 * self.n_fluid].chunks_exact(3).map(|c| Vec3::new(c[0], c[1], c[2])).collect();
        for side in [ffi::WALLS_MIRROR, ffi::WALLS_PROJECT] {
            let (ids, start, planes) = self.gather(h, &ps, providers, side);
            let n = ids.len() as u32;
            // SAFETY: ids has n entries, start n + 1, planes 6 floats per plane.
            must(unsafe {
                ffi::vxl_sph_set_wall_contacts(self.h.as_ptr(), 0, side,
                                               if n > 0 { ids.as_ptr() } else { std::ptr::null() },
                                               if n > 0 { start.as_ptr() } else { std::ptr::null() }, n,
                                               if planes.is_empty() { std::ptr::null() } else { planes.as_ptr() },
                                               (planes.len() / 6) as u32)
            }, "vxl_sph_set_wall_contacts");
        }
    }
}

/// `PhysGpuBackend` of this library (no data: the fluid work goes through the stepper).
pub struct B200Backend;

impl PhysGpuBackend for B200Backend {
    fn name(&self) -> &'static str {
        "b200-cuda-wcsph"
    }

    fn available(&self) -> bool {
        // SAFETY: no arguments; the call only probes for an sm_100 device.
        unsafe { ffi::vxl_sph_abi_version() == ffi::ABI_VERSION && ffi::vxl_sph_backend_available() == 1 }
    }
}
