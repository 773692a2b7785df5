//! The C ABI of libvxl_sph (include/vxl_sph.h), declared for Rust. Every struct is
//! `#[repr(C)]` with the header's field order; every call returns a status whose values 0-5
//! are the reference's `FfiError` (crates/vxl-phys-ffi/src/lib.rs:26-33) and 6-9 are
//! additions (invalid argument, CUDA error, out of memory, device error flag). This module
//! is the only `unsafe` surface of the crate.
#![allow(non_camel_case_types, dead_code)]

use std::os::raw::{c_char, c_int, c_void};

pub const ABI_VERSION: u32 = 1;

pub const OK: u32 = 0;
pub const NULL_POINTER: u32 = 1;
pub const VERSION_MISMATCH: u32 = 2;
pub const SIZE_MISMATCH: u32 = 3;
pub const NOT_READY: u32 = 4;
pub const PANIC_CAUGHT: u32 = 5;
pub const INVALID_ARGUMENT: u32 = 6;
pub const CUDA_ERROR: u32 = 7;
pub const OUT_OF_MEMORY: u32 = 8;
pub const DEVICE_FAULT_FLAG: u32 = 9;

pub const PROVIDER_FACES: u32 = 0;
pub const PROVIDER_CONVEX: u32 = 1;
pub const DENSITY_WALK: u32 = 0;
pub const DENSITY_GROUPED: u32 = 1;
pub const WALLS_MIRROR: u32 = 0;
pub const WALLS_PROJECT: u32 = 1;

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct BlockHeader {
    pub size: u32,
    pub version: u32,
}

impl BlockHeader {
    pub fn of<T>() -> Self {
        Self { size: std::mem::size_of::<T>() as u32, version: ABI_VERSION }
    }
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct Params {
    pub hdr: BlockHeader,
    pub rest_density: f32,
    pub smoothing_radius: f32,
    pub xsph_viscosity: f32,
    pub tensile_instability_suppression: u32,
    pub sound_speed: f32,
    pub gamma_tait: f32,
    pub substeps: u32,
    pub boundary_layers: u32,
    pub gravity: [f32; 3],
    pub max_speed_frac: f32,
    pub artificial_viscosity: f32,
    pub particle_mass: f32,
    pub max_bins: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct Desc {
    pub hdr: BlockHeader,
    pub params: Params,
    pub n_fluid: u64,
    pub n_boundary: u64,
    pub pos_xyz: *const f32,
    pub vel_xyz: *const f32,
    pub pmass: *const f32,
    pub device: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct Span {
    pub body: u32,
    pub origin: [f32; 3],
    pub start: u32,
    pub end: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct Reaction {
    pub body: u32,
    pub force: [f32; 3],
    pub torque: [f32; 3],
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct GridInfo {
    pub hdr: BlockHeader,
    pub min: [f32; 3],
    pub inv: f32,
    pub bin: f32,
    pub dims: [u32; 3],
    pub total: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct Stats {
    pub hdr: BlockHeader,
    pub n_fluid: u64,
    pub n_boundary: u64,
    pub cells: u64,
    pub launches_last_tick: u64,
    pub device_bytes: u64,
    pub last_tick_ms: f32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct Tuning {
    pub hdr: BlockHeader,
    pub block: u32,
    pub tile: u32,
    pub waves: u32,
    pub density: u32,
    pub ms_per_substep: f32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct BodyPose {
    pub body: u32,
    pub pos: [f32; 3],
    pub rot: [f32; 4],
    pub linvel: [f32; 3],
    pub angvel: [f32; 3],
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct RigidBody {
    pub pose: BodyPose,
    pub inv_mass: f32,
    pub local_inv_inertia: [f32; 3],
    pub dynamic: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct WallPlane {
    pub normal: [f32; 3],
    pub offset: f32,
    pub axis: u32,
    pub sign: f32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct Provider {
    pub kind: u32,
    pub first_plane: u32,
    pub nplanes: u32,
    pub has_bounds: u32,
    pub bounds_min: [f32; 3],
    pub bounds_max: [f32; 3],
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct RequestStatus {
    pub hdr: BlockHeader,
    pub state: u32,
    pub ticks_done: u32,
    pub ticks_total: u32,
    pub pad: u32,
    pub submit_s: f64,
    pub admit_s: f64,
    pub done_s: f64,
    pub tick_p50_ms: f64,
    pub tick_p99_ms: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ServeReport {
    pub hdr: BlockHeader,
    pub active: u32,
    pub queued: u32,
    pub admitted: u32,
    pub retired: u32,
    pub particles: u64,
    pub device_bytes_in_use: u64,
}

/// Opaque handle of a resident scene (or batch of scenes).
pub enum Handle {}
/// Opaque handle of the served form.
pub enum Server {}

extern "C" {
    pub fn vxl_sph_abi_version() -> u32;
    pub fn vxl_sph_last_error() -> *const c_char;
    pub fn vxl_sph_backend_name() -> *const c_char;
    pub fn vxl_sph_backend_available() -> c_int;
    pub fn vxl_sph_lattice_mass(params: *const Params, spacing: f32, out_mass: *mut f32) -> u32;
    pub fn vxl_sph_boundary_lattice(shape: u32, half: *const f32, radius: f32, spacing: f32, h: f32, layers: u32,
                                    out_xyz: *mut f32, cap: u64, n: *mut u64, volume: *mut f32) -> u32;
    pub fn vxl_sph_create(desc: *const Desc, out: *mut *mut Handle) -> u32;
    pub fn vxl_sph_destroy(h: *mut Handle) -> u32;
    pub fn vxl_sph_upload_boundary(h: *mut Handle, n_fluid: u64, pos_xyz: *const f32, vel_xyz: *const f32,
                                   nb: u64) -> u32;
    pub fn vxl_sph_step_tick(h: *mut Handle, dt_tick: f32, spans: *const Span, nspans: u32,
                             out_reactions: *mut Reaction) -> u32;
    pub fn vxl_sph_step_tick_async(h: *mut Handle, dt_tick: f32, spans: *const Span, nspans: u32) -> u32;
    pub fn vxl_sph_sync(h: *mut Handle, out_reactions: *mut Reaction, nspans: u32) -> u32;
    pub fn vxl_sph_substep(h: *mut Handle, dt: f32) -> u32;
    pub fn vxl_sph_bounds(h: *mut Handle, lo: *mut f32, hi: *mut f32) -> u32;
    pub fn vxl_sph_read_state(h: *mut Handle, pos_xyz: *mut f32, vel_xyz: *mut f32) -> u32;
    pub fn vxl_sph_write_state(h: *mut Handle, pos_xyz: *const f32, vel_xyz: *const f32) -> u32;
    pub fn vxl_sph_set_record(h: *mut Handle, on: c_int) -> u32;
    pub fn vxl_sph_read_fields(h: *mut Handle, dens: *mut f32, press: *mut f32, acc_xyz: *mut f32,
                               xsph_xyz: *mut f32, bforce_xyz: *mut f32) -> u32;
    pub fn vxl_sph_export_grid(h: *mut Handle, items: *mut u32, start: *mut u32, start_cap: u64, bins: *mut u32,
                               info: *mut GridInfo) -> u32;
    pub fn vxl_sph_export_neighbors(h: *mut Handle, offsets: *mut u64, offsets_len: u64, entries: *mut u32,
                                    entries_cap: u64, total: *mut u64) -> u32;
    pub fn vxl_sph_get_stats(h: *mut Handle, out: *mut Stats) -> u32;
    pub fn vxl_sph_set_stream(h: *mut Handle, cuda_stream: *mut c_void) -> u32;
    pub fn vxl_sph_set_profile(h: *mut Handle, on: c_int) -> u32;
    pub fn vxl_sph_profile_read(h: *mut Handle, k: u32, name: *mut *const c_char, total_ms: *mut f64,
                                launches: *mut u64) -> u32;
    pub fn vxl_sph_create_batch(descs: *const Desc, n: u32, device: i32, cell_capacity: u64,
                                out: *mut *mut Handle) -> u32;
    pub fn vxl_sph_scene_count(h: *mut Handle) -> u32;
    pub fn vxl_sph_read_state_scene(h: *mut Handle, scene: u32, pos_xyz: *mut f32, vel_xyz: *mut f32) -> u32;
    pub fn vxl_sph_write_state_scene(h: *mut Handle, scene: u32, pos_xyz: *const f32, vel_xyz: *const f32) -> u32;
    pub fn vxl_sph_upload_boundary_scene(h: *mut Handle, scene: u32, pos_xyz: *const f32, vel_xyz: *const f32,
                                         nb: u64) -> u32;
    pub fn vxl_sph_set_spans_scene(h: *mut Handle, scene: u32, spans: *const Span, nspans: u32) -> u32;
    pub fn vxl_sph_export_grid_scene(h: *mut Handle, scene: u32, items: *mut u32, start: *mut u32, start_cap: u64,
                                     bins: *mut u32, info: *mut GridInfo) -> u32;
    pub fn vxl_sph_read_fields_scene(h: *mut Handle, scene: u32, dens: *mut f32, press: *mut f32,
                                     acc_xyz: *mut f32, xsph_xyz: *mut f32, bforce_xyz: *mut f32) -> u32;
    pub fn vxl_sph_reactions_all(h: *mut Handle, out: *mut Reaction, cap: u32, n: *mut u32) -> u32;
    pub fn vxl_sph_set_tuning(h: *mut Handle, t: *const Tuning) -> u32;
    pub fn vxl_sph_get_tuning(h: *mut Handle, t: *mut Tuning) -> u32;
    pub fn vxl_sph_autotune(h: *mut Handle, dt_tick: f32, trials: u32, best: *mut Tuning) -> u32;
    pub fn vxl_sph_request_state(h: *mut Handle) -> u32;
    pub fn vxl_sph_take_state(h: *mut Handle, pos_xyz: *mut f32, n: u64) -> u32;
    pub fn vxl_sph_set_body_lattice(h: *mut Handle, scene: u32, local_xyz: *const f32, body_index: *const u32,
                                    nb: u64, nbodies: u32) -> u32;
    pub fn vxl_sph_set_body_poses(h: *mut Handle, scene: u32, poses: *const BodyPose, nbodies: u32) -> u32;
    pub fn vxl_sph_set_rigid_bodies(h: *mut Handle, scene: u32, bodies: *const RigidBody, n: u32) -> u32;
    pub fn vxl_sph_step_coupled(h: *mut Handle, dt_tick: f32, rigid_substeps: u32, gravity: *const f32,
                                max_linear_velocity: f32, max_angular_velocity: f32, out_reactions: *mut Reaction,
                                nspans: u32) -> u32;
    pub fn vxl_sph_read_rigid_bodies(h: *mut Handle, scene: u32, out: *mut RigidBody, n: u32) -> u32;
    pub fn vxl_sph_set_providers(h: *mut Handle, scene: u32, providers: *const Provider, nproviders: u32,
                                 planes: *const WallPlane, nplanes: u32) -> u32;
    pub fn vxl_sph_set_wall_contacts(h: *mut Handle, scene: u32, side: u32, ids: *const u32, start: *const u32,
                                     n_entries: u32, planes: *const f32, n_planes: u32) -> u32;
    pub fn vxl_sph_serve_create(device: i32, budget_bytes: u64, max_scenes: u32, out: *mut *mut Server) -> u32;
    pub fn vxl_sph_serve_destroy(s: *mut Server) -> u32;
    pub fn vxl_sph_serve_submit(s: *mut Server, desc: *const Desc, ticks: u32, out_id: *mut u64) -> u32;
    pub fn vxl_sph_serve_step(s: *mut Server, dt_tick: f32, report: *mut ServeReport) -> u32;
    pub fn vxl_sph_serve_set_batch_cap(s: *mut Server, max_fluid_particles: u64) -> u32;
    pub fn vxl_sph_serve_poll(s: *mut Server, id: u64, out: *mut RequestStatus) -> u32;
    pub fn vxl_sph_serve_read(s: *mut Server, id: u64, pos_xyz: *mut f32, vel_xyz: *mut f32) -> u32;
    pub fn vxl_sph_serve_tick_times(s: *mut Server, id: u64, out_ms: *mut f64, cap: u32, n: *mut u32) -> u32;
    pub fn vxl_sph_build_grid_static(d_pos_xyz: *const f32, n: u32, h: f32, max_bins: u32, d_items: *mut u32,
                                     d_start: *mut u32, start_cap: u64, info: *mut GridInfo,
                                     cuda_stream: *mut c_void) -> u32;
}
