/*
 * vxl_sph.h — C ABI of the B200 (sm_100a) WCSPH fluid step.
 *
 * Drop-in for the fluid GPU tier of bfxh/RUST-WL. The reference's seam is the Rust
 * trait `FluidStepper` (crates/vxl-phys-core/src/interop.rs:293-316), implemented by
 * `GpuFluidStepper` (crates/vxl-phys-gpu/src/pipeline/stepper.rs:22-147) and
 * registered with `World::set_fluid_stepper` (crates/vxl-phys/src/world_step/
 * fluid_stepper.rs:46-58). A Rust shim implements that trait over these entry points.
 *
 * Conventions follow crates/vxl-phys-ffi/src/lib.rs:
 *   - every struct that crosses the boundary starts with {u32 size; u32 version}
 *     (BlockHeader, lib.rs:18-21), checked against VXL_SPH_ABI_VERSION (lib.rs:13);
 *   - status codes extend FfiError (lib.rs:26-33): the first six values are identical;
 *   - calls are batch-only (whole particle arrays, never one particle at a time);
 *   - no C++ exception or CUDA error crosses the boundary: both become a status code
 *     and a message readable through vxl_sph_last_error().
 *
 * Arrays of vectors are AoS float triples (x, y, z) — the reference's `Vec3` layout
 * (#[repr(C)] { f32 x, y, z }, crates/vxl-phys-core/src/math.rs:8-14) — in the
 * reference's particle index order: fluid prefix [0, n_fluid) then boundary suffix.
 * Host pointers are borrowed for the duration of the call only.
 *
 * Threading: one handle must not be driven from two threads at once (the reference's
 * FluidStepper is used through &mut self). Distinct handles are independent.
 */
#ifndef VXL_SPH_H
#define VXL_SPH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VXL_SPH_ABI_VERSION 1u

/* crates/vxl-phys-ffi/src/lib.rs:26-33 (FfiError); values 6.. are additions. */
typedef enum vxl_status {
  VXL_OK = 0,
  VXL_NULL_POINTER = 1,
  VXL_VERSION_MISMATCH = 2,
  VXL_SIZE_MISMATCH = 3,
  VXL_NOT_READY = 4,
  VXL_PANIC_CAUGHT = 5,
  VXL_INVALID_ARGUMENT = 6,
  VXL_CUDA_ERROR = 7,
  VXL_OUT_OF_MEMORY = 8,
  VXL_DEVICE_FAULT_FLAG = 9 /* a kernel raised its error flag (see vxl_sph_last_error) */
} vxl_status;

/* crates/vxl-phys-ffi/src/lib.rs:18-21 (BlockHeader). */
typedef struct vxl_block_header {
  uint32_t size;
  uint32_t version;
} vxl_block_header;

/* crates/vxl-phys-fluid/src/config.rs:6-68 (FluidConfig; field meaning and defaults
 * identical). particle_mass is the fluid particle mass `FluidSystem::mass`
 * (fluid_access.rs:27-42, see vxl_sph_lattice_mass); max_bins is the cell budget of
 * crates/vxl-phys-core/src/grid.rs:20 (0 = 1<<21). */
typedef struct vxl_sph_params {
  vxl_block_header hdr;
  float rest_density;
  float smoothing_radius;
  float xsph_viscosity;
  uint32_t tensile_instability_suppression;
  float sound_speed;
  float gamma_tait;
  uint32_t substeps;
  uint32_t boundary_layers;
  float gravity[3];
  float max_speed_frac;
  float artificial_viscosity;
  float particle_mass;
  uint32_t max_bins;
} vxl_sph_params;

/* Full particle set at creation: `FluidStepper::step`'s pos/vel/pmass
 * (crates/vxl-phys-core/src/interop.rs:296-304), fluid prefix + boundary suffix. */
typedef struct vxl_sph_desc {
  vxl_block_header hdr;
  vxl_sph_params params;
  uint64_t n_fluid;
  uint64_t n_boundary;
  const float* pos_xyz;  /* 3 * (n_fluid + n_boundary) */
  const float* vel_xyz;  /* 3 * (n_fluid + n_boundary) */
  const float* pmass;    /* n_fluid + n_boundary; fluid entries must equal particle_mass */
  int32_t device;        /* CUDA device ordinal */
} vxl_sph_desc;

/* One boundary segment (crates/vxl-phys-fluid/src/system.rs:41-42): body id, body
 * origin (torque pivot), [start, end) in global particle index. */
typedef struct vxl_sph_span {
  uint32_t body;
  float origin[3];
  uint32_t start;
  uint32_t end;
} vxl_sph_span;

/* Per-body reaction (crates/vxl-phys-fluid/src/fluid_access.rs:109-113):
 * tick-averaged force and torque about the body origin. */
typedef struct vxl_sph_reaction {
  uint32_t body;
  float force[3];
  float torque[3];
} vxl_sph_reaction;

/* Grid description of the last substep (crates/vxl-phys-fluid/src/grid.rs:168-175,
 * NeighborGrid): min corner, 1/bin, bin, dims, cell count. */
typedef struct vxl_sph_grid_info {
  vxl_block_header hdr;
  float min[3];
  float inv;
  float bin;
  uint32_t dims[3];
  uint64_t total;
} vxl_sph_grid_info;

typedef struct vxl_sph_handle vxl_sph_handle;

/* crates/vxl-phys-ffi/src/lib.rs:13 (ABI_VERSION). */
uint32_t vxl_sph_abi_version(void);

/* Thread-local message for the last non-OK status returned on this thread. */
const char* vxl_sph_last_error(void);

/* PhysGpuBackend::name / ::available (crates/vxl-phys-gpu/src/lib.rs:20-29):
 * backend name, and 1 when a device with compute capability 10.x is present. */
const char* vxl_sph_backend_name(void);
int vxl_sph_backend_available(void);

/* Lattice mass calibration m = rho0 / sum_lattice W
 * (crates/vxl-phys-fluid/src/fluid_access.rs:27-42). Host-only arithmetic. */
vxl_status vxl_sph_lattice_mass(const vxl_sph_params* params, float spacing, float* out_mass);

/* Two-layer Akinci boundary lattice of a box (half extents) or sphere (radius) in body
 * space (crates/vxl-phys-fluid/src/boundary.rs:67-88, box_faces :208-232,
 * sphere_shell :237-258, volume_from_self_sum :95-129). shape: 0 = box, 1 = sphere.
 * Writes min(count, cap) points (xyz) and the calibrated per-particle volume; *out_count
 * receives the full count (call with cap = 0 to size the buffer). */
vxl_status vxl_sph_boundary_lattice(uint32_t shape, const float half[3], float radius, float spacing,
                                    float h, uint32_t layers, float* out_pts_xyz, uint64_t cap,
                                    uint64_t* out_count, float* out_volume);

/* Create a resident scene (the reference builds its `Packet` once from the full set,
 * crates/vxl-phys-gpu/src/pipeline/stepper.rs:36-61). */
vxl_status vxl_sph_create(const vxl_sph_desc* desc, vxl_sph_handle** out);
vxl_status vxl_sph_destroy(vxl_sph_handle* h);

/* Re-upload the boundary segment (positions/velocities of boundary particles
 * [n_fluid, n_fluid + nb)), as GpuFluidStepper::step does each tick through
 * upload_boundary_segment (crates/vxl-phys-gpu/src/pipeline/coupling.rs:20-50).
 * A length mismatch is VXL_SIZE_MISMATCH, never truncation (coupling.rs:22-33). */
vxl_status vxl_sph_upload_boundary(vxl_sph_handle* h, uint64_t n_fluid, const float* pos_xyz,
                                   const float* vel_xyz, uint64_t nb);

/* Advance one tick of `substeps` substeps (FluidSystem::step, crates/vxl-phys-fluid/
 * src/fluid_step.rs:75-89) and return the tick-averaged per-span reactions
 * (aggregate_reactions, fluid_boundary.rs:10-28). out_reactions may be NULL when
 * nspans == 0. Synchronous: returns after the reactions are on the host. */
vxl_status vxl_sph_step_tick(vxl_sph_handle* h, float dt_tick, const vxl_sph_span* spans,
                             uint32_t nspans, vxl_sph_reaction* out_reactions);

/* Enqueue one tick without waiting (the reference's run_deferred,
 * crates/vxl-phys-gpu/src/pipeline.rs:607-609); vxl_sph_sync waits and, when
 * out_reactions is given, copies the reactions of the last enqueued tick. */
vxl_status vxl_sph_step_tick_async(vxl_sph_handle* h, float dt_tick, const vxl_sph_span* spans,
                                   uint32_t nspans);
vxl_status vxl_sph_sync(vxl_sph_handle* h, vxl_sph_reaction* out_reactions, uint32_t nspans);

/* One substep only (FluidSystem::substep, fluid_step.rs:91-127): per-step parity. */
vxl_status vxl_sph_substep(vxl_sph_handle* h, float dt);

/* Tight AABB of the fluid particles (FluidStepper::bounds, interop.rs:306-309;
 * the GPU tier reads it from the device, readback.rs:111-154). */
vxl_status vxl_sph_bounds(vxl_sph_handle* h, float lo[3], float hi[3]);

/* State in reference index order (Packet::read_state / snapshot / restore,
 * crates/vxl-phys-gpu/src/pipeline.rs:768-776). Arrays are 3 * n_total floats;
 * either pointer may be NULL. */
vxl_status vxl_sph_read_state(vxl_sph_handle* h, float* pos_xyz, float* vel_xyz);
vxl_status vxl_sph_write_state(vxl_sph_handle* h, const float* pos_xyz, const float* vel_xyz);

/* Per-particle results of the last substep in reference index order (the
 * reference's densities()/pressures()/accelerations()/boundary_forces() and xsph,
 * fluid_access.rs:149-171). acc/xsph are recorded only while recording is on
 * (vxl_sph_set_record); dens/press always. Any pointer may be NULL. */
vxl_status vxl_sph_set_record(vxl_sph_handle* h, int on);
vxl_status vxl_sph_read_fields(vxl_sph_handle* h, float* dens, float* press, float* acc_xyz,
                               float* xsph_xyz, float* bforce_xyz);

/* Neighbour table of the last substep (FluidSystem::neighbor_grid,
 * crates/vxl-phys-fluid/src/fluid_access.rs:125-133): items[n_total] = particle
 * index per cell-ordered slot, start[total+1], bins[n_total] = cell of each particle.
 * start_cap is the capacity of start in entries. Any array may be NULL. */
vxl_status vxl_sph_export_grid(vxl_sph_handle* h, uint32_t* items, uint32_t* start, uint64_t start_cap,
                               uint32_t* bins, vxl_sph_grid_info* info);

/* Neighbour lists of the last substep, as its density pass recorded them and its force
 * pass and boundary reactions read them: for particle i (reference index order) the
 * neighbours j != i within h, in the walk order of UniformGrid::for_neighbors_in
 * (crates/vxl-phys-fluid/src/grid.rs:115-155, over the table FluidSystem::neighbor_grid
 * exposes, fluid_access.rs:125-133) — every neighbour of a fluid particle, the fluid ones
 * of a boundary particle (the terms of fluid_density.rs:17-70). CSR: offsets[n_total + 1]
 * (offsets_len must be n_total + 1) and entries[offsets[i] .. offsets[i + 1]]. With
 * entries NULL only offsets and *total are written (call once to size, once to fill);
 * entries_cap below the total is VXL_SIZE_MISMATCH. Lists longer than the recorded cap
 * are walked again from that substep's sorted positions, as the consumers do. Valid until
 * the next substep starts. */
vxl_status vxl_sph_export_neighbors(vxl_sph_handle* h, uint64_t* offsets, uint64_t offsets_len, uint32_t* entries,
                                    uint64_t entries_cap, uint64_t* total);

/* Counts for the caller's own accounting: particles, cells of the last substep,
 * kernel launches of the last tick, bytes of device memory held. */
typedef struct vxl_sph_stats {
  vxl_block_header hdr;
  uint64_t n_fluid;
  uint64_t n_boundary;
  uint64_t cells;
  uint64_t launches_last_tick;
  uint64_t device_bytes;
  float last_tick_ms; /* device time of the last tick (CUDA events), 0 if unknown */
} vxl_sph_stats;
vxl_status vxl_sph_get_stats(vxl_sph_handle* h, vxl_sph_stats* out);

/* Run the handle's work on a caller-owned CUDA stream (a cudaStream_t passed as
 * void*; NULL returns to the handle's own stream). Lets a caller order the step with
 * its own work and time it with events on that stream. */
vxl_status vxl_sph_set_stream(vxl_sph_handle* h, void* cuda_stream);

/* Per-kernel device timers, the device counterpart of the reference's phase
 * accumulators (FluidSystem::phase_us, crates/vxl-phys-fluid/src/fluid_step.rs:
 * 98-126, 129-138): with profiling on, every kernel launch of a tick is bracketed by
 * CUDA events on the launching stream and the elapsed times are accumulated per kernel
 * when the next tick starts or on vxl_sph_profile_read. Switching on resets the
 * accumulators. */
vxl_status vxl_sph_set_profile(vxl_sph_handle* h, int on);
/* Kernel k of the accumulator table: name (static string), total device ms and
 * launch count. Returns VXL_INVALID_ARGUMENT when k is past the last kernel. */
vxl_status vxl_sph_profile_read(vxl_sph_handle* h, uint32_t k, const char** name, double* total_ms,
                                uint64_t* launches);

/* ------------------------------------------------------------------ batched form
 * One handle can hold many independent scenes (the batched workload): they are packed
 * into one particle pool and stepped together, one launch per kernel per substep for
 * all scenes, with each scene's own constants and grid (a segmented sort on
 * scene-offset cell keys) and the particle passes run as persistent kernels over a
 * (scene, tile) work list. No counterpart in the reference (its GPU tier steps one
 * Packet); each scene's results equal a plain handle's for the same inputs. */

/* Create a handle holding n scenes (descs[i] as for vxl_sph_create; all on `device`;
 * all must share `substeps` to be stepped by vxl_sph_step_tick). cell_capacity bounds
 * the sum of the scenes' cells per substep (0 = the sum of their max_bins, capped at
 * 2^28); a substep that would exceed it is skipped and reported as
 * VXL_DEVICE_FAULT_FLAG. */
vxl_status vxl_sph_create_batch(const vxl_sph_desc* descs, uint32_t n, int32_t device, uint64_t cell_capacity,
                                vxl_sph_handle** out);
uint32_t vxl_sph_scene_count(vxl_sph_handle* h);

/* Per-scene variants of the plain calls (scene-local particle indices). */
vxl_status vxl_sph_read_state_scene(vxl_sph_handle* h, uint32_t scene, float* pos_xyz, float* vel_xyz);
vxl_status vxl_sph_write_state_scene(vxl_sph_handle* h, uint32_t scene, const float* pos_xyz, const float* vel_xyz);
vxl_status vxl_sph_upload_boundary_scene(vxl_sph_handle* h, uint32_t scene, const float* pos_xyz,
                                         const float* vel_xyz, uint64_t nb);
vxl_status vxl_sph_set_spans_scene(vxl_sph_handle* h, uint32_t scene, const vxl_sph_span* spans, uint32_t nspans);
vxl_status vxl_sph_export_grid_scene(vxl_sph_handle* h, uint32_t scene, uint32_t* items, uint32_t* start,
                                     uint64_t start_cap, uint32_t* bins, vxl_sph_grid_info* info);
vxl_status vxl_sph_read_fields_scene(vxl_sph_handle* h, uint32_t scene, float* dens, float* press,
                                     float* acc_xyz, float* xsph_xyz, float* bforce_xyz);
/* Reactions of every span of every scene from the last tick, in scene order then span
 * order; *n receives the count (call with cap = 0 to size). */
vxl_status vxl_sph_reactions_all(vxl_sph_handle* h, vxl_sph_reaction* out, uint32_t cap, uint32_t* n);

/* Launch shape of the particle passes: threads per block (128 or 256), slots per tile
 * (a multiple of 128, at least one block) and the scheduling: waves = 0 runs one block
 * per tile, waves = k > 0 runs k x the occupancy limit of persistent blocks that draw
 * tiles from a counter. density selects the density kernel of scenes without provider
 * walls: VXL_SPH_DENSITY_WALK (one thread per particle walking its own cells, threads
 * ordered by cell octant) or VXL_SPH_DENSITY_GROUPED (eight lanes per cell octant sharing
 * one staged stream of candidates); both give the same results. Default {256, 256, 0,
 * WALK}. */
#define VXL_SPH_DENSITY_WALK 0u
#define VXL_SPH_DENSITY_GROUPED 1u
typedef struct vxl_sph_tuning {
  vxl_block_header hdr;
  uint32_t block;
  uint32_t tile;
  uint32_t waves;
  uint32_t density;     /* VXL_SPH_DENSITY_* */
  float ms_per_substep; /* filled by vxl_sph_autotune: device time of the chosen shape */
} vxl_sph_tuning;
vxl_status vxl_sph_set_tuning(vxl_sph_handle* h, const vxl_sph_tuning* t);
vxl_status vxl_sph_get_tuning(vxl_sph_handle* h, vxl_sph_tuning* t);
/* Autotuner: times every candidate shape on the handle's own scenes (`trials` substeps
 * each, from a snapshot of the state that is restored afterwards) and keeps the fastest;
 * then times the other density kernels at that shape and keeps the fastest.
 * Results are identical for every shape; only the time differs. */
vxl_status vxl_sph_autotune(vxl_sph_handle* h, float dt_tick, uint32_t trials, vxl_sph_tuning* best);

/* ------------------------------------------------------------------ deferred state readback
 * The GPU tier's pipelined readback (Packet::run_deferred + take_deferred_state,
 * crates/vxl-phys-gpu/src/pipeline.rs:603-609, pipeline/readback.rs:229-262): request enqueues,
 * after whatever is already enqueued on the handle's stream (e.g. vxl_sph_step_tick_async),
 * a copy of every particle's position (reference order; for a batch, scene after scene) into
 * a pinned buffer the handle owns and returns without waiting; take waits for that copy and
 * writes it out. The device-to-host copy runs on a stream of its own, so work enqueued after
 * the request (the next tick) does not wait for it, and the host's wait overlaps the tick:
 * renderers draw the previous tick. A second request waits for a copy not yet taken. */
vxl_status vxl_sph_request_state(vxl_sph_handle* h);
/* n: every particle of the handle (the sum over its scenes), as at the request. */
vxl_status vxl_sph_take_state(vxl_sph_handle* h, float* pos_xyz, uint64_t n);

/* ------------------------------------------------------------------ moving bodies on the device
 * The reference rebuilds the boundary segment on the host every tick from the bodies'
 * poses (set_boundary_particles, crates/vxl-phys-fluid/src/fluid_step.rs:13-53) and the GPU
 * tier uploads it (crates/vxl-phys-gpu/src/pipeline/coupling.rs:20-50). With the body-frame
 * lattice resident on the device, a tick needs only the poses: each boundary particle k of
 * body b becomes p = pos_b + rotate(rot_b, L_k), v = linvel_b + angvel_b x (p - pos_b), with
 * the reference's f32 operation order, bit for bit what vxl_sph_upload_boundary would be
 * given. pmass (the lattice volume) is unchanged. */
typedef struct vxl_sph_body_pose {
  uint32_t body;       /* body id (informational) */
  float pos[3];        /* body origin (the lattice's frame) */
  float rot[4];        /* unit quaternion x, y, z, w */
  float linvel[3];
  float angvel[3];
} vxl_sph_body_pose;

/* local_xyz[3 k..3 k+3): boundary particle k's lattice point in its body's frame;
 * body_index[k] < nbodies: its body's position in the pose array. nb must equal the
 * scene's boundary count. Plain handles use scene 0. */
vxl_status vxl_sph_set_body_lattice(vxl_sph_handle* h, uint32_t scene, const float* local_xyz,
                                    const uint32_t* body_index, uint64_t nb, uint32_t nbodies);
/* Rebuild the scene's boundary segment from `nbodies` poses (same count as the lattice). */
vxl_status vxl_sph_set_body_poses(vxl_sph_handle* h, uint32_t scene, const vxl_sph_body_pose* poses,
                                  uint32_t nbodies);

/* ------------------------------------------------------------------ coupling loop on the device
 * The facade's fluid coupling (crates/vxl-phys/src/world_step.rs) without its rigid contact
 * solver: the scene's lattice bodies (vxl_sph_set_body_lattice) become rigid bodies that stay
 * on the device. Each vxl_sph_step_coupled runs `rigid_substeps` rigid substeps per body in the
 * reference's order — the gravity field adds m g, the fluid reaction pass adds the previous
 * tick's tick-averaged reaction of the body's span, Integrator::integrate_velocities (speed
 * clamps) and integrate_positions (crates/vxl-phys-integrate/src/lib.rs:18-60) — then rebuilds
 * the boundary segment from the new poses and steps one fluid tick, whose reactions drive the
 * next call. Spans (vxl_sph_set_spans_scene) are matched to bodies by body id and take the
 * body's position as the torque origin. Bodies are not kept out of walls or each other: that
 * is the contact solver's work, which this library does not do. */
typedef struct vxl_sph_rigid_body {
  vxl_sph_body_pose pose;       /* position (= lattice origin), rotation, velocities */
  float inv_mass;               /* 1 / mass (mass.rs: box m = rho * 8 hx hy hz) */
  float local_inv_inertia[3];   /* body-frame inverse inertia diagonal */
  uint32_t dynamic;             /* 0: static (never moves), 1: dynamic */
} vxl_sph_rigid_body;

/* One rigid body per lattice body, in lattice body order. */
vxl_status vxl_sph_set_rigid_bodies(vxl_sph_handle* h, uint32_t scene, const vxl_sph_rigid_body* bodies,
                                    uint32_t n);
/* One coupled tick of every scene with rigid bodies (synchronous; reactions as for
 * vxl_sph_step_tick, nspans of them in span order). */
vxl_status vxl_sph_step_coupled(vxl_sph_handle* h, float dt_tick, uint32_t rigid_substeps, const float gravity[3],
                                float max_linear, float max_angular, vxl_sph_reaction* out_reactions,
                                uint32_t nspans);
vxl_status vxl_sph_read_rigid_bodies(vxl_sph_handle* h, uint32_t scene, vxl_sph_rigid_body* out, uint32_t n);

/* ------------------------------------------------------------------ provider walls
 * Analytic boundary providers of a scene, queried on the device every substep: the
 * reference's provider tier of the fluid step (FluidSystem::set_boundaries,
 * crates/vxl-phys-fluid/src/fluid_access.rs:184-186). For each fluid particle the density
 * pass collects up to 8 provider planes within h (wall_planes_in, fluid_density.rs:76-118)
 * and adds, after each neighbour's term, its mirror ghosts in those planes
 * (fluid_density.rs:38-47); after integration, fluid particles inside a provider are pushed
 * out and lose their inward normal velocity, and those pushed closer than 0.2 h to an
 * earlier-indexed pushed particle are separated (boundary_pass / separate_coincident,
 * fluid_boundary.rs:45-128). Providers are queried in the order given, planes in array order.
 *   VXL_SPH_PROVIDER_FACES: independent axis-aligned half-space faces (axis, plane = offset,
 *     sign = outward normal along the axis): a face reports a contact when
 *     (p[axis] - plane) * sign <= 2 probe (the fluid crate's FloorY / Tank providers,
 *     crates/vxl-phys-fluid/src/tests.rs:9-110).
 *   VXL_SPH_PROVIDER_CONVEX: a convex solid {x : normal . x <= offset for every plane};
 *     the plane of largest normal . x - offset decides (HalfSpaceSet,
 *     crates/vxl-phys-terrain/src/plane_set.rs:60-76, 166-181).
 * Other providers (voxel terrain, meshes, splats) stay on the host: they are not on this
 * path. n = 0 removes the scene's providers. */
#define VXL_SPH_PROVIDER_FACES 0u
#define VXL_SPH_PROVIDER_CONVEX 1u
#define VXL_SPH_MAX_PROVIDER_PLANES 64u  /* planes per scene, and providers per scene */
typedef struct vxl_sph_wall_plane {
  float normal[3];  /* CONVEX: outward unit normal */
  float offset;     /* CONVEX: offset d; FACES: the face's plane coordinate */
  uint32_t axis;    /* FACES: 0, 1, 2 */
  float sign;       /* FACES: +1 or -1 */
} vxl_sph_wall_plane;

typedef struct vxl_sph_provider {
  uint32_t kind;             /* VXL_SPH_PROVIDER_* */
  uint32_t first_plane;      /* planes [first_plane, first_plane + nplanes) */
  uint32_t nplanes;
  uint32_t has_bounds;       /* 1: skip the provider beyond its bounds + h (ProviderColliders::bounds) */
  float bounds_min[3];
  float bounds_max[3];
} vxl_sph_provider;

vxl_status vxl_sph_set_providers(vxl_sph_handle* h, uint32_t scene, const vxl_sph_provider* providers,
                                 uint32_t nproviders, const vxl_sph_wall_plane* planes, uint32_t nplanes);

/* Provider walls of ANY ProviderColliders (voxel terrain, meshes, splats, SDFs), as the
 * reference's GPU tier feeds them (GpuFluidStepper::gather_walls,
 * crates/vxl-phys-gpu/src/pipeline/stepper.rs:118-137; gather_wall_contacts /
 * gather_wall_project_contacts and WallStage::upload, pipeline/walls.rs:100-215): once per
 * tick the caller reads the fluid positions, queries its providers on the host and uploads
 * two contact tables. side 0 (mirror): for each fluid particle the planes of
 * contacts_point(bid, p, h) with 0 < sdf < h; side 1 (projection): those of
 * contacts_point_boundary(bid, p, h) with sdf < h; at most 8 per particle, sdf =
 * (p - point) . normal. ids[n_entries] are ascending scene-local fluid indices, entry e
 * owns planes [start[e], start[e + 1]) (start has n_entries + 1 values from 0 to
 * n_planes) and planes holds n_planes x (point xyz, outward normal xyz). The tables then
 * act as one more provider of the scene, after its analytic ones, for every substep until
 * replaced: each substep the mirror planes within 0 < sdf < h of the particle's current
 * position give its mirror ghosts (fluid_density.rs:25-47), and after integration the
 * projection planes push penetrating particles out (fluid_boundary.rs:45-128), with the
 * coincident-particle separation of the CPU path. n_entries = 0 clears that side. */
#define VXL_SPH_WALLS_MIRROR 0u
#define VXL_SPH_WALLS_PROJECT 1u
vxl_status vxl_sph_set_wall_contacts(vxl_sph_handle* h, uint32_t scene, uint32_t side, const uint32_t* ids,
                                     const uint32_t* start, uint32_t n_entries, const float* planes,
                                     uint32_t n_planes);

/* ------------------------------------------------------------------ served form
 * A request loop (the served workload): scene-step requests are submitted at any time,
 * admitted while their device footprint fits an HBM budget, stepped together with
 * every other admitted scene, and retired when their tick count is reached; the set of
 * scenes is repacked at substep boundaries (admission and retirement happen between
 * substeps, so a request admitted while others run starts on the next substep). No
 * counterpart in the reference. Scene state stays on the device from admission to
 * retirement; a retired scene's final state is kept on the host for vxl_sph_serve_read. */
typedef struct vxl_sph_server vxl_sph_server;

typedef struct vxl_sph_request_status {
  vxl_block_header hdr;
  uint32_t state;        /* 0 queued, 1 running, 2 done, 3 rejected */
  uint32_t ticks_done;
  uint32_t ticks_total;
  uint32_t pad;
  double submit_s;       /* host clock (seconds since the server was created) */
  double admit_s;
  double done_s;
  double tick_p50_ms;    /* wall time per tick of this request while it ran */
  double tick_p99_ms;
} vxl_sph_request_status;

typedef struct vxl_sph_serve_report {
  vxl_block_header hdr;
  uint32_t active;       /* scenes stepped by this call */
  uint32_t queued;
  uint32_t admitted;     /* admitted before this substep */
  uint32_t retired;      /* retired before this substep */
  uint64_t particles;    /* fluid particles advanced by this substep */
  uint64_t device_bytes_in_use;
} vxl_sph_serve_report;

/* budget_bytes: device memory the scenes may use (particle slots and cells);
 * max_scenes: scene table size. */
vxl_status vxl_sph_serve_create(int32_t device, uint64_t budget_bytes, uint32_t max_scenes, vxl_sph_server** out);
vxl_status vxl_sph_serve_destroy(vxl_sph_server* s);
/* Queue one request: a scene (copied) to be stepped `ticks` ticks of desc->params.substeps
 * substeps each. Rejected (state 3, VXL_OUT_OF_MEMORY) if it can never fit the budget. */
vxl_status vxl_sph_serve_submit(vxl_sph_server* s, const vxl_sph_desc* desc, uint32_t ticks, uint64_t* out_id);
/* Retire finished scenes, admit queued ones that fit, then advance every admitted scene by
 * one substep of its own dt = dt_tick / substeps. Synchronous. */
vxl_status vxl_sph_serve_step(vxl_sph_server* s, float dt_tick, vxl_sph_serve_report* report);
/* Latency knob of the served form: admission stops while the admitted scenes hold
 * max_fluid_particles fluid particles or more (a request larger than that is admitted
 * when nothing else runs), which bounds the work of each substep and so the per-tick
 * latency of admitted requests, at the cost of queueing the rest longer. 0 (the
 * default) admits while the memory budget allows. No counterpart in the reference. */
vxl_status vxl_sph_serve_set_batch_cap(vxl_sph_server* s, uint64_t max_fluid_particles);
vxl_status vxl_sph_serve_poll(vxl_sph_server* s, uint64_t id, vxl_sph_request_status* out);
/* Positions/velocities of a running or finished request (scene-local order). */
vxl_status vxl_sph_serve_read(vxl_sph_server* s, uint64_t id, float* pos_xyz, float* vel_xyz);
/* Wall time of each completed tick of a request, in milliseconds, in tick order (from
 * its admission, or the end of its previous tick, to the end of the substep that
 * completed the tick). Writes min(cap, ticks done) values and sets *n to ticks done. */
vxl_status vxl_sph_serve_tick_times(vxl_sph_server* s, uint64_t id, double* out_ms, uint32_t cap, uint32_t* n);

/* Neighbour-table build that allocates nothing. No counterpart in the reference: it is
 * for callers that cannot allocate device memory while they run — an engine that
 * reserves one fixed arena for all GPU work at start-up and forbids further cudaMalloc,
 * or a per-frame plugin that must not call cudaMalloc/cudaFree because both can
 * synchronise the device and stall its frame loop.
 *
 * Builds, on the current device, the same table a substep builds (cell keys by the
 * reference's grid rule, particles grouped by cell in ascending index): d_pos_xyz is
 * 3*n floats of device memory; d_items receives n particle indices; d_start receives
 * total+1 slot offsets and must hold max_bins+1 entries; *info (host memory) receives
 * the grid. Work runs on cuda_stream (a cudaStream_t, or NULL) and the call returns
 * after it has finished.
 *
 * Limits: n <= 524,288 particles and max_bins <= 524,288 cells (0 means 524,288);
 * larger sizes return VXL_INVALID_ARGUMENT. Working memory is one fixed array of about
 * 8.4 MB inside the library, held by every GPU that loads it until the process exits;
 * the call makes no cudaMalloc, cudaFree or other allocating call of its own. The first
 * call on a device is the set-up: the CUDA runtime loads the library's device code there
 * (mapping the array, which takes device memory and may synchronise the device), the
 * call looks the array's address up (cudaGetSymbolAddress) and raises one kernel's
 * shared-memory limit. Make that first call at start-up, as a warm-up (n = 1 will do),
 * before reserving the rest of the device's memory; later calls on that device take no
 * device memory. Every call is synchronous (it copies the grid box back and waits for
 * its stream), so no call may be made inside stream capture. Every call reuses the same
 * array (the counts it needs zeroed are cleared at the start of each call), so calls
 * that overlap on the GPU — from two streams or two host threads — race and must not be
 * made. Cells of any size are sorted in bounded time (warp, shared-memory rank, or a
 * bitmap of the particle indices for cells above 2,048 entries). */
vxl_status vxl_sph_build_grid_static(const float* d_pos_xyz, uint32_t n, float h, uint32_t max_bins,
                                     uint32_t* d_items, uint32_t* d_start, uint64_t start_cap,
                                     vxl_sph_grid_info* info, void* cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* VXL_SPH_H */
