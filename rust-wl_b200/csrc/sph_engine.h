// Host side of the multi-scene WCSPH engine (sph_engine.cuh holds the kernels).
//
// An Engine owns one pool of particle slots on one GPU and any number of resident
// scenes packed into it without gaps. It steps all active scenes together, one launch
// per kernel per substep, and captures whole ticks as CUDA graphs. The plain C ABI handle
// is an Engine holding one scene; the batched and served forms hold many.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "vxl_sph.h"

namespace vxl {

struct SceneDev;
struct TileDev;
struct EngineCtl;
struct SpanDev;
struct LongSpan;
struct BodyPoseDev;
struct RigidBodyDev;
struct ProviderDev;
struct ContactTableDev;
struct WallPlaneDev;

// Launch shape of the particle passes (chosen by the autotuner for batches).
struct Tuning {
  uint32_t block = 256;   // threads per block of the density/force passes (128 or 256)
  uint32_t tile = 256;    // slots per tile (a multiple of 128, at least one block)
  uint32_t waves = 0;     // 0: one block per tile; k > 0: persistent, k x the occupancy limit
  uint32_t density = 0;   // density kernel without provider walls: 0 per-particle walk, 1 grouped segments
};

struct SceneInfo {
  uint64_t id = 0;
  uint32_t base = 0, nf = 0, nb = 0;
  uint32_t substeps = 1;
  float particle_mass = 0.f;
  vxl_sph_params params{};
};

class Engine {
 public:
  // slot_cap particles and cell_cap cells of capacity; nbr_cap neighbour-list entries per
  // particle. Allocates everything up front.
  static vxl_status create(int device, uint64_t slot_cap, uint64_t cell_cap, uint32_t scene_cap,
                           Engine** out);
  ~Engine();

  int device() const { return device_; }
  cudaStream_t stream() const { return stream_; }
  void set_stream(cudaStream_t s);
  uint64_t used_slots() const { return used_; }
  uint64_t slot_cap() const { return slot_cap_; }
  uint64_t cell_cap() const { return cell_cap_; }
  uint64_t device_bytes() const { return device_bytes_; }
  uint64_t launches_last_tick() const { return launches_last_tick_; }
  const std::vector<SceneInfo>& scenes() const { return scenes_; }
  static uint64_t bytes_per_slot(uint32_t nbr_cap);
  static uint64_t bytes_per_cell();

  // Append a scene at the end of the pool (reference order input: fluid prefix then
  // boundary suffix, xyz triples). Validates like vxl_sph_create.
  vxl_status add_scene(const vxl_sph_params& p, uint64_t nf, uint64_t nb, const float* pos, const float* vel,
                       const float* pmass, uint64_t id, uint32_t* out_index);
  // Drop scenes (by index) and close the gaps by moving the later scenes down.
  vxl_status remove_scenes(const std::vector<uint32_t>& indices);

  vxl_status upload_boundary(uint32_t scene, const float* pos, const float* vel, uint64_t nb);
  // Device-side boundary rebuild: the body-frame lattice point and body index of every
  // boundary particle (reference order), then per tick only the bodies' poses.
  vxl_status set_body_lattice(uint32_t scene, const float* local_xyz, const uint32_t* body_index, uint64_t nb,
                              uint32_t nbodies);
  vxl_status set_body_poses(uint32_t scene, const vxl_sph_body_pose* poses, uint32_t nbodies);
  // Device-side coupling loop without contacts: the scene's bodies (one per lattice body,
  // same order) as rigid bodies; each coupled tick integrates them from the previous tick's
  // reactions, rebuilds the boundary segment from their poses and steps the fluid tick.
  vxl_status set_rigid_bodies(uint32_t scene, const vxl_sph_rigid_body* bodies, uint32_t n);
  vxl_status step_coupled_async(float dt_tick, uint32_t rigid_substeps, const float gravity[3], float max_linear,
                                float max_angular);
  vxl_status read_rigid_bodies(uint32_t scene, vxl_sph_rigid_body* out, uint32_t n);
  // Provider walls of a scene (analytic ProviderColliders queried on the device every
  // substep: mirror ghosts in the density, projection and separation after integration).
  vxl_status set_wall_contacts(uint32_t scene, uint32_t side, const uint32_t* ids, const uint32_t* start,
                               uint32_t n_entries, const float* planes, uint32_t n_planes);
  vxl_status set_providers(uint32_t scene, const vxl_sph_provider* providers, uint32_t n,
                           const vxl_sph_wall_plane* planes, uint32_t nplanes);
  vxl_status write_state(uint32_t scene, const float* pos, const float* vel);
  vxl_status read_state(uint32_t scene, float* pos, float* vel);
  // Deferred readback of every slot's position (reference order, scene after scene):
  // request enqueues the copy into a pinned buffer and returns; take waits and copies out.
  vxl_status request_state();
  vxl_status take_state(float* pos, uint64_t n);
  vxl_status read_fields(uint32_t scene, float* dens, float* press, float* acc, float* xsph, float* bforce);
  vxl_status export_neighbors(uint32_t scene, uint64_t* offsets, uint64_t offsets_len, uint32_t* entries,
                              uint64_t entries_cap, uint64_t* total);
  vxl_status export_grid(uint32_t scene, uint32_t* items, uint32_t* start, uint64_t start_cap, uint32_t* bins,
                         vxl_sph_grid_info* info);
  vxl_status bounds(uint32_t scene, float lo[3], float hi[3]);

  // Spans in scene-local particle indices, per scene (reactions of the plain/batched tick).
  vxl_status set_spans(uint32_t scene, const vxl_sph_span* spans, uint32_t n);
  // One tick of every scene (all scenes must share `substeps`), tick-averaged reactions.
  vxl_status step_tick_async(float dt_tick);
  vxl_status sync(std::vector<vxl_sph_reaction>* reactions);
  // One substep of every scene with per-scene dt (the served form), or of one scene
  // count (the plain vxl_sph_substep).
  vxl_status substep(const std::vector<float>& dt_per_scene);

  void set_record(bool on) { record_ = on; }
  bool record() const { return record_; }
  void set_use_graph(bool on) { use_graph_ = on; }
  void set_tuning(const Tuning& t);
  const Tuning& tuning() const { return tuning_; }
  vxl_status set_profile(bool on);
  vxl_status profile_read(uint32_t k, const char** name, double* ms, uint64_t* launches);
  bool ran_substep() const { return ran_substep_; }
  // Time every candidate launch shape over `trials` substeps on the resident scenes
  // (from a snapshot that is restored afterwards) and keep the fastest.
  vxl_status autotune(float dt_tick, uint32_t trials, Tuning* best, float* best_ms);
  uint32_t cells_last() ;
  uint32_t slow_gathers();

 private:
  Engine() = default;
  vxl_status alloc_all();
  void free_all();
  vxl_status recompute_scene_boxes(uint32_t scene);
  vxl_status rebuild_tiles();
  vxl_status stage_spans();
  vxl_status push_scene_records(const std::vector<float>& dt);
  void enqueue_substep(bool with_reactions);
  void enqueue_tick(float dt_tick);
  vxl_status finish();
  void prof_collect();
  int prof_begin(int kid, cudaStream_t st);
  void prof_end(int i, cudaStream_t st);
  void record_event(cudaEvent_t e, cudaStream_t st);
  void join_side();

  template <class T>
  vxl_status dalloc(T** p, size_t count);

  int device_ = 0;
  cudaStream_t stream_ = nullptr, own_stream_ = nullptr;
  // Reaction branch (boundary reactions + per-span sums) forked off the substep onto its
  // own stream after the density pass and joined before the next sort overwrites its
  // inputs (or at the end of the tick / substep call).
  cudaStream_t side_ = nullptr;
  cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr;
  bool side_pending_ = false;
  // per-body reaction sums: a third stream, forked after k_e_bforce and joined only where
  // bforce / bpos / breact change (the next k_e_bforce, the tick's end, host reads)
  cudaStream_t react_ = nullptr;
  cudaEvent_t ev_rfork_ = nullptr, ev_rjoin_ = nullptr;
  bool react_pending_ = false;
  void join_side_only();
  uint64_t slot_cap_ = 0, cell_cap_ = 0, used_ = 0;
  uint32_t scene_cap_ = 0, nbr_cap_ = 64;
  uint64_t device_bytes_ = 0;
  std::vector<SceneInfo> scenes_;
  std::vector<uint32_t> scene_bodies_;  // bodies of each scene's lattice (0: none set)

  // pool (slot_cap_)
  void* pos_[2] = {nullptr, nullptr};
  void* vel_[2] = {nullptr, nullptr};
  uint32_t* orig_ = nullptr;
  uint32_t* slot_of_ = nullptr;
  void* cellrank_ = nullptr;
  void* items_ = nullptr;
  void* rc_ = nullptr;
  float* press_ = nullptr;
  void* acc_ = nullptr;
  void* xsph_ = nullptr;
  void* bforce_ = nullptr;
  void* bpos_ = nullptr;
  uint16_t* nbr_ = nullptr;  // neighbour lists: 16-bit plane-relative entries, list position major
  uint32_t* nbr_n_ = nullptr;
  uint32_t* halves_ = nullptr;  // 4 words per 32 slots: upper-half masks along x, y, z
  uint32_t* xorder_ = nullptr;  // density order of the provider-wall variant at doubled bins (lower x halves first)
  uint32_t* order_ = nullptr;   // grouped density pass: slots of each chunk ordered by octant
  void* segs_ = nullptr;        // grouped density pass: segments (first position, count | scene << 4)
  float4* blocal_ = nullptr;         // body-frame lattice per boundary slot (reference order), lazily
  BodyPoseDev* poses_d_ = nullptr;   // poses of one scene's bodies (staged per call)
  uint32_t poses_cap_ = 0;
  std::vector<std::vector<vxl_sph_rigid_body>> rigid_;  // per scene (empty: not coupled)
  RigidBodyDev* rb_d_ = nullptr;  // all scenes' rigid bodies, scene after scene
  uint32_t rb_cap_ = 0, rb_n_ = 0;
  std::vector<uint32_t> rb_off_;  // first rigid body of each scene
  bool rb_dirty_ = false;         // host bodies changed: upload before the next coupled tick
  bool rb_have_reaction_ = false;  // breact holds the previous coupled tick's reactions
  bool rb_live_ = false;           // rb_d_ holds the bodies' current (evolved) states
  vxl_status rb_pull();
  void rb_layout();
  // provider walls
  std::vector<std::vector<vxl_sph_provider>> prov_h_;     // per scene (first_plane into wplanes_h_[q])
  std::vector<std::vector<vxl_sph_wall_plane>> wplanes_h_;
  ProviderDev* prov_d_ = nullptr;    // all scenes' providers, scene after scene
  WallPlaneDev* wplanes_d_ = nullptr;
  uint32_t prov_cap_ = 0, wplanes_cap_ = 0;
  uint32_t* pflag_ = nullptr;   // per reference index: pushed this substep
  void* pnsum_ = nullptr;       // float4 per reference index: normal sum, scene
  uint32_t* plist_ = nullptr;   // pushed reference indices, ascending
  uint32_t* pblk_ = nullptr;    // pushed count per chunk
  std::vector<uint32_t> prov_first_st_, prov_count_st_;  // per scene, as staged on the device
  bool walls_any_ = false;      // some scene has providers (selects the walls kernels)
  vxl_status stage_walls();
  // contact tables (any ProviderColliders, gathered by the caller once per tick): per side
  // (0 mirror, 1 projection) and scene, the entries' scene-local fluid ids, their plane
  // offsets and the planes (point xyz, normal xyz); on the device, all scenes' tables
  // concatenated with global reference ids
  std::vector<std::vector<uint32_t>> ct_ids_h_[2], ct_start_h_[2];
  std::vector<std::vector<float>> ct_pl_h_[2];
  uint32_t* ct_ent_d_[2] = {nullptr, nullptr};  // per global reference index: entry + 1, 0 = none
  uint32_t* ct_ids_d_[2] = {nullptr, nullptr};
  uint32_t* ct_start_d_[2] = {nullptr, nullptr};
  float4* ct_pl_d_[2] = {nullptr, nullptr};
  uint64_t ct_ids_cap_[2] = {0, 0}, ct_pl_cap_[2] = {0, 0};
  bool scene_has_table(uint32_t q) const;
  vxl_status upload_tables();
  ContactTableDev ctab(int side) const;
  float* snap_h_ = nullptr;  // pinned, 3 floats per slot
  float* snap_d_ = nullptr;  // device copy in reference order, the source of the host copy
  uint64_t snap_cap_ = 0, snap_n_ = 0;
  cudaEvent_t ev_snap_ = nullptr, ev_snap_ready_ = nullptr;
  cudaStream_t snap_stream_ = nullptr;  // the host copy runs here, beside the next tick's kernels
  bool snap_pending_ = false;
  float* stage_ = nullptr;  // 8 floats per slot: staging for host transfers
  // cells (cell_cap_ + 1)
  uint32_t* counts_ = nullptr;
  uint32_t* wet_ = nullptr;  // per cell: the substep epoch of the last substep it held fluid
  uint32_t* start_ = nullptr;
  uint32_t* partial_ = nullptr;
  // scenes / tiles / control
  SceneDev* sc_d_ = nullptr;
  SceneDev* sc_h_ = nullptr;  // pinned mirror (pushed when dt or membership changes)
  TileDev* tiles_d_ = nullptr;
  std::vector<TileDev>* tiles_h_ = nullptr;
  uint32_t ntiles_ = 0, nbtiles_ = 0, tiles_cap_ = 0;
  EngineCtl* ctl_d_ = nullptr;
  EngineCtl* ctl_h_ = nullptr;  // pinned
  // reactions
  std::vector<std::vector<vxl_sph_span>> spans_local_;
  SpanDev* spans_d_ = nullptr;
  SpanDev* spans_h_ = nullptr;  // pinned
  LongSpan* longs_d_ = nullptr;
  LongSpan* longs_h_ = nullptr;  // pinned
  float* breact_d_ = nullptr;
  float* breact_h_ = nullptr;  // pinned
  uint32_t nspans_ = 0, nlongs_ = 0, spans_cap_ = 0, longs_cap_ = 0;
  bool spans_dirty_ = true;
  std::vector<uint32_t> span_scene_;  // scene of each global span (for the results)

  bool record_ = false;
  bool ran_substep_ = false;
  bool use_graph_ = true;
  Tuning tuning_;
  int grid_density_ = 0, grid_force_ = 0, grid_bforce_ = 0;
  int grid_seg_ = 148;  // persistent grid of the grouped density pass (SMs x resident blocks)
  // graph of one tick
  cudaGraphExec_t graph_ = nullptr;
  uint32_t graph_epoch_ = 0;
  uint32_t graph_key_ = 0;
  uint32_t membership_epoch_ = 0;
  uint64_t launches_counter_ = 0, launches_last_tick_ = 0;
  // profiling
  bool prof_ = false, capturing_ = false, prof_pending_ = false;
  std::vector<cudaEvent_t> prof_ev_;
  std::vector<int> prof_kid_;
  size_t prof_used_ = 0;
  double prof_ms_[24] = {};
  uint64_t prof_n_[24] = {};
};

// Thread-local error message shared by all entry points (vxl_sph_last_error).
vxl_status set_error(vxl_status s, const std::string& msg);

}  // namespace vxl
