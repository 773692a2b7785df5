// Host orchestration of the multi-scene WCSPH engine: allocation, scene admission and
// repacking, the tile work list, substep/tick launch sequences (captured as CUDA graphs),
// per-kernel device timers, and the per-scene export paths.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "sph_engine.cuh"
#include "sph_engine.h"
#include "vxl_sph_internal.h"

namespace vxl {

namespace {

thread_local std::string g_last_error;

#define CU(call)                                                                                 \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) return set_error(VXL_CUDA_ERROR, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

constexpr int kThreads = 256;
constexpr uint32_t kBoundaryTile = 128;  // boundary particles per tile of the reaction pass
inline uint32_t blocks_for(uint64_t n, int t = kThreads) { return (uint32_t)((n + t - 1) / t); }

enum KernelId : int {
  KID_CELLOFF, KID_KEYS, KID_SCAN_PARTIAL, KID_SCAN_FINAL, KID_PLACE, KID_CANON,
  KID_DENSITY, KID_FORCE, KID_BFORCE, KID_REACT_LONG, KID_REACT_SPANS, KID_SCALE, KID_HALFMASK, KID_WALLS,
  KID_GROUPS, KID_COUNT
};
const char* const kKernelNames[KID_COUNT] = {
    "k_celloff", "k_keys", "k_scan_partial", "k_scan_final", "k_place", "k_canon",
    "k_density", "k_force", "k_bforce", "k_react_long", "k_react_spans", "k_scale", "k_halfmask", "k_walls",
    "k_groups"};
constexpr int kSegWarps = 8;  // warps per block of the grouped density pass

constexpr size_t kSceneHostBytes = offsetof(SceneDev, g);

// crates/vxl-phys-fluid/src/fluid_access.rs:8-13: h, h2, k6, ks, w0, B in f32 with the
// reference's operation order (host code is built with -ffp-contract=off).
SphConst make_const(const vxl_sph_params& p, uint64_t nf, uint64_t nt, uint32_t max_bins) {
  SphConst k{};
  const float h = std::fmax(p.smoothing_radius, 1e-5f);
  const float h2 = h * h;
  const float pi = 3.14159265358979323846f;
  k.h = h;
  k.h2 = h2;
  k.k6 = 315.0f / (64.0f * pi * vxl_powi(h, 9));
  k.ks = 45.0f / (pi * vxl_powi(h, 6));
  k.w0 = k.k6 * h2 * h2 * h2;
  k.b_tait = p.sound_speed * p.sound_speed * p.rest_density / p.gamma_tait;
  k.mass = p.particle_mass;
  k.rho0 = p.rest_density;
  k.gamma = p.gamma_tait;
  k.eps = p.xsph_viscosity;
  k.alpha_c = p.artificial_viscosity * p.sound_speed;
  k.h001 = 0.01f * h2;
  k.gx = p.gravity[0];
  k.gy = p.gravity[1];
  k.gz = p.gravity[2];
  k.clamp_p = p.tensile_instability_suppression ? 1u : 0u;
  k.gamma7 = std::fabs(p.gamma_tait - 7.0f) < 1e-6f ? 1u : 0u;
  k.n_fluid = (uint32_t)nf;
  k.n_total = (uint32_t)nt;
  k.max_bins = max_bins;
  return k;
}

}  // namespace

vxl_status set_error(vxl_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

}  // namespace vxl

// Shared by every translation unit of the library (declared in vxl_sph_internal.h).
void vxl_set_last_error(const char* msg) { vxl::set_error(VXL_OK, msg ? msg : ""); }
const char* vxl_get_last_error() { return vxl::g_last_error.c_str(); }

namespace vxl {

uint64_t Engine::bytes_per_slot(uint32_t nbr_cap) {
  // pos, vel (x2), orig, slot_of, cellrank, items, rc, press, acc, xsph, bforce, bpos,
  // neighbour list + count, staging, half masks, density thread orders (walls variant and
  // grouped pass), density segments
  return 4 * 16 + 4 + 4 + 8 + 8 + 8 + 4 + 16 + 16 + 16 + 16 + (uint64_t)nbr_cap * 2 + 4 + 32 + 1 + 4 + 4 + 8;
}

uint64_t Engine::bytes_per_cell() { return 12; }  // counts, start, wet

template <class T>
vxl_status Engine::dalloc(T** p, size_t count) {
  size_t bytes = count * sizeof(T);
  if (bytes == 0) bytes = sizeof(T);
  cudaError_t e = cudaMalloc((void**)p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return set_error(VXL_OUT_OF_MEMORY, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  device_bytes_ += bytes;
  return VXL_OK;
}

vxl_status Engine::create(int device, uint64_t slot_cap, uint64_t cell_cap, uint32_t scene_cap, Engine** out) {
  *out = nullptr;
  if (slot_cap == 0) slot_cap = 1;
  if (slot_cap >= (1ull << 31)) return set_error(VXL_INVALID_ARGUMENT, "more than 2^31 particle slots");
  if (cell_cap == 0 || cell_cap >= (1ull << 31)) return set_error(VXL_INVALID_ARGUMENT, "cell capacity out of range");
  auto* e = new (std::nothrow) Engine();
  if (!e) return set_error(VXL_OUT_OF_MEMORY, "host allocation failed");
  e->device_ = device;
  e->slot_cap_ = slot_cap;
  e->cell_cap_ = cell_cap;
  e->scene_cap_ = scene_cap ? scene_cap : 1;
  e->tiles_h_ = new std::vector<TileDev>();
  cudaError_t ce = cudaSetDevice(device);
  if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&e->own_stream_, cudaStreamNonBlocking);
  if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&e->side_, cudaStreamNonBlocking);
  if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->ev_fork_, cudaEventDisableTiming);
  if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->ev_join_, cudaEventDisableTiming);
  if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&e->react_, cudaStreamNonBlocking);
  if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->ev_rfork_, cudaEventDisableTiming);
  if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->ev_rjoin_, cudaEventDisableTiming);
  if (ce != cudaSuccess) {
    cudaGetLastError();
    delete e;  // the destructor releases tiles_h_
    return set_error(VXL_CUDA_ERROR, std::string("no usable CUDA device: ") + cudaGetErrorString(ce));
  }
  e->stream_ = e->own_stream_;
  vxl_status s = e->alloc_all();
  if (s != VXL_OK) {
    delete e;
    return s;
  }
  e->set_tuning(Tuning{});
  *out = e;
  return VXL_OK;
}

vxl_status Engine::alloc_all() {
  vxl_status s = VXL_OK;
  auto A = [&](vxl_status r) {
    if (s == VXL_OK) s = r;
  };
  const size_t n = slot_cap_;
  A(dalloc((float4**)&pos_[0], n));
  A(dalloc((float4**)&pos_[1], n));
  A(dalloc((float4**)&vel_[0], n));
  A(dalloc((float4**)&vel_[1], n));
  A(dalloc(&orig_, n));
  A(dalloc(&slot_of_, n));
  A(dalloc((uint2**)&cellrank_, n));
  A(dalloc((uint2**)&items_, n));
  A(dalloc((float2**)&rc_, n));
  A(dalloc(&press_, n));
  A(dalloc((float4**)&acc_, n));
  A(dalloc((float4**)&xsph_, n));
  A(dalloc((float4**)&bforce_, n));
  A(dalloc((float4**)&bpos_, n));
  A(dalloc(&nbr_, (size_t)nbr_cap_ * n));
  A(dalloc(&nbr_n_, n));
  A(dalloc(&halves_, 4 * (n / 32 + 2)));
  A(dalloc(&stage_, 8 * n));
  A(dalloc(&counts_, cell_cap_ + 1));
  A(dalloc(&wet_, cell_cap_ + 1));
  A(dalloc(&xorder_, slot_cap_));
  A(dalloc(&order_, slot_cap_));
  A(dalloc((uint2**)&segs_, slot_cap_));
  A(dalloc(&start_, cell_cap_ + 1));
  A(dalloc(&partial_, cell_cap_ / kScanTile + 2));
  A(dalloc(&sc_d_, scene_cap_));
  tiles_cap_ = (uint32_t)(n / 64 + 2ull * scene_cap_ + 2);  // particle tiles (>= 128 slots) + boundary tiles
  A(dalloc(&tiles_d_, tiles_cap_));
  A(dalloc(&ctl_d_, 1));
  if (s != VXL_OK) return s;
  CU(cudaMallocHost((void**)&sc_h_, scene_cap_ * sizeof(SceneDev)));
  CU(cudaMallocHost((void**)&ctl_h_, sizeof(EngineCtl)));
  std::memset(sc_h_, 0, scene_cap_ * sizeof(SceneDev));
  std::memset(ctl_h_, 0, sizeof(EngineCtl));
  CU(cudaMemsetAsync(counts_, 0, (cell_cap_ + 1) * 4, stream_));
  CU(cudaMemsetAsync(wet_, 0, (cell_cap_ + 1) * 4, stream_));
  CU(cudaMemsetAsync(start_, 0, (cell_cap_ + 1) * 4, stream_));
  CU(cudaMemsetAsync(ctl_d_, 0, sizeof(EngineCtl), stream_));
  CU(cudaMemsetAsync(sc_d_, 0, scene_cap_ * sizeof(SceneDev), stream_));
  CU(cudaMemsetAsync(acc_, 0, n * 16, stream_));
  CU(cudaMemsetAsync(xsph_, 0, n * 16, stream_));
  CU(cudaMemsetAsync(bforce_, 0, n * 16, stream_));
  CU(cudaMemsetAsync(rc_, 0, n * 8, stream_));
  CU(cudaMemsetAsync(press_, 0, n * 4, stream_));
  CU(cudaStreamSynchronize(stream_));
  return VXL_OK;
}

void Engine::free_all() {
  if (graph_) cudaGraphExecDestroy(graph_);
  graph_ = nullptr;
  void* d[] = {pos_[0], pos_[1], vel_[0], vel_[1], orig_, slot_of_, cellrank_, items_, rc_, press_, acc_, xsph_,
               bforce_, bpos_, nbr_, nbr_n_, halves_, xorder_, order_, segs_, stage_, counts_, wet_, start_, partial_, sc_d_, tiles_d_, ctl_d_, spans_d_,
               longs_d_, breact_d_};
  for (void* p : d)
    if (p) cudaFree(p);
  void* hp[] = {sc_h_, ctl_h_, spans_h_, longs_h_, breact_h_};
  for (void* p : hp)
    if (p) cudaFreeHost(p);
  if (snap_h_) cudaFreeHost(snap_h_);
  snap_h_ = nullptr;
  if (snap_d_) cudaFree(snap_d_);
  snap_d_ = nullptr;
  if (ev_snap_) cudaEventDestroy(ev_snap_);
  ev_snap_ = nullptr;
  if (ev_snap_ready_) cudaEventDestroy(ev_snap_ready_);
  ev_snap_ready_ = nullptr;
  if (snap_stream_) cudaStreamDestroy(snap_stream_);
  snap_stream_ = nullptr;
  if (rb_d_) cudaFree(rb_d_);
  rb_d_ = nullptr;
  void* wd[] = {prov_d_,      wplanes_d_,    pflag_,        pnsum_,        plist_,   pblk_,
                ct_ent_d_[0], ct_ent_d_[1],  ct_ids_d_[0],  ct_ids_d_[1],  ct_start_d_[0],
                ct_start_d_[1], ct_pl_d_[0], ct_pl_d_[1]};
  for (void* p : wd)
    if (p) cudaFree(p);
  prov_d_ = nullptr;
  wplanes_d_ = nullptr;
  pflag_ = plist_ = pblk_ = nullptr;
  for (int k = 0; k < 2; ++k) {
    ct_ent_d_[k] = ct_ids_d_[k] = ct_start_d_[k] = nullptr;
    ct_pl_d_[k] = nullptr;
  }
  pnsum_ = nullptr;
  if (blocal_) cudaFree(blocal_);
  if (poses_d_) cudaFree(poses_d_);
  blocal_ = nullptr;
  poses_d_ = nullptr;
  for (cudaEvent_t e : prof_ev_) cudaEventDestroy(e);
  prof_ev_.clear();
  if (own_stream_) cudaStreamDestroy(own_stream_);
  own_stream_ = nullptr;
  if (side_) cudaStreamDestroy(side_);
  side_ = nullptr;
  if (ev_fork_) cudaEventDestroy(ev_fork_);
  if (ev_join_) cudaEventDestroy(ev_join_);
  ev_fork_ = ev_join_ = nullptr;
  if (react_) cudaStreamDestroy(react_);
  react_ = nullptr;
  if (ev_rfork_) cudaEventDestroy(ev_rfork_);
  if (ev_rjoin_) cudaEventDestroy(ev_rjoin_);
  ev_rfork_ = ev_rjoin_ = nullptr;
}

Engine::~Engine() {
  cudaSetDevice(device_);
  if (stream_) cudaStreamSynchronize(stream_);
  if (side_) cudaStreamSynchronize(side_);
  if (react_) cudaStreamSynchronize(react_);
  free_all();
  delete tiles_h_;
}

void Engine::set_stream(cudaStream_t s) {
  prof_collect();
  cudaStreamSynchronize(stream_);
  stream_ = s ? s : own_stream_;
}

void Engine::set_tuning(const Tuning& t) {
  tuning_ = t;
  if (tuning_.block != 128 && tuning_.block != 256) tuning_.block = 256;
  if (tuning_.tile < tuning_.block) tuning_.tile = tuning_.block;
  tuning_.tile = (tuning_.tile / 128) * 128;
  if (tuning_.waves > 4) tuning_.waves = 4;
  if (tuning_.density > 1) tuning_.density = 0;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_);
  int occ_d = 1, occ_f = 1, occ_b = 1;
  if (tuning_.block == 128) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_d, k_e_density<128>, 128, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_f, k_e_force<128>, 128, 0);
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_d, k_e_density<256>, 256, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_f, k_e_force<256>, 256, 0);
  }
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_b, k_e_bforce, 128, 0);
  int occ_s = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_s, k_e_density_seg<kSegWarps>, kSegWarps * 32, 0);
  grid_seg_ = sms * std::max(1, occ_s);
  cudaGetLastError();
  // waves == 0: one block per tile (the grid is sized from the tile count at launch)
  grid_density_ = sms * std::max(1, occ_d) * (int)tuning_.waves;
  grid_force_ = sms * std::max(1, occ_f) * (int)tuning_.waves;
  grid_bforce_ = tuning_.waves ? sms * std::max(1, occ_b) : 0;
  if (graph_) {
    cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
  }
  rebuild_tiles();
}

vxl_status Engine::rebuild_tiles() {
  tiles_h_->clear();
  for (uint32_t q = 0; q < scenes_.size(); ++q) {
    const SceneInfo& si = scenes_[q];
    const uint32_t n = si.nf + si.nb;
    for (uint32_t f = 0; f < n; f += tuning_.tile)
      tiles_h_->push_back(TileDev{q, si.base + f, std::min(tuning_.tile, n - f), 0u});
  }
  ntiles_ = (uint32_t)tiles_h_->size();
  // boundary tiles (reference order) of the reaction pass, after the particle tiles
  for (uint32_t q = 0; q < scenes_.size(); ++q) {
    const SceneInfo& si = scenes_[q];
    for (uint32_t f = 0; f < si.nb; f += kBoundaryTile)
      tiles_h_->push_back(TileDev{q, si.base + si.nf + f, std::min(kBoundaryTile, si.nb - f), 0u});
  }
  nbtiles_ = (uint32_t)tiles_h_->size() - ntiles_;
  if (ntiles_ + nbtiles_ > tiles_cap_) return set_error(VXL_INVALID_ARGUMENT, "tile list above capacity");
  if (!tiles_h_->empty()) {
    CU(cudaMemcpyAsync(tiles_d_, tiles_h_->data(), tiles_h_->size() * sizeof(TileDev), cudaMemcpyHostToDevice,
                       stream_));
    CU(cudaStreamSynchronize(stream_));
  }
  ++membership_epoch_;
  return VXL_OK;
}

// Push the host-written part of every scene record (constants, dt, slot range).
vxl_status Engine::push_scene_records(const std::vector<float>& dt) {
  for (uint32_t q = 0; q < scenes_.size(); ++q) {
    SceneDev& r = sc_h_[q];
    const SceneInfo& si = scenes_[q];
    r.k = make_const(si.params, si.nf, si.nf + si.nb, si.params.max_bins ? si.params.max_bins : (1u << 21));
    r.k.mass = si.particle_mass;
    r.dt = dt.empty() ? 0.f : dt[q];
    r.vmax = r.dt > 0.f ? si.params.max_speed_frac * r.k.h / r.dt : 0.f;  // fluid_step.rs:112
    r.vmax2 = r.vmax * r.vmax;
    r.base = si.base;
    r.count = si.nf + si.nb;
    r.prov_first = q < prov_first_st_.size() ? prov_first_st_[q] : 0u;
    r.prov_count = q < prov_count_st_.size() ? prov_count_st_[q] : 0u;
  }
  if (!scenes_.empty()) {
    CU(cudaMemcpy2DAsync(sc_d_, sizeof(SceneDev), sc_h_, sizeof(SceneDev), kSceneHostBytes, scenes_.size(),
                         cudaMemcpyHostToDevice, stream_));
    CU(cudaStreamSynchronize(stream_));
  }
  return VXL_OK;
}

vxl_status Engine::recompute_scene_boxes(uint32_t q) {
  static const uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
  const SceneInfo& si = scenes_[q];
  const uint32_t n = si.nf + si.nb;
  CU(cudaMemcpyAsync(sc_d_[q].fbox, init, sizeof(init), cudaMemcpyHostToDevice, stream_));
  CU(cudaMemcpyAsync(sc_d_[q].bbox, init, sizeof(init), cudaMemcpyHostToDevice, stream_));
  if (n) {
    k_e_bbox<<<blocks_for(n), kThreads, 0, stream_>>>((const float4*)pos_[0], si.base, n, 1, sc_d_[q].fbox);
    k_e_bbox<<<blocks_for(n), kThreads, 0, stream_>>>((const float4*)pos_[0], si.base, n, 0, sc_d_[q].bbox);
  }
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(stream_));
  return VXL_OK;
}

vxl_status Engine::add_scene(const vxl_sph_params& p, uint64_t nf, uint64_t nb, const float* pos, const float* vel,
                             const float* pmass, uint64_t id, uint32_t* out_index) {
  const uint64_t nt = nf + nb;
  if (nt > 0 && (!pos || !vel)) return set_error(VXL_NULL_POINTER, "pos/vel is NULL");
  if (nb > 0 && !pmass) return set_error(VXL_NULL_POINTER, "pmass is NULL with boundary particles");
  const uint32_t max_bins = p.max_bins ? p.max_bins : (1u << 21);
  if (max_bins > (1u << 21)) return set_error(VXL_INVALID_ARGUMENT, "max_bins above 2^21");
  if (!(p.particle_mass > 0.0f) || !(p.rest_density > 0.0f) || !(p.gamma_tait > 0.0f))
    return set_error(VXL_INVALID_ARGUMENT, "particle_mass, rest_density and gamma_tait must be positive");
  if (pmass)
    for (uint64_t i = 0; i < nf; ++i)
      if (pmass[i] != p.particle_mass) return set_error(VXL_INVALID_ARGUMENT, "fluid pmass must equal params.particle_mass");
  for (uint64_t i = nf; i < nt; ++i)
    if (!(pmass[i] > 0.0f)) return set_error(VXL_INVALID_ARGUMENT, "boundary pmass must be positive");
  if (used_ + nt > slot_cap_) return set_error(VXL_OUT_OF_MEMORY, "particle pool full");
  if (scenes_.size() >= scene_cap_) return set_error(VXL_OUT_OF_MEMORY, "scene table full");
  CU(cudaSetDevice(device_));
  prof_collect();
  CU(cudaStreamSynchronize(stream_));
  SceneInfo si;
  si.id = id;
  si.base = (uint32_t)used_;
  si.nf = (uint32_t)nf;
  si.nb = (uint32_t)nb;
  si.substeps = p.substeps ? p.substeps : 1;
  si.particle_mass = p.particle_mass;
  si.params = p;
  si.params.max_bins = max_bins;
  const uint32_t q = (uint32_t)scenes_.size();
  scenes_.push_back(si);
  used_ += nt;
  if (nt) {
    CU(cudaMemcpyAsync(stage_, pos, nt * 12, cudaMemcpyHostToDevice, stream_));
    CU(cudaMemcpyAsync(stage_ + 3 * nt, vel, nt * 12, cudaMemcpyHostToDevice, stream_));
    if (nb) CU(cudaMemcpyAsync(stage_ + 6 * nt, pmass, nt * 4, cudaMemcpyHostToDevice, stream_));
    k_e_init_scene<<<blocks_for(nt), kThreads, 0, stream_>>>(stage_, stage_ + 3 * nt, stage_ + 6 * nt,
                                                              (float4*)pos_[0], (float4*)vel_[0], orig_, slot_of_,
                                                              (float4*)bpos_, si.base, (uint32_t)nt, (uint32_t)nf,
                                                              p.particle_mass);
    CU(cudaGetLastError());
  }
  vxl_status s = push_scene_records({});
  if (s == VXL_OK) s = recompute_scene_boxes(q);
  if (s == VXL_OK) s = rebuild_tiles();
  spans_local_.resize(scenes_.size());
  scene_bodies_.resize(scenes_.size(), 0);
  spans_dirty_ = true;
  if (out_index) *out_index = q;
  return s;
}

vxl_status Engine::remove_scenes(const std::vector<uint32_t>& indices) {
  if (indices.empty()) return VXL_OK;
  CU(cudaSetDevice(device_));
  prof_collect();
  CU(cudaStreamSynchronize(stream_));
  {
    vxl_status pst = rb_pull();  // coupled bodies' evolved states, in the old layout
    if (pst != VXL_OK) return pst;
  }
  std::vector<bool> drop(scenes_.size(), false);
  for (uint32_t i : indices)
    if (i < scenes_.size()) drop[i] = true;
  std::vector<SceneInfo> keep;
  std::vector<std::vector<vxl_sph_span>> keep_spans;
  std::vector<uint32_t> keep_bodies;
  std::vector<uint4> moves;
  uint32_t next = 0;
  for (uint32_t q = 0; q < scenes_.size(); ++q) {
    if (drop[q]) continue;
    SceneInfo si = scenes_[q];
    const uint32_t n = si.nf + si.nb;
    moves.push_back(make_uint4(si.base, next, n, 0u));
    si.base = next;
    next += n;
    keep.push_back(si);
    keep_spans.push_back(q < spans_local_.size() ? spans_local_[q] : std::vector<vxl_sph_span>());
    keep_bodies.push_back(q < scene_bodies_.size() ? scene_bodies_[q] : 0u);
  }
  // copy every kept scene into the second buffer set at its new base, then back
  if (!moves.empty() && next > 0) {
    uint4* moves_d = (uint4*)stage_;  // staging holds >= 8 floats per slot
    CU(cudaMemcpyAsync(moves_d, moves.data(), moves.size() * sizeof(uint4), cudaMemcpyHostToDevice, stream_));
    uint32_t* orig_tmp = (uint32_t*)items_;
    float4* bpos_tmp = (float4*)bforce_;
    uint32_t maxn = 0;
    for (auto& m : moves) maxn = std::max(maxn, m.z);
    dim3 grid(std::max(1u, std::min(blocks_for(maxn), 1024u)), (uint32_t)moves.size());
    k_e_move<<<grid, kThreads, 0, stream_>>>((const float4*)pos_[0], (const float4*)vel_[0], orig_,
                                             (const float4*)bpos_, (float4*)pos_[1], (float4*)vel_[1], orig_tmp,
                                             bpos_tmp, moves_d);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(pos_[0], pos_[1], (size_t)next * 16, cudaMemcpyDeviceToDevice, stream_));
    CU(cudaMemcpyAsync(vel_[0], vel_[1], (size_t)next * 16, cudaMemcpyDeviceToDevice, stream_));
    CU(cudaMemcpyAsync(orig_, orig_tmp, (size_t)next * 4, cudaMemcpyDeviceToDevice, stream_));
    CU(cudaMemcpyAsync(bpos_, bpos_tmp, (size_t)next * 16, cudaMemcpyDeviceToDevice, stream_));
    if (blocal_) {  // body lattices move with their scenes (reference order, like bpos)
      float4* tmp = (float4*)xsph_;
      for (auto& m : moves)
        if (m.z) CU(cudaMemcpyAsync(tmp + m.y, blocal_ + m.x, (size_t)m.z * 16, cudaMemcpyDeviceToDevice, stream_));
      CU(cudaMemcpyAsync(blocal_, tmp, (size_t)next * 16, cudaMemcpyDeviceToDevice, stream_));
    }
    k_e_slot_of<<<blocks_for(next), kThreads, 0, stream_>>>(orig_, slot_of_, next);
    CU(cudaGetLastError());
  }
  scenes_.swap(keep);
  spans_local_.swap(keep_spans);
  scene_bodies_.swap(keep_bodies);
  if (!prov_h_.empty()) {  // provider walls follow their scenes
    std::vector<std::vector<vxl_sph_provider>> kp;
    std::vector<std::vector<vxl_sph_wall_plane>> kw;
    for (uint32_t q = 0; q < drop.size(); ++q)
      if (!drop[q]) {
        kp.push_back(q < prov_h_.size() ? prov_h_[q] : std::vector<vxl_sph_provider>());
        kw.push_back(q < wplanes_h_.size() ? wplanes_h_[q] : std::vector<vxl_sph_wall_plane>());
      }
    prov_h_.swap(kp);
    wplanes_h_.swap(kw);
    prov_first_st_.clear();  // restaged below, after the slots have moved
    prov_count_st_.clear();
  }
  for (int side = 0; side < 2; ++side) {  // contact tables follow their scenes
    if (ct_ids_h_[side].empty()) continue;
    std::vector<std::vector<uint32_t>> ki, ks;
    std::vector<std::vector<float>> kpl;
    for (uint32_t q = 0; q < drop.size(); ++q)
      if (!drop[q] && q < ct_ids_h_[side].size()) {
        ki.push_back(ct_ids_h_[side][q]);
        ks.push_back(ct_start_h_[side][q]);
        kpl.push_back(ct_pl_h_[side][q]);
      }
    ct_ids_h_[side].swap(ki);
    ct_start_h_[side].swap(ks);
    ct_pl_h_[side].swap(kpl);
  }
  if (!rigid_.empty()) {  // coupled bodies follow their scenes
    std::vector<std::vector<vxl_sph_rigid_body>> keep_rigid;
    for (uint32_t q = 0; q < drop.size(); ++q)
      if (!drop[q]) keep_rigid.push_back(q < rigid_.size() ? rigid_[q] : std::vector<vxl_sph_rigid_body>());
    rigid_.swap(keep_rigid);
    rb_dirty_ = true;
    rb_have_reaction_ = false;
  }
  used_ = next;
  spans_dirty_ = true;
  vxl_status s = push_scene_records({});
  for (uint32_t q = 0; s == VXL_OK && q < scenes_.size(); ++q) s = recompute_scene_boxes(q);
  if (s == VXL_OK) s = rebuild_tiles();
  if (s == VXL_OK && !prov_h_.empty()) s = stage_walls();
  return s;
}

vxl_status Engine::upload_boundary(uint32_t q, const float* pos, const float* vel, uint64_t nb) {
  if (q >= scenes_.size()) return set_error(VXL_INVALID_ARGUMENT, "scene index out of range");
  const SceneInfo& si = scenes_[q];
  if (nb != si.nb) return set_error(VXL_SIZE_MISMATCH, "boundary segment length differs from the scene (rebuild the scene)");
  if (nb == 0) return VXL_OK;
  if (!pos || !vel) return set_error(VXL_NULL_POINTER, "pos/vel is NULL");
  CU(cudaSetDevice(device_));
  static const uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
  CU(cudaMemcpyAsync(stage_, pos, nb * 12, cudaMemcpyHostToDevice, stream_));
  CU(cudaMemcpyAsync(stage_ + 3 * nb, vel, nb * 12, cudaMemcpyHostToDevice, stream_));
  CU(cudaMemcpyAsync(sc_d_[q].bbox, init, sizeof(init), cudaMemcpyHostToDevice, stream_));
  k_e_upload_boundary<<<blocks_for(nb), kThreads, 0, stream_>>>(stage_, stage_ + 3 * nb, (float4*)pos_[0],
                                                                 (float4*)vel_[0], slot_of_, (float4*)bpos_,
                                                                 sc_d_[q].bbox, si.base, si.nf, si.nb);
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(stream_));  // the caller's arrays are borrowed for this call only
  return VXL_OK;
}

vxl_status Engine::set_body_lattice(uint32_t q, const float* local_xyz, const uint32_t* body_index, uint64_t nb,
                                    uint32_t nbodies) {
  if (q >= scenes_.size()) return set_error(VXL_INVALID_ARGUMENT, "scene index out of range");
  const SceneInfo& si = scenes_[q];
  if (nb != si.nb) return set_error(VXL_SIZE_MISMATCH, "lattice length differs from the boundary segment");
  if (nb == 0) return VXL_OK;
  if (!local_xyz || !body_index) return set_error(VXL_NULL_POINTER, "lattice arrays are NULL");
  if (nbodies == 0) return set_error(VXL_INVALID_ARGUMENT, "nbodies must be > 0");
  for (uint64_t k = 0; k < nb; ++k)
    if (body_index[k] >= nbodies) return set_error(VXL_INVALID_ARGUMENT, "body index past nbodies");
  CU(cudaSetDevice(device_));
  if (!blocal_) {
    vxl_status st = dalloc(&blocal_, slot_cap_);
    if (st != VXL_OK) return st;
  }
  std::vector<float4> h(nb);
  for (uint64_t k = 0; k < nb; ++k) {
    uint32_t b = body_index[k];
    float w;
    std::memcpy(&w, &b, 4);
    h[k] = make_float4(local_xyz[3 * k], local_xyz[3 * k + 1], local_xyz[3 * k + 2], w);
  }
  CU(cudaMemcpyAsync(blocal_ + si.base + si.nf, h.data(), nb * sizeof(float4), cudaMemcpyHostToDevice, stream_));
  CU(cudaStreamSynchronize(stream_));
  if (scene_bodies_.size() < scenes_.size()) scene_bodies_.resize(scenes_.size(), 0);
  scene_bodies_[q] = nbodies;
  return VXL_OK;
}

// ---------------------------------------------------------------- coupled rigid bodies

static RigidBodyDev to_dev(const vxl_sph_rigid_body& b) {
  const vxl_sph_body_pose& p = b.pose;
  return RigidBodyDev{p.pos[0], p.pos[1], p.pos[2], p.rot[0], p.rot[1], p.rot[2], p.rot[3],
                      p.linvel[0], p.linvel[1], p.linvel[2], p.angvel[0], p.angvel[1], p.angvel[2],
                      b.inv_mass, b.local_inv_inertia[0], b.local_inv_inertia[1], b.local_inv_inertia[2],
                      b.dynamic ? 1u : 0u, ~0u};
}

static void from_dev(const RigidBodyDev& d, vxl_sph_rigid_body& b) {
  vxl_sph_body_pose& p = b.pose;
  p.pos[0] = d.px; p.pos[1] = d.py; p.pos[2] = d.pz;
  p.rot[0] = d.qx; p.rot[1] = d.qy; p.rot[2] = d.qz; p.rot[3] = d.qw;
  p.linvel[0] = d.vx; p.linvel[1] = d.vy; p.linvel[2] = d.vz;
  p.angvel[0] = d.wx; p.angvel[1] = d.wy; p.angvel[2] = d.wz;
}

// Bring the device's evolved bodies back into the host copies (before the device array
// is rebuilt from them).
vxl_status Engine::rb_pull() {
  if (!rb_live_ || !rb_d_ || rb_n_ == 0) return VXL_OK;
  std::vector<RigidBodyDev> h(rb_n_);
  CU(cudaMemcpyAsync(h.data(), rb_d_, rb_n_ * sizeof(RigidBodyDev), cudaMemcpyDeviceToHost, stream_));
  CU(cudaStreamSynchronize(stream_));
  for (uint32_t q = 0; q < rigid_.size() && q < rb_off_.size(); ++q)
    for (uint32_t b = 0; b < rigid_[q].size(); ++b) from_dev(h[rb_off_[q] + b], rigid_[q][b]);
  rb_live_ = false;
  return VXL_OK;
}

void Engine::rb_layout() {
  rb_off_.assign(scenes_.size(), 0);
  uint32_t n = 0;
  for (uint32_t q = 0; q < scenes_.size(); ++q) {
    rb_off_[q] = n;
    if (q < rigid_.size()) n += (uint32_t)rigid_[q].size();
  }
  rb_n_ = n;
}

vxl_status Engine::set_rigid_bodies(uint32_t q, const vxl_sph_rigid_body* bodies, uint32_t n) {
  if (q >= scenes_.size()) return set_error(VXL_INVALID_ARGUMENT, "scene index out of range");
  if (n && !bodies) return set_error(VXL_NULL_POINTER, "bodies is NULL");
  if (q >= scene_bodies_.size() || scene_bodies_[q] == 0)
    return set_error(VXL_NOT_READY, "set the body lattice (vxl_sph_set_body_lattice) first");
  if (n != scene_bodies_[q]) return set_error(VXL_SIZE_MISMATCH, "one rigid body per lattice body");
  for (uint32_t b = 0; b < n; ++b)
    if (bodies[b].dynamic && !(bodies[b].inv_mass > 0.0f))
      return set_error(VXL_INVALID_ARGUMENT, "a dynamic body needs inv_mass > 0");
  CU(cudaSetDevice(device_));
  prof_collect();
  vxl_status st = rb_pull();  // keep the other scenes' evolved bodies
  if (st != VXL_OK) return st;
  if (rigid_.size() < scenes_.size()) rigid_.resize(scenes_.size());
  rigid_[q].assign(bodies, bodies + n);
  rb_dirty_ = true;
  rb_have_reaction_ = false;
  spans_dirty_ = true;  // spans map to the bodies by id
  return VXL_OK;
}

vxl_status Engine::step_coupled_async(float dt_tick, uint32_t rigid_substeps, const float g[3], float max_linear,
                                      float max_angular) {
  if (!(dt_tick > 0.0f) || !std::isfinite(dt_tick)) return set_error(VXL_INVALID_ARGUMENT, "dt_tick must be > 0");
  if (rigid_substeps == 0) return set_error(VXL_INVALID_ARGUMENT, "rigid_substeps must be > 0");
  if (!g) return set_error(VXL_NULL_POINTER, "gravity is NULL");
  CU(cudaSetDevice(device_));
  bool any = false;
  for (auto& v : rigid_) any = any || !v.empty();
  if (!any) return set_error(VXL_NOT_READY, "no rigid bodies set (vxl_sph_set_rigid_bodies)");
  prof_collect();
  if (spans_dirty_ || rb_dirty_) {
    vxl_status st = rb_pull();
    if (st != VXL_OK) return st;
    rb_layout();
    st = stage_spans();  // maps spans to rigid bodies (needs rb_off_)
    if (st != VXL_OK) return st;
    std::vector<RigidBodyDev> h(rb_n_);
    for (uint32_t q = 0; q < rigid_.size(); ++q)
      for (uint32_t b = 0; b < rigid_[q].size(); ++b) h[rb_off_[q] + b] = to_dev(rigid_[q][b]);
    for (uint32_t k = 0; k < nspans_; ++k)
      if (spans_h_[k].rigid != ~0u) h[spans_h_[k].rigid].span = k;
    if (rb_n_ > rb_cap_) {
      if (rb_d_) cudaFree(rb_d_);
      rb_d_ = nullptr;
      rb_cap_ = 0;
      vxl_status s2 = dalloc(&rb_d_, rb_n_);
      if (s2 != VXL_OK) return s2;
      rb_cap_ = rb_n_;
      if (graph_) {  // the reaction kernels read the body array
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
      }
    }
    CU(cudaMemcpyAsync(rb_d_, h.data(), rb_n_ * sizeof(RigidBodyDev), cudaMemcpyHostToDevice, stream_));
    CU(cudaStreamSynchronize(stream_));
    rb_live_ = true;
    rb_dirty_ = false;
  }
  // 1. rigid substeps from the previous coupled tick's reactions
  const float dt = dt_tick / (float)rigid_substeps;
  k_rigid_step<<<blocks_for(rb_n_, 64), 64, 0, stream_>>>(rb_d_, rb_n_, breact_d_,
                                                           (rb_have_reaction_ && breact_d_) ? 1 : 0, g[0], g[1], g[2],
                                                           dt, rigid_substeps, max_linear, max_angular);
  CU(cudaGetLastError());
  // 2. boundary segments from the new poses
  static const uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
  for (uint32_t q = 0; q < scenes_.size(); ++q) {
    if (q >= rigid_.size() || rigid_[q].empty() || scenes_[q].nb == 0) continue;
    const SceneInfo& si = scenes_[q];
    CU(cudaMemcpyAsync(sc_d_[q].bbox, init, sizeof(init), cudaMemcpyHostToDevice, stream_));
    k_e_body_rebuild<<<blocks_for(si.nb), kThreads, 0, stream_>>>(blocal_, rb_d_ + rb_off_[q], (float4*)pos_[0],
                                                                   (float4*)vel_[0], slot_of_, (float4*)bpos_,
                                                                   sc_d_[q].bbox, si.base, si.nf, si.nb);
    CU(cudaGetLastError());
  }
  // 3. the fluid tick; its tick-averaged reactions drive the next call's rigid substeps
  vxl_status st = step_tick_async(dt_tick);
  if (st != VXL_OK) return st;
  rb_have_reaction_ = nspans_ > 0;
  return VXL_OK;
}

// ---------------------------------------------------------------- provider walls

bool Engine::scene_has_table(uint32_t q) const {
  for (int side = 0; side < 2; ++side)
    if (q < ct_ids_h_[side].size() && !ct_ids_h_[side][q].empty()) return true;
  return false;
}

ContactTableDev Engine::ctab(int side) const {
  return ContactTableDev{ct_ent_d_[side], ct_start_d_[side], ct_pl_d_[side]};
}

// The contact tables of one side of a scene, as the reference's GPU tier uploads them per
// tick (WallStage::upload, crates/vxl-phys-gpu/src/pipeline/walls.rs:100-121).
vxl_status Engine::set_wall_contacts(uint32_t q, uint32_t side, const uint32_t* ids, const uint32_t* start,
                                     uint32_t n, const float* planes, uint32_t nplanes) {
  if (q >= scenes_.size()) return set_error(VXL_INVALID_ARGUMENT, "scene index out of range");
  if (side > 1u) return set_error(VXL_INVALID_ARGUMENT, "side must be 0 (mirror) or 1 (projection)");
  if (n && (!ids || !start)) return set_error(VXL_NULL_POINTER, "ids/start is NULL with entries");
  if (nplanes && !planes) return set_error(VXL_NULL_POINTER, "planes is NULL");
  const SceneInfo& si = scenes_[q];
  if (n) {
    if (start[0] != 0u || start[n] != nplanes) return set_error(VXL_SIZE_MISMATCH, "start must run from 0 to n_planes");
    for (uint32_t e = 0; e < n; ++e) {
      if (ids[e] >= si.nf) return set_error(VXL_INVALID_ARGUMENT, "contact id is not a fluid particle");
      if (e && ids[e] <= ids[e - 1]) return set_error(VXL_INVALID_ARGUMENT, "contact ids must ascend");
      if (start[e + 1] < start[e] || start[e + 1] - start[e] > kMaxWallPlanes)
        return set_error(VXL_INVALID_ARGUMENT, "each entry holds 0..8 planes");
    }
    for (uint64_t k = 0; k < 6ull * nplanes; ++k)
      if (!std::isfinite(planes[k])) return set_error(VXL_INVALID_ARGUMENT, "planes must be finite");
  } else if (nplanes) {
    return set_error(VXL_SIZE_MISMATCH, "planes without entries");
  }
  CU(cudaSetDevice(device_));
  prof_collect();
  for (int k = 0; k < 2; ++k)
    if (ct_ids_h_[k].size() < scenes_.size()) {
      ct_ids_h_[k].resize(scenes_.size());
      ct_start_h_[k].resize(scenes_.size());
      ct_pl_h_[k].resize(scenes_.size());
    }
  const bool had = scene_has_table(q);
  ct_ids_h_[side][q].assign(ids, ids + n);
  ct_start_h_[side][q].assign(start, start + (n ? n + 1 : 0));
  ct_pl_h_[side][q].assign(planes, planes + 6ull * nplanes);
  if (had != scene_has_table(q)) return stage_walls();  // the scene's provider list changes
  return upload_tables();
}

// All scenes' contact tables to the device (stream-ordered before the next tick); device
// arrays grow by doubling, and a tick graph that holds their old addresses is dropped.
vxl_status Engine::upload_tables() {
  bool any = false;
  for (int side = 0; side < 2; ++side)
    for (const auto& v : ct_ids_h_[side]) any = any || !v.empty();
  if (!any && !ct_ent_d_[0]) return VXL_OK;
  bool moved = false;
  for (int side = 0; side < 2; ++side) {
    std::vector<uint32_t> gids, gstart(1, 0u);
    std::vector<float4> gpl;
    for (uint32_t q = 0; q < scenes_.size() && q < ct_ids_h_[side].size(); ++q) {
      const auto& ids = ct_ids_h_[side][q];
      const auto& st = ct_start_h_[side][q];
      const auto& pl = ct_pl_h_[side][q];
      for (size_t e = 0; e < ids.size(); ++e) {
        gids.push_back((uint32_t)scenes_[q].base + ids[e]);
        for (uint32_t k = st[e]; k < st[e + 1]; ++k) {
          const float* c = &pl[6ull * k];
          gpl.push_back(make_float4(c[0], c[1], c[2], 0.0f));
          gpl.push_back(make_float4(c[3], c[4], c[5], 0.0f));
        }
        gstart.push_back((uint32_t)(gpl.size() / 2));
      }
    }
    if (!ct_ent_d_[side]) {
      vxl_status s = dalloc(&ct_ent_d_[side], slot_cap_);
      if (s != VXL_OK) return s;
      moved = true;
    }
    if (gids.size() + 1 > ct_ids_cap_[side]) {
      const uint64_t cap = std::max<uint64_t>(2 * ct_ids_cap_[side], gids.size() + 1);
      if (ct_ids_d_[side]) cudaFree(ct_ids_d_[side]);
      if (ct_start_d_[side]) cudaFree(ct_start_d_[side]);
      ct_ids_d_[side] = ct_start_d_[side] = nullptr;
      ct_ids_cap_[side] = 0;
      vxl_status s = dalloc(&ct_ids_d_[side], cap);
      if (s == VXL_OK) s = dalloc(&ct_start_d_[side], cap);
      if (s != VXL_OK) return s;
      ct_ids_cap_[side] = cap;
      moved = true;
    }
    if (gpl.size() + 2 > ct_pl_cap_[side]) {
      const uint64_t cap = std::max<uint64_t>(2 * ct_pl_cap_[side], gpl.size() + 2);
      if (ct_pl_d_[side]) cudaFree(ct_pl_d_[side]);
      ct_pl_d_[side] = nullptr;
      ct_pl_cap_[side] = 0;
      vxl_status s = dalloc(&ct_pl_d_[side], cap);
      if (s != VXL_OK) return s;
      ct_pl_cap_[side] = cap;
      moved = true;
    }
    CU(cudaMemsetAsync(ct_ent_d_[side], 0, std::max<uint64_t>(used_, 1) * 4, stream_));
    if (!gids.empty()) {
      CU(cudaMemcpyAsync(ct_ids_d_[side], gids.data(), gids.size() * 4, cudaMemcpyHostToDevice, stream_));
      CU(cudaMemcpyAsync(ct_start_d_[side], gstart.data(), gstart.size() * 4, cudaMemcpyHostToDevice, stream_));
      if (!gpl.empty())
        CU(cudaMemcpyAsync(ct_pl_d_[side], gpl.data(), gpl.size() * 16, cudaMemcpyHostToDevice, stream_));
      k_e_ctab_scatter<<<blocks_for(gids.size()), kThreads, 0, stream_>>>(ct_ids_d_[side], (uint32_t)gids.size(),
                                                                          ct_ent_d_[side]);
      CU(cudaGetLastError());
    }
  }
  // the host vectors are freed on return: wait until the pageable copies have been taken
  CU(cudaStreamSynchronize(stream_));
  if (moved && graph_) {
    cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
  }
  return VXL_OK;
}

vxl_status Engine::set_providers(uint32_t q, const vxl_sph_provider* pr, uint32_t n, const vxl_sph_wall_plane* planes,
                                 uint32_t nplanes) {
  if (q >= scenes_.size()) return set_error(VXL_INVALID_ARGUMENT, "scene index out of range");
  if (n && !pr) return set_error(VXL_NULL_POINTER, "providers is NULL");
  if (nplanes && !planes) return set_error(VXL_NULL_POINTER, "planes is NULL");
  if (n > VXL_SPH_MAX_PROVIDER_PLANES || nplanes > VXL_SPH_MAX_PROVIDER_PLANES)
    return set_error(VXL_INVALID_ARGUMENT, "at most 64 providers and 64 planes per scene");
  auto finite3 = [](const float* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); };
  for (uint32_t i = 0; i < n; ++i) {
    const vxl_sph_provider& p = pr[i];
    if (p.kind != VXL_SPH_PROVIDER_FACES && p.kind != VXL_SPH_PROVIDER_CONVEX)
      return set_error(VXL_INVALID_ARGUMENT, "unknown provider kind");
    if (p.first_plane > nplanes || p.nplanes > nplanes - p.first_plane)
      return set_error(VXL_INVALID_ARGUMENT, "provider planes out of range");
    if (p.has_bounds > 1u || (p.has_bounds && (!finite3(p.bounds_min) || !finite3(p.bounds_max))))
      return set_error(VXL_INVALID_ARGUMENT, "provider bounds must be finite");
    for (uint32_t k = p.first_plane; k < p.first_plane + p.nplanes; ++k) {
      const vxl_sph_wall_plane& w = planes[k];
      if (!std::isfinite(w.offset)) return set_error(VXL_INVALID_ARGUMENT, "plane offset must be finite");
      if (p.kind == VXL_SPH_PROVIDER_FACES && (w.axis > 2u || (w.sign != 1.0f && w.sign != -1.0f)))
        return set_error(VXL_INVALID_ARGUMENT, "a face needs axis 0..2 and sign +1 or -1");
      if (p.kind == VXL_SPH_PROVIDER_CONVEX && !finite3(w.normal))
        return set_error(VXL_INVALID_ARGUMENT, "plane normal must be finite");
    }
  }
  CU(cudaSetDevice(device_));
  prof_collect();
  if (prov_h_.size() < scenes_.size()) {
    prov_h_.resize(scenes_.size());
    wplanes_h_.resize(scenes_.size());
  }
  prov_h_[q].assign(pr, pr + n);
  wplanes_h_[q].assign(planes, planes + nplanes);
  return stage_walls();
}

// Upload every scene's providers and planes (global plane indices), size the per-substep
// buffers of the wall passes, and republish the scene records. Runs with the device idle.
vxl_status Engine::stage_walls() {
  CU(cudaStreamSynchronize(stream_));
  if (side_) CU(cudaStreamSynchronize(side_));
  if (react_) CU(cudaStreamSynchronize(react_));
  side_pending_ = react_pending_ = false;
  std::vector<ProviderDev> hp;
  std::vector<WallPlaneDev> hw;
  prov_first_st_.assign(scenes_.size(), 0u);
  prov_count_st_.assign(scenes_.size(), 0u);
  if (prov_h_.size() < scenes_.size()) {
    prov_h_.resize(scenes_.size());
    wplanes_h_.resize(scenes_.size());
  }
  for (uint32_t q = 0; q < scenes_.size(); ++q) {
    prov_first_st_[q] = (uint32_t)hp.size();
    prov_count_st_[q] = (uint32_t)prov_h_[q].size();
    const uint32_t wbase = (uint32_t)hw.size();
    for (const vxl_sph_wall_plane& w : wplanes_h_[q]) {
      WallPlaneDev d{};
      d.nx = w.normal[0];
      d.ny = w.normal[1];
      d.nz = w.normal[2];
      d.d = w.offset;
      d.axis = w.axis;
      d.sign = w.sign;
      hw.push_back(d);
    }
    for (const vxl_sph_provider& p : prov_h_[q]) {
      ProviderDev d{};
      d.kind = p.kind;
      d.first = wbase + p.first_plane;
      d.count = p.nplanes;
      d.has_bounds = p.has_bounds;
      d.bminx = p.bounds_min[0];
      d.bminy = p.bounds_min[1];
      d.bminz = p.bounds_min[2];
      d.bmaxx = p.bounds_max[0];
      d.bmaxy = p.bounds_max[1];
      d.bmaxz = p.bounds_max[2];
      hp.push_back(d);
    }
    if (scene_has_table(q)) {  // the contact tables come after the analytic providers
      ProviderDev d{};
      d.kind = kProviderTable;
      hp.push_back(d);
      ++prov_count_st_[q];
    }
  }
  walls_any_ = !hp.empty();
  if (hp.size() > prov_cap_) {
    if (prov_d_) cudaFree(prov_d_);
    prov_d_ = nullptr;
    prov_cap_ = 0;
    vxl_status s = dalloc(&prov_d_, hp.size());
    if (s != VXL_OK) return s;
    prov_cap_ = (uint32_t)hp.size();
  }
  if (hw.size() > wplanes_cap_) {
    if (wplanes_d_) cudaFree(wplanes_d_);
    wplanes_d_ = nullptr;
    wplanes_cap_ = 0;
    vxl_status s = dalloc(&wplanes_d_, hw.size());
    if (s != VXL_OK) return s;
    wplanes_cap_ = (uint32_t)hw.size();
  }
  if (!hp.empty()) CU(cudaMemcpy(prov_d_, hp.data(), hp.size() * sizeof(ProviderDev), cudaMemcpyHostToDevice));
  if (!hw.empty()) CU(cudaMemcpy(wplanes_d_, hw.data(), hw.size() * sizeof(WallPlaneDev), cudaMemcpyHostToDevice));
  if (walls_any_ && !pflag_) {
    vxl_status s = dalloc(&pflag_, slot_cap_);
    if (s == VXL_OK) s = dalloc((float4**)&pnsum_, slot_cap_);
    if (s == VXL_OK) s = dalloc(&plist_, slot_cap_);
    if (s == VXL_OK) s = dalloc(&pblk_, slot_cap_ / kPushedChunk + 2);
    if (s != VXL_OK) return s;
  }
  if (pflag_) CU(cudaMemset(pflag_, 0, slot_cap_ * sizeof(uint32_t)));
  {
    vxl_status s = upload_tables();
    if (s != VXL_OK) return s;
  }
  std::vector<float> dts(scenes_.size());
  for (uint32_t q = 0; q < scenes_.size(); ++q) dts[q] = sc_h_[q].dt;
  vxl_status s = push_scene_records(dts);
  if (s != VXL_OK) return s;
  if (graph_) {  // the tick's kernels and buffers changed
    cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
  }
  return VXL_OK;
}

vxl_status Engine::read_rigid_bodies(uint32_t q, vxl_sph_rigid_body* out, uint32_t n) {
  if (q >= scenes_.size()) return set_error(VXL_INVALID_ARGUMENT, "scene index out of range");
  if (q >= rigid_.size() || rigid_[q].empty()) return set_error(VXL_NOT_READY, "no rigid bodies in this scene");
  if (n != rigid_[q].size()) return set_error(VXL_SIZE_MISMATCH, "n differs from the scene's rigid bodies");
  if (!out) return set_error(VXL_NULL_POINTER, "out is NULL");
  CU(cudaSetDevice(device_));
  prof_collect();
  if (rb_live_ && rb_d_) {
    std::vector<RigidBodyDev> h(n);
    CU(cudaMemcpyAsync(h.data(), rb_d_ + rb_off_[q], n * sizeof(RigidBodyDev), cudaMemcpyDeviceToHost, stream_));
    CU(cudaStreamSynchronize(stream_));
    for (uint32_t b = 0; b < n; ++b) {
      out[b] = rigid_[q][b];
      from_dev(h[b], out[b]);
    }
  } else {
    for (uint32_t b = 0; b < n; ++b) out[b] = rigid_[q][b];
  }
  return VXL_OK;
}

vxl_status Engine::set_body_poses(uint32_t q, const vxl_sph_body_pose* poses, uint32_t nbodies) {
  if (q >= scenes_.size()) return set_error(VXL_INVALID_ARGUMENT, "scene index out of range");
  if (q >= scene_bodies_.size() || scene_bodies_[q] == 0)
    return set_error(VXL_NOT_READY, "no body lattice set for this scene");
  if (nbodies != scene_bodies_[q]) return set_error(VXL_SIZE_MISMATCH, "pose count differs from the lattice's bodies");
  if (!poses) return set_error(VXL_NULL_POINTER, "poses is NULL");
  const SceneInfo& si = scenes_[q];
  CU(cudaSetDevice(device_));
  prof_collect();
  CU(cudaStreamSynchronize(stream_));
  if (nbodies > poses_cap_) {
    if (poses_d_) cudaFree(poses_d_);
    poses_d_ = nullptr;
    poses_cap_ = 0;
    vxl_status st = dalloc(&poses_d_, nbodies);
    if (st != VXL_OK) return st;
    poses_cap_ = nbodies;
  }
  std::vector<BodyPoseDev> h(nbodies);
  for (uint32_t b = 0; b < nbodies; ++b) {
    const vxl_sph_body_pose& p = poses[b];
    h[b] = BodyPoseDev{p.pos[0], p.pos[1], p.pos[2], p.rot[0], p.rot[1], p.rot[2], p.rot[3],
                       p.linvel[0], p.linvel[1], p.linvel[2], p.angvel[0], p.angvel[1], p.angvel[2]};
  }
  static const uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
  CU(cudaMemcpyAsync(poses_d_, h.data(), nbodies * sizeof(BodyPoseDev), cudaMemcpyHostToDevice, stream_));
  CU(cudaMemcpyAsync(sc_d_[q].bbox, init, sizeof(init), cudaMemcpyHostToDevice, stream_));
  k_e_body_rebuild<<<blocks_for(si.nb), kThreads, 0, stream_>>>(blocal_, poses_d_, (float4*)pos_[0],
                                                                 (float4*)vel_[0], slot_of_, (float4*)bpos_,
                                                                 sc_d_[q].bbox, si.base, si.nf, si.nb);
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(stream_));  // the caller's poses are borrowed for this call only
  return VXL_OK;
}

vxl_status Engine::write_state(uint32_t q, const float* pos, const float* vel) {
  if (q >= scenes_.size()) return set_error(VXL_INVALID_ARGUMENT, "scene index out of range");
  const SceneInfo& si = scenes_[q];
  const uint32_t n = si.nf + si.nb;
  if (n == 0) return VXL_OK;
  CU(cudaSetDevice(device_));
  if (pos) CU(cudaMemcpyAsync(stage_, pos, (size_t)n * 12, cudaMemcpyHostToDevice, stream_));
  if (vel) CU(cudaMemcpyAsync(stage_ + 3 * (size_t)n, vel, (size_t)n * 12, cudaMemcpyHostToDevice, stream_));
  k_e_write_scene<<<blocks_for(n), kThreads, 0, stream_>>>(pos ? stage_ : nullptr, vel ? stage_ + 3 * (size_t)n : nullptr,
                                                            (float4*)pos_[0], (float4*)vel_[0], orig_, (float4*)bpos_,
                                                            si.base, n, si.nf);
  CU(cudaGetLastError());
  if (pos) return recompute_scene_boxes(q);  // synchronises
  CU(cudaStreamSynchronize(stream_));
  return VXL_OK;
}

vxl_status Engine::read_state(uint32_t q, float* pos, float* vel) {
  if (q >= scenes_.size()) return set_error(VXL_INVALID_ARGUMENT, "scene index out of range");
  const SceneInfo& si = scenes_[q];
  const uint32_t n = si.nf + si.nb;
  if (n == 0) return VXL_OK;
  CU(cudaSetDevice(device_));
  float* dp = stage_;
  float* dv = stage_ + 3 * (size_t)n;
  k_e_read_scene<<<blocks_for(n), kThreads, 0, stream_>>>((const float4*)pos_[0], (const float4*)vel_[0], orig_,
                                                           pos ? dp : nullptr, vel ? dv : nullptr, si.base, n);
  if (pos) CU(cudaMemcpyAsync(pos, dp, (size_t)n * 12, cudaMemcpyDeviceToHost, stream_));
  if (vel) CU(cudaMemcpyAsync(vel, dv, (size_t)n * 12, cudaMemcpyDeviceToHost, stream_));
  CU(cudaStreamSynchronize(stream_));
  return VXL_OK;
}

vxl_status Engine::request_state() {
  CU(cudaSetDevice(device_));
  const uint64_t n = used_;
  if (!ev_snap_) CU(cudaEventCreateWithFlags(&ev_snap_, cudaEventDisableTiming));
  if (!ev_snap_ready_) CU(cudaEventCreateWithFlags(&ev_snap_ready_, cudaEventDisableTiming));
  if (!snap_stream_) CU(cudaStreamCreateWithFlags(&snap_stream_, cudaStreamNonBlocking));
  if (snap_pending_) {  // a copy not yet taken still reads snap_d_ and writes snap_h_
    CU(cudaEventSynchronize(ev_snap_));
    snap_pending_ = false;
  }
  if (n > snap_cap_) {
    if (snap_h_) cudaFreeHost(snap_h_);
    if (snap_d_) cudaFree(snap_d_);
    snap_h_ = nullptr;
    snap_d_ = nullptr;
    snap_cap_ = 0;
    CU(cudaMallocHost((void**)&snap_h_, n * 12));
    if (cudaMalloc((void**)&snap_d_, n * 12) != cudaSuccess) {
      cudaGetLastError();
      return set_error(VXL_OUT_OF_MEMORY, "no device memory for the state copy");
    }
    snap_cap_ = n;
  }
  // the positions in reference order are gathered behind the enqueued work on the handle's
  // stream; the device-to-host copy then runs on a stream of its own, so the next tick's
  // kernels do not wait for it
  if (n) {
    k_e_read_scene<<<blocks_for(n), kThreads, 0, stream_>>>((const float4*)pos_[0], nullptr, orig_, snap_d_,
                                                             nullptr, 0u, (uint32_t)n);
    CU(cudaGetLastError());
  }
  CU(cudaEventRecord(ev_snap_ready_, stream_));
  CU(cudaStreamWaitEvent(snap_stream_, ev_snap_ready_, 0));
  if (n) CU(cudaMemcpyAsync(snap_h_, snap_d_, n * 12, cudaMemcpyDeviceToHost, snap_stream_));
  CU(cudaEventRecord(ev_snap_, snap_stream_));
  snap_n_ = n;
  snap_pending_ = true;
  return VXL_OK;
}

vxl_status Engine::take_state(float* pos, uint64_t n) {
  if (!snap_pending_) return set_error(VXL_NOT_READY, "no state requested");
  if (n != snap_n_) return set_error(VXL_SIZE_MISMATCH, "n differs from the particles of the requested state");
  if (n && !pos) return set_error(VXL_NULL_POINTER, "pos is NULL");
  CU(cudaSetDevice(device_));
  CU(cudaEventSynchronize(ev_snap_));
  // copy out in parallel chunks for large states (one thread moves ~10 GB/s)
  const size_t bytes = n * 12;
  const size_t nthr = bytes >= (64u << 20) ? std::min<size_t>(8, std::max<unsigned>(1, std::thread::hardware_concurrency())) : 1;
  const size_t chunk = ((bytes / nthr) + 63) & ~size_t(63);
  std::vector<std::thread> th;
  for (size_t t = 1; t < nthr && t * chunk < bytes; ++t)
    th.emplace_back([=] {
      std::memcpy((char*)pos + t * chunk, (const char*)snap_h_ + t * chunk, std::min(chunk, bytes - t * chunk));
    });
  std::memcpy(pos, snap_h_, std::min(chunk, bytes));
  for (auto& x : th) x.join();
  return VXL_OK;
}

vxl_status Engine::read_fields(uint32_t q, float* dens, float* press, float* acc, float* xsph, float* bforce) {
  if (q >= scenes_.size()) return set_error(VXL_INVALID_ARGUMENT, "scene index out of range");
  const SceneInfo& si = scenes_[q];
  const uint32_t n = si.nf + si.nb;
  if (n == 0) return VXL_OK;
  if ((acc || xsph) && !record_) return set_error(VXL_NOT_READY, "acc/xsph are recorded only with set_record(1)");
  CU(cudaSetDevice(device_));
  float* d_d = stage_;
  float* d_p = stage_ + (size_t)n;
  float* d_a = stage_ + 2 * (size_t)n;
  float* d_x = stage_ + 5 * (size_t)n;
  k_e_read_fields<<<blocks_for(n), kThreads, 0, stream_>>>((const float2*)rc_, press_, (const float4*)acc_,
                                                            (const float4*)xsph_, orig_, dens ? d_d : nullptr,
                                                            press ? d_p : nullptr, acc ? d_a : nullptr,
                                                            xsph ? d_x : nullptr, si.base, n);
  if (dens) CU(cudaMemcpyAsync(dens, d_d, (size_t)n * 4, cudaMemcpyDeviceToHost, stream_));
  if (press) CU(cudaMemcpyAsync(press, d_p, (size_t)n * 4, cudaMemcpyDeviceToHost, stream_));
  if (acc) CU(cudaMemcpyAsync(acc, d_a, (size_t)n * 12, cudaMemcpyDeviceToHost, stream_));
  if (xsph) CU(cudaMemcpyAsync(xsph, d_x, (size_t)n * 12, cudaMemcpyDeviceToHost, stream_));
  if (bforce && si.nb) {
    std::vector<float> tmp((size_t)si.nb * 4);
    CU(cudaMemcpyAsync(tmp.data(), (float4*)bforce_ + si.base + si.nf, (size_t)si.nb * 16, cudaMemcpyDeviceToHost,
                       stream_));
    CU(cudaStreamSynchronize(stream_));
    for (uint32_t k = 0; k < si.nb; ++k)
      for (int a = 0; a < 3; ++a) bforce[3 * k + a] = tmp[4 * k + a];
  }
  CU(cudaStreamSynchronize(stream_));
  return VXL_OK;
}

vxl_status Engine::export_grid(uint32_t q, uint32_t* items, uint32_t* start, uint64_t start_cap, uint32_t* bins,
                               vxl_sph_grid_info* info) {
  if (q >= scenes_.size()) return set_error(VXL_INVALID_ARGUMENT, "scene index out of range");
  if (!ran_substep_) return set_error(VXL_NOT_READY, "no substep has run yet");
  const SceneInfo& si = scenes_[q];
  const uint32_t n = si.nf + si.nb;
  CU(cudaSetDevice(device_));
  SceneDev rec;
  CU(cudaMemcpyAsync(&rec, sc_d_ + q, sizeof(SceneDev), cudaMemcpyDeviceToHost, stream_));
  CU(cudaStreamSynchronize(stream_));
  const uint64_t total = rec.cells;
  if (info) {
    info->min[0] = rec.g.minx;
    info->min[1] = rec.g.miny;
    info->min[2] = rec.g.minz;
    info->inv = rec.g.inv;
    info->bin = rec.g.bin;
    info->dims[0] = rec.g.nx;
    info->dims[1] = rec.g.ny;
    info->dims[2] = rec.g.nz;
    info->total = total;
  }
  uint32_t* tmp = (uint32_t*)stage_;
  if (start) {
    if (start_cap < total + 1) return set_error(VXL_SIZE_MISMATCH, "start buffer smaller than cells + 1");
    // the scene's slice of the global table, rebased to scene-local slots on the host
    CU(cudaMemcpyAsync(start, start_ + rec.cell_off, (total + 1) * 4, cudaMemcpyDeviceToHost, stream_));
    CU(cudaStreamSynchronize(stream_));
    for (uint64_t c = 0; c <= total; ++c) start[c] -= rec.base;
  }
  if (items && n) {
    k_e_export_items<<<blocks_for(n), kThreads, 0, stream_>>>(orig_, si.base, n, tmp);
    CU(cudaMemcpyAsync(items, tmp, (size_t)n * 4, cudaMemcpyDeviceToHost, stream_));
    CU(cudaStreamSynchronize(stream_));
  }
  if (bins && n) {
    k_e_export_bins<<<blocks_for(std::max<uint64_t>(total, 1)), kThreads, 0, stream_>>>(start_, orig_, sc_d_, q, tmp);
    CU(cudaMemcpyAsync(bins, tmp, (size_t)n * 4, cudaMemcpyDeviceToHost, stream_));
    CU(cudaStreamSynchronize(stream_));
  }
  CU(cudaGetLastError());
  return VXL_OK;
}

vxl_status Engine::export_neighbors(uint32_t q, uint64_t* offsets, uint64_t offsets_len, uint32_t* entries,
                                    uint64_t entries_cap, uint64_t* total) {
  if (q >= scenes_.size()) return set_error(VXL_INVALID_ARGUMENT, "scene index out of range");
  if (!offsets) return set_error(VXL_NULL_POINTER, "offsets is NULL");
  if (!ran_substep_) return set_error(VXL_NOT_READY, "no substep has run yet");
  const SceneInfo& si = scenes_[q];
  const uint32_t n = si.nf + si.nb;
  if (offsets_len != (uint64_t)n + 1) return set_error(VXL_SIZE_MISMATCH, "offsets must hold n_total + 1 entries");
  CU(cudaSetDevice(device_));
  uint32_t* cnt = (uint32_t*)stage_;
  std::vector<uint32_t> counts(n);
  if (n) {
    k_e_export_nbr_counts<<<blocks_for(n), kThreads, 0, stream_>>>(nbr_n_, orig_, si.base, n, cnt);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(counts.data(), cnt, (size_t)n * 4, cudaMemcpyDeviceToHost, stream_));
    CU(cudaStreamSynchronize(stream_));
  }
  uint64_t acc = 0;
  for (uint32_t i = 0; i < n; ++i) {
    offsets[i] = acc;
    acc += counts[i];
  }
  offsets[n] = acc;
  if (total) *total = acc;
  if (!entries || acc == 0) return VXL_OK;
  if (entries_cap < acc) return set_error(VXL_SIZE_MISMATCH, "entries buffer smaller than the list total");
  unsigned long long* off_d = nullptr;
  uint32_t* ent_d = nullptr;
  cudaError_t ce = cudaMalloc(&off_d, ((size_t)n + 1) * 8);
  if (ce == cudaSuccess) ce = cudaMalloc(&ent_d, (size_t)acc * 4);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(off_d, offsets, ((size_t)n + 1) * 8, cudaMemcpyHostToDevice, stream_);
  if (ce == cudaSuccess) {
    k_e_export_nbr_entries<<<blocks_for(n), kThreads, 0, stream_>>>(
        (const float4*)pos_[1], start_, sc_d_, q, orig_, nbr_, nbr_n_, nbr_cap_, (uint32_t)slot_cap_, off_d, ent_d);
    ce = cudaGetLastError();
  }
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(entries, ent_d, (size_t)acc * 4, cudaMemcpyDeviceToHost, stream_);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(stream_);
  cudaFree(off_d);
  cudaFree(ent_d);
  if (ce != cudaSuccess) return set_error(VXL_CUDA_ERROR, std::string("neighbour export: ") + cudaGetErrorString(ce));
  return VXL_OK;
}

vxl_status Engine::bounds(uint32_t q, float lo[3], float hi[3]) {
  if (q >= scenes_.size()) return set_error(VXL_INVALID_ARGUMENT, "scene index out of range");
  CU(cudaSetDevice(device_));
  uint32_t box[6];
  CU(cudaMemcpyAsync(box, sc_d_[q].fbox, sizeof(box), cudaMemcpyDeviceToHost, stream_));
  CU(cudaStreamSynchronize(stream_));
  for (int a = 0; a < 3; ++a) {
    lo[a] = vxl_o2f_host(box[a]);
    hi[a] = vxl_o2f_host(box[3 + a]);
  }
  if (!(std::isfinite(lo[0]) && std::isfinite(hi[0]))) return set_error(VXL_NOT_READY, "no fluid bounds");
  return VXL_OK;
}

vxl_status Engine::set_spans(uint32_t q, const vxl_sph_span* spans, uint32_t n) {
  if (q >= scenes_.size()) return set_error(VXL_INVALID_ARGUMENT, "scene index out of range");
  if (n && !spans) return set_error(VXL_NULL_POINTER, "spans is NULL with nspans > 0");
  const SceneInfo& si = scenes_[q];
  std::vector<vxl_sph_span> v(spans, spans + n);
  for (uint32_t k = 0; k < n; ++k)
    if (v[k].start < si.nf || v[k].end < v[k].start || v[k].end > si.nf + si.nb)
      return set_error(VXL_INVALID_ARGUMENT, "span " + std::to_string(k) + " is outside the boundary segment");
  if (spans_local_.size() < scenes_.size()) spans_local_.resize(scenes_.size());
  const auto& old = spans_local_[q];
  bool same = old.size() == v.size() && (v.empty() || std::memcmp(old.data(), v.data(), v.size() * sizeof(vxl_sph_span)) == 0);
  if (!same) {
    spans_local_[q] = v;
    spans_dirty_ = true;
  }
  return VXL_OK;
}

// Global span and chunk tables (pinned mirrors, copied inside the tick graph).
vxl_status Engine::stage_spans() {
  if (!spans_dirty_) return VXL_OK;
  prof_collect();
  CU(cudaStreamSynchronize(stream_));
  std::vector<SpanDev> sp;
  std::vector<LongSpan> ch;
  span_scene_.clear();
  for (uint32_t q = 0; q < scenes_.size() && q < spans_local_.size(); ++q)
    for (const vxl_sph_span& s : spans_local_[q]) {
      const uint32_t gs = scenes_[q].base + s.start, ge = scenes_[q].base + s.end;
      const uint32_t idx = (uint32_t)sp.size();
      uint32_t rigid = ~0u;  // coupled rigid body of this span (same body id in the same scene)
      if (q < rigid_.size() && q < rb_off_.size())
        for (uint32_t b = 0; b < rigid_[q].size(); ++b)
          if (rigid_[q][b].pose.body == s.body) {
            rigid = rb_off_[q] + b;
            break;
          }
      sp.push_back(SpanDev{s.body, s.origin[0], s.origin[1], s.origin[2], gs, ge, rigid});
      span_scene_.push_back(q);
      if (ge - gs > kReactExactSpan) ch.push_back(LongSpan{idx, gs, ge, 0u});  // a block of its own
    }
  const uint32_t ns = (uint32_t)sp.size(), nc = (uint32_t)ch.size();
  if (!spans_h_ || ns > spans_cap_ || nc > longs_cap_) {
    void* d[] = {spans_d_, longs_d_, breact_d_};
    for (void* p : d)
      if (p) cudaFree(p);
    void* hp[] = {spans_h_, longs_h_, breact_h_};
    for (void* p : hp)
      if (p) cudaFreeHost(p);
    spans_d_ = nullptr; longs_d_ = nullptr; breact_d_ = nullptr;
    spans_h_ = nullptr; longs_h_ = nullptr; breact_h_ = nullptr;
    const uint32_t cap = std::max<uint32_t>(ns, 64), ccap = std::max<uint32_t>(nc, 256);
    vxl_status s;
    if ((s = dalloc(&spans_d_, cap)) != VXL_OK) return s;
    if ((s = dalloc(&longs_d_, ccap)) != VXL_OK) return s;
    if ((s = dalloc(&breact_d_, (size_t)cap * 6)) != VXL_OK) return s;
    CU(cudaMallocHost((void**)&spans_h_, cap * sizeof(SpanDev)));
    CU(cudaMallocHost((void**)&longs_h_, ccap * sizeof(LongSpan)));
    CU(cudaMallocHost((void**)&breact_h_, cap * 6 * sizeof(float)));
    spans_cap_ = cap;
    longs_cap_ = ccap;
  }
  if (ns) std::memcpy(spans_h_, sp.data(), ns * sizeof(SpanDev));
  if (nc) std::memcpy(longs_h_, ch.data(), nc * sizeof(LongSpan));
  nspans_ = ns;
  nlongs_ = nc;
  spans_dirty_ = false;
  rb_dirty_ = true;              // the bodies' span indices follow the staging
  rb_have_reaction_ = false;     // reactions are indexed by the old staging
  if (graph_) {
    cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
  }
  return VXL_OK;
}

// ---------------------------------------------------------------- profiling

void Engine::record_event(cudaEvent_t e, cudaStream_t st) {
  if (capturing_) cudaEventRecordWithFlags(e, st, cudaEventRecordExternal);
  else cudaEventRecord(e, st);
}

int Engine::prof_begin(int kid, cudaStream_t st) {
  if (!prof_) return -1;
  if (2 * prof_used_ + 2 > prof_ev_.size()) return -1;  // pre-created in set_profile
  const size_t i = prof_used_++;
  prof_kid_[i] = kid;
  record_event(prof_ev_[2 * i], st);
  return (int)i;
}

void Engine::prof_end(int i, cudaStream_t st) {
  if (i >= 0) record_event(prof_ev_[2 * i + 1], st);
}

void Engine::join_side_only() {
  if (side_pending_) {
    cudaStreamWaitEvent(stream_, ev_join_, 0);
    side_pending_ = false;
  }
}

void Engine::join_side() {
  join_side_only();
  if (react_pending_) {
    cudaStreamWaitEvent(stream_, ev_rjoin_, 0);
    react_pending_ = false;
  }
}

void Engine::prof_collect() {
  if (!prof_pending_) return;
  cudaStreamSynchronize(stream_);
  for (size_t i = 0; i < prof_used_; ++i) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, prof_ev_[2 * i], prof_ev_[2 * i + 1]) == cudaSuccess) {
      prof_ms_[prof_kid_[i]] += ms;
      prof_n_[prof_kid_[i]] += 1;
    } else {
      cudaGetLastError();
    }
  }
  prof_pending_ = false;
}

vxl_status Engine::set_profile(bool on) {
  CU(cudaSetDevice(device_));
  prof_collect();
  prof_ = on;
  uint32_t sub = 1;
  for (auto& s : scenes_) sub = std::max(sub, s.substeps);
  const size_t need = 2 * ((size_t)sub * (KID_COUNT + 2) + 8);
  while (prof_ && prof_ev_.size() < need) {
    cudaEvent_t e;
    CU(cudaEventCreate(&e));
    prof_ev_.push_back(e);
  }
  prof_kid_.resize(prof_ev_.size() / 2);
  for (int k = 0; k < KID_COUNT; ++k) {
    prof_ms_[k] = 0.0;
    prof_n_[k] = 0;
  }
  if (graph_) {
    cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
  }
  return VXL_OK;
}

vxl_status Engine::profile_read(uint32_t k, const char** name, double* ms, uint64_t* launches) {
  if (k >= (uint32_t)KID_COUNT) return set_error(VXL_INVALID_ARGUMENT, "kernel index past the table");
  CU(cudaSetDevice(device_));
  prof_collect();
  if (name) *name = kKernelNames[k];
  if (ms) *ms = prof_ms_[k];
  if (launches) *launches = prof_n_[k];
  return VXL_OK;
}

#define LAUNCH_ON(kid, stream, ...)   \
  do {                                \
    int pe_ = prof_begin(kid, stream);\
    __VA_ARGS__;                      \
    prof_end(pe_, stream);            \
    launches_counter_ += 1;           \
  } while (0)

#define LAUNCH(kid, ...)          \
  do {                            \
    int pe_ = prof_begin(kid, stream_); \
    __VA_ARGS__;                  \
    prof_end(pe_, stream_);       \
    launches_counter_ += 1;       \
  } while (0)

// ---------------------------------------------------------------- stepping

void Engine::enqueue_substep(bool with_reactions) {
  cudaStream_t st = stream_;
  const uint32_t S = (uint32_t)scenes_.size();
  const uint32_t key_blocks = std::min<uint32_t>(std::max<uint32_t>(ntiles_, 1), 148 * 8);
  uint64_t nb_total = 0;
  for (auto& s : scenes_) nb_total += s.nb;
  const float4* p0 = (const float4*)pos_[0];
  const float4* v0 = (const float4*)vel_[0];
  const float4* p1 = (const float4*)pos_[1];
  const float4* v1 = (const float4*)vel_[1];
  // The previous substep's boundary-force pass reads this substep's inputs-to-be (scene
  // grids, cell table, sorted buffer, permutation, lists, work counters): join it first.
  // Its reaction sums read only bforce / bpos and go on beside this substep.
  join_side_only();
  LAUNCH(KID_CELLOFF, k_e_celloff<<<1, 1024, 0, st>>>(sc_d_, S, ctl_d_, (uint32_t)cell_cap_));
  LAUNCH(KID_KEYS, k_e_keys<<<key_blocks, kThreads, 0, st>>>(p0, sc_d_, tiles_d_, ntiles_, ctl_d_, counts_,
                                                             (uint2*)cellrank_, halves_,
                                                             (uint32_t)(4 * (used_ / 32 + 1)), wet_));
  LAUNCH(KID_SCAN_PARTIAL, k_e_scan_partial<<<148 * 4, kScanThreads, 0, st>>>(counts_, ctl_d_, partial_, start_));
  LAUNCH(KID_SCAN_FINAL, k_e_scan_final<<<148 * 4, kScanThreads, 0, st>>>(counts_, ctl_d_, partial_, start_));
  LAUNCH(KID_PLACE, k_e_place<<<key_blocks, kThreads, 0, st>>>((const uint2*)cellrank_, start_, orig_, tiles_d_,
                                                               ntiles_, ctl_d_, (uint2*)items_));
  LAUNCH(KID_CANON, k_e_canon<<<148 * 8, 256, 0, st>>>((const uint2*)items_, start_, ctl_d_, p0, v0, (float4*)pos_[1],
                                                       (float4*)vel_[1], orig_, slot_of_));
  // half-cell masks and the thread order of the density pass: for the provider-wall variant
  // the masks, then x halves first per cell; otherwise the masks with the octant-major order
  // per chunk of a tile (and the segments of the grouped kernel) in one pass
  if (walls_any_) {
    LAUNCH(KID_HALFMASK, k_e_halfmask<<<key_blocks, kThreads, 0, st>>>(p1, sc_d_, tiles_d_, ntiles_, ctl_d_, halves_));
    LAUNCH(KID_HALFMASK, k_e_xorder<<<148 * 8, kThreads, 0, st>>>(start_, ctl_d_, halves_, xorder_));
  } else {
    LAUNCH(KID_GROUPS, k_e_groups<<<key_blocks, kGroupChunk, 0, st>>>(p1, sc_d_, tiles_d_, ntiles_, ctl_d_, order_,
                                                                      (uint2*)segs_, halves_));
  }
  const uint32_t stride = (uint32_t)slot_cap_;
  const uint32_t* walk_order = order_;
  const bool rec = record_;
  const uint32_t per_tile = std::max<uint32_t>(ntiles_, 1);
  const uint32_t gd = grid_density_ ? (uint32_t)grid_density_ : per_tile;
  const uint32_t gf = grid_force_ ? (uint32_t)grid_force_ : per_tile;
  const uint32_t gb = grid_bforce_ ? (uint32_t)grid_bforce_ : std::max<uint32_t>(nbtiles_, 1);
  if (walls_any_) {  // provider walls: the variant with mirror ghosts
    if (tuning_.block == 128)
      LAUNCH(KID_DENSITY, k_e_density<128, true><<<gd, 128, 0, st>>>(
                              p1, start_, sc_d_, tiles_d_, ntiles_, ctl_d_, halves_, (float2*)rc_, press_, nbr_, nbr_n_,
                              nbr_cap_, stride, wet_, xorder_, prov_d_, wplanes_d_, orig_, ctab(0)));
    else
      LAUNCH(KID_DENSITY, k_e_density<256, true><<<gd, 256, 0, st>>>(
                              p1, start_, sc_d_, tiles_d_, ntiles_, ctl_d_, halves_, (float2*)rc_, press_, nbr_, nbr_n_,
                              nbr_cap_, stride, wet_, xorder_, prov_d_, wplanes_d_, orig_, ctab(0)));
  } else if (tuning_.density == 1) {
    LAUNCH(KID_DENSITY, k_e_density_seg<kSegWarps><<<grid_seg_, kSegWarps * 32, 0, st>>>(
                            p1, start_, sc_d_, ctl_d_, halves_, order_, (const uint2*)segs_, (float2*)rc_, press_, nbr_,
                            nbr_n_, nbr_cap_, stride, wet_));
  } else if (tuning_.block == 128) {
    LAUNCH(KID_DENSITY, k_e_density<128><<<gd, 128, 0, st>>>(p1, start_, sc_d_, tiles_d_, ntiles_, ctl_d_, halves_,
                                                             (float2*)rc_, press_, nbr_, nbr_n_, nbr_cap_, stride, wet_,
                                                             walk_order));
  } else {
    LAUNCH(KID_DENSITY, k_e_density<256><<<gd, 256, 0, st>>>(p1, start_, sc_d_, tiles_d_, ntiles_, ctl_d_, halves_,
                                                             (float2*)rc_, press_, nbr_, nbr_n_, nbr_cap_, stride, wet_,
                                                             walk_order));
  }
  // Reaction branch on the side stream: it reads only the sorted buffer, the densities and
  // the lists, so it runs beside the force pass (which writes the other buffer).
  const bool bforce = nb_total > 0 && ((with_reactions && nspans_ > 0) || rec);
  const bool react = with_reactions && nspans_ > 0;
  if (bforce || react) {
    cudaEventRecord(ev_fork_, st);
    cudaStreamWaitEvent(side_, ev_fork_, 0);
    if (react_pending_) {  // the previous substep's sums still read bforce
      cudaStreamWaitEvent(side_, ev_rjoin_, 0);
      react_pending_ = false;
    }
    if (bforce)
      LAUNCH_ON(KID_BFORCE, side_,
                k_e_bforce<<<gb, 128, 0, side_>>>(p1, v1, (const float2*)rc_, start_, orig_, nbr_, nbr_n_, nbr_cap_,
                                                  stride, sc_d_, slot_of_, tiles_d_ + ntiles_, nbtiles_, ctl_d_,
                                                  (float4*)bforce_));
    cudaEventRecord(ev_join_, side_);
    side_pending_ = true;
    if (react) {
      cudaEventRecord(ev_rfork_, side_);
      cudaStreamWaitEvent(react_, ev_rfork_, 0);
      if (nlongs_)  // the long spans (tank walls), a block each
        LAUNCH_ON(KID_REACT_LONG, react_,
                  k_react_long<<<nlongs_, kReactThreads, 0, react_>>>((const float4*)bforce_, (const float4*)bpos_,
                                                                       spans_d_, longs_d_, rb_d_, ctl_d_, breact_d_));
      LAUNCH_ON(KID_REACT_SPANS, react_,
                k_react_spans<<<(nspans_ + kReactSpanWarps - 1) / kReactSpanWarps, 32 * kReactSpanWarps, 0, react_>>>(
                    (const float4*)bforce_, (const float4*)bpos_, spans_d_, rb_d_, ctl_d_, breact_d_, nspans_));
      cudaEventRecord(ev_rjoin_, react_);
      react_pending_ = true;
    }
  }
  if (tuning_.block == 128)
    LAUNCH(KID_FORCE, k_e_force<128><<<gf, 128, 0, st>>>(
                          p1, v1, (const float2*)rc_, start_, nbr_, nbr_n_, nbr_cap_, stride, sc_d_, tiles_d_,
                          ntiles_, ctl_d_, (float4*)pos_[0], (float4*)vel_[0], rec ? (float4*)acc_ : nullptr,
                          rec ? (float4*)xsph_ : nullptr));
  else
    LAUNCH(KID_FORCE, k_e_force<256><<<gf, 256, 0, st>>>(
                          p1, v1, (const float2*)rc_, start_, nbr_, nbr_n_, nbr_cap_, stride, sc_d_, tiles_d_,
                          ntiles_, ctl_d_, (float4*)pos_[0], (float4*)vel_[0], rec ? (float4*)acc_ : nullptr,
                          rec ? (float4*)xsph_ : nullptr));
  if (walls_any_) {
    // boundary_pass of the scenes with providers, on the integrated state (pos_[0], vel_[0],
    // same slot order as the sorted buffer, so orig_ / slot_of_ apply)
    const uint32_t nref = (uint32_t)used_;
    const uint32_t nblk = std::max<uint32_t>((nref + kPushedChunk - 1) / kPushedChunk, 1);
    LAUNCH(KID_WALLS, k_e_wall_project<<<key_blocks, kThreads, 0, st>>>(
                          (float4*)pos_[0], (float4*)vel_[0], sc_d_, tiles_d_, ntiles_, ctl_d_, prov_d_, wplanes_d_,
                          orig_, pflag_, (float4*)pnsum_, ctab(1)));
    LAUNCH(KID_WALLS, k_e_pushed_count<<<nblk, kThreads, 0, st>>>(pflag_, nref, ctl_d_, pblk_));
    LAUNCH(KID_WALLS, k_e_pushed_emit<<<nblk, kThreads, 0, st>>>(pflag_, nref, pblk_, ctl_d_, plist_));
    LAUNCH(KID_WALLS, k_e_separate_check<<<148 * 2, kThreads, 0, st>>>((const float4*)pos_[0], sc_d_, plist_,
                                                                          (const float4*)pnsum_, slot_of_, ctl_d_));
    LAUNCH(KID_WALLS, k_e_separate<<<1, 1024, 0, st>>>((float4*)pos_[0], sc_d_, S, plist_, (const float4*)pnsum_,
                                                         slot_of_, ctl_d_));
    LAUNCH(KID_WALLS, k_e_wall_rebox<<<key_blocks, kThreads, 0, st>>>((const float4*)pos_[0], sc_d_, tiles_d_,
                                                                        ntiles_, ctl_d_));
  }
}

void Engine::enqueue_tick(float /*dt_tick*/) {
  cudaStream_t st = stream_;
  const uint32_t sub = scenes_.empty() ? 1 : scenes_[0].substeps;
  if (nspans_ > 0) {
    cudaMemcpyAsync(spans_d_, spans_h_, nspans_ * sizeof(SpanDev), cudaMemcpyHostToDevice, st);
    if (nlongs_) cudaMemcpyAsync(longs_d_, longs_h_, nlongs_ * sizeof(LongSpan), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(breact_d_, 0, nspans_ * 6 * sizeof(float), st);
  }
  for (uint32_t s = 0; s < sub; ++s) enqueue_substep(true);
  join_side();
  if (nspans_ > 0) {
    if (sub > 1) {
      const float inv = 1.0f / (float)sub;  // fluid_step.rs:85
      LAUNCH(KID_SCALE, k_scale<<<blocks_for(nspans_ * 6), kThreads, 0, st>>>(breact_d_, nspans_ * 6, inv));
    }
    cudaMemcpyAsync(breact_h_, breact_d_, nspans_ * 6 * sizeof(float), cudaMemcpyDeviceToHost, st);
  }
  cudaMemcpyAsync(ctl_h_, ctl_d_, sizeof(EngineCtl), cudaMemcpyDeviceToHost, st);
}

vxl_status Engine::step_tick_async(float dt_tick) {
  if (!(dt_tick > 0.0f) || !std::isfinite(dt_tick)) return set_error(VXL_INVALID_ARGUMENT, "dt_tick must be > 0");
  CU(cudaSetDevice(device_));
  if (scenes_.empty()) return VXL_OK;
  const uint32_t sub = scenes_[0].substeps;
  bool any_fluid = false;
  for (auto& s : scenes_) {
    if (s.substeps != sub) return set_error(VXL_INVALID_ARGUMENT, "scenes of one tick must share substeps");
    any_fluid = any_fluid || s.nf > 0;
  }
  if (!any_fluid) return VXL_OK;  // fluid_step.rs:93-95: boundary particles are not driven alone
  // per-scene substep dt = dt_tick / substeps (fluid_step.rs:77)
  const float dt = dt_tick / (float)sub;
  bool push = false;
  for (uint32_t q = 0; q < scenes_.size(); ++q)
    if (sc_h_[q].dt != dt) push = true;
  prof_collect();
  if (push) {
    CU(cudaStreamSynchronize(stream_));
    vxl_status s = push_scene_records(std::vector<float>(scenes_.size(), dt));
    if (s != VXL_OK) return s;
  }
  vxl_status s = stage_spans();
  if (s != VXL_OK) return s;
  const uint32_t key = (record_ ? 1u : 0u) | (prof_ ? 2u : 0u) | (walls_any_ ? 4u : 0u) | (sub << 3);
  launches_counter_ = 0;
  if (!use_graph_) {
    prof_used_ = 0;
    enqueue_tick(dt_tick);
    prof_pending_ = prof_;
    launches_last_tick_ = launches_counter_;
    CU(cudaGetLastError());
    ran_substep_ = true;
    return VXL_OK;
  }
  if (!graph_ || graph_key_ != key || graph_epoch_ != membership_epoch_) {
    if (graph_) {
      cudaGraphExecDestroy(graph_);
      graph_ = nullptr;
    }
    cudaGraph_t g = nullptr;
    prof_used_ = 0;
    CU(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    capturing_ = true;
    enqueue_tick(dt_tick);
    capturing_ = false;
    CU(cudaStreamEndCapture(stream_, &g));
    cudaError_t e = cudaGraphInstantiate(&graph_, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return set_error(VXL_CUDA_ERROR, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    graph_key_ = key;
    graph_epoch_ = membership_epoch_;
    launches_last_tick_ = launches_counter_;
  }
  CU(cudaGraphLaunch(graph_, stream_));
  prof_pending_ = prof_;
  ran_substep_ = true;
  return VXL_OK;
}

vxl_status Engine::finish() {
  CU(cudaStreamSynchronize(stream_));
  prof_collect();
  if (ctl_h_->err & kErrGridLoop) return set_error(VXL_DEVICE_FAULT_FLAG, "grid box doubling loop did not settle");
  if (ctl_h_->err & kErrCellCap) {
    ctl_h_->err = 0;
    cudaMemsetAsync(&ctl_d_->err, 0, 4, stream_);
    // the skipped substeps left the state as it was but emptied the fluid AABB
    // accumulators (reset by the grid-box pass): rebuild them from the state
    for (uint32_t q = 0; q < scenes_.size(); ++q) {
      vxl_status s = recompute_scene_boxes(q);
      if (s != VXL_OK) return s;
    }
    cudaStreamSynchronize(stream_);
    return set_error(VXL_DEVICE_FAULT_FLAG,
                     "the scenes' cells exceed the engine's cell capacity; the tick was skipped, state unchanged");
  }
  return VXL_OK;
}

vxl_status Engine::sync(std::vector<vxl_sph_reaction>* out) {
  CU(cudaSetDevice(device_));
  vxl_status s = finish();
  if (s != VXL_OK) return s;
  if (out) {
    out->resize(nspans_);
    for (uint32_t q = 0; q < nspans_; ++q) {
      (*out)[q].body = spans_h_[q].body;
      for (int a = 0; a < 3; ++a) {
        (*out)[q].force[a] = breact_h_[6 * q + a];
        (*out)[q].torque[a] = breact_h_[6 * q + 3 + a];
      }
    }
  }
  return VXL_OK;
}

vxl_status Engine::substep(const std::vector<float>& dt) {
  CU(cudaSetDevice(device_));
  if (scenes_.empty()) return VXL_OK;
  if (dt.size() != scenes_.size()) return set_error(VXL_SIZE_MISMATCH, "one dt per scene");
  bool any_fluid = false;
  for (auto& s : scenes_) any_fluid = any_fluid || s.nf > 0;
  if (!any_fluid) return VXL_OK;
  prof_collect();
  bool push = false;
  for (uint32_t q = 0; q < scenes_.size(); ++q)
    if (sc_h_[q].dt != dt[q]) push = true;
  if (push) {
    CU(cudaStreamSynchronize(stream_));
    vxl_status s = push_scene_records(dt);
    if (s != VXL_OK) return s;
  }
  prof_used_ = 0;
  launches_counter_ = 0;
  enqueue_substep(false);
  join_side();
  cudaMemcpyAsync(ctl_h_, ctl_d_, sizeof(EngineCtl), cudaMemcpyDeviceToHost, stream_);
  prof_pending_ = prof_;
  launches_last_tick_ = launches_counter_;
  CU(cudaGetLastError());
  ran_substep_ = true;
  return finish();
}

vxl_status Engine::autotune(float dt_tick, uint32_t trials, Tuning* best, float* best_ms) {
  if (!(dt_tick > 0.0f)) return set_error(VXL_INVALID_ARGUMENT, "dt_tick must be > 0");
  CU(cudaSetDevice(device_));
  if (scenes_.empty() || used_ == 0) return set_error(VXL_NOT_READY, "no scene to tune on");
  prof_collect();
  CU(cudaStreamSynchronize(stream_));
  const bool prof_was = prof_;
  prof_ = false;
  const uint32_t S = (uint32_t)scenes_.size();
  std::vector<float> dt(S);
  for (uint32_t q = 0; q < S; ++q) dt[q] = dt_tick / (float)scenes_[q].substeps;
  vxl_status st = push_scene_records(dt);
  if (st != VXL_OK) return st;
  // snapshot of the state the trials start from
  const size_t n = used_;
  void* snap = nullptr;
  const size_t bytes = n * (16 + 16 + 4 + 16) + S * sizeof(SceneDev);
  if (cudaMalloc(&snap, bytes) != cudaSuccess) {
    cudaGetLastError();
    return set_error(VXL_OUT_OF_MEMORY, "autotune snapshot");
  }
  char* sp = (char*)snap;
  float4* s_pos = (float4*)sp;
  float4* s_vel = (float4*)(sp + n * 16);
  float4* s_bpos = (float4*)(sp + n * 32);
  uint32_t* s_orig = (uint32_t*)(sp + n * 48);
  SceneDev* s_sc = (SceneDev*)(sp + n * 52);
  auto copy_all = [&](bool save) -> vxl_status {
    cudaMemcpyKind k = cudaMemcpyDeviceToDevice;
    CU(cudaMemcpyAsync(save ? (void*)s_pos : pos_[0], save ? pos_[0] : (void*)s_pos, n * 16, k, stream_));
    CU(cudaMemcpyAsync(save ? (void*)s_vel : vel_[0], save ? vel_[0] : (void*)s_vel, n * 16, k, stream_));
    CU(cudaMemcpyAsync(save ? (void*)s_bpos : bpos_, save ? bpos_ : (void*)s_bpos, n * 16, k, stream_));
    CU(cudaMemcpyAsync(save ? (void*)s_orig : (void*)orig_, save ? (void*)orig_ : (void*)s_orig, n * 4, k, stream_));
    CU(cudaMemcpyAsync(save ? (void*)s_sc : (void*)sc_d_, save ? (void*)sc_d_ : (void*)s_sc, S * sizeof(SceneDev), k,
                       stream_));
    if (!save) k_e_slot_of<<<blocks_for(n), kThreads, 0, stream_>>>(orig_, slot_of_, (uint32_t)n);
    CU(cudaStreamSynchronize(stream_));
    return VXL_OK;
  };
  st = copy_all(true);
  const Tuning was = tuning_;
  Tuning best_t = was;
  float best_v = 1e30f;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // candidates: block {128, 256} x tile {1, 2, 4} blocks x (one block per tile, or
  // persistent at 1 or 2 x the occupancy limit)
  const uint32_t blocks[2] = {128, 256};
  const uint32_t tile_mult[3] = {1, 2, 4};
  const uint32_t waves_c[3] = {0, 1, 2};
  for (uint32_t bi = 0; st == VXL_OK && bi < 2; ++bi)
    for (uint32_t ti = 0; st == VXL_OK && ti < 3; ++ti)
      for (uint32_t wi = 0; st == VXL_OK && wi < 3; ++wi) {
        st = copy_all(false);
        if (st != VXL_OK) break;
        set_tuning(Tuning{blocks[bi], blocks[bi] * tile_mult[ti], waves_c[wi], was.density});
        enqueue_substep(false);  // warm-up
        cudaEventRecord(e0, stream_);
        for (uint32_t r = 0; r < trials; ++r) enqueue_substep(false);
        join_side();
        cudaEventRecord(e1, stream_);
        if (cudaStreamSynchronize(stream_) != cudaSuccess) {
          st = set_error(VXL_CUDA_ERROR, "autotune trial failed");
          break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms /= (float)trials;
        if (ms < best_v) {
          best_v = ms;
          best_t = tuning_;
        }
      }
  // the other density kernels at the best shape (provider-wall scenes use their own variant)
  for (uint32_t dv = 0; st == VXL_OK && !walls_any_ && dv < 2; ++dv) {
    if (dv == best_t.density) continue;
    Tuning other = best_t;
    other.density = dv;
    st = copy_all(false);
    if (st != VXL_OK) break;
    set_tuning(other);
    enqueue_substep(false);
    cudaEventRecord(e0, stream_);
    for (uint32_t r = 0; r < trials; ++r) enqueue_substep(false);
    join_side();
    cudaEventRecord(e1, stream_);
    if (cudaStreamSynchronize(stream_) != cudaSuccess) {
      st = set_error(VXL_CUDA_ERROR, "autotune trial failed");
      break;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= (float)trials;
    if (ms < best_v) {
      best_v = ms;
      best_t = tuning_;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st == VXL_OK) st = copy_all(false);
  set_tuning(st == VXL_OK ? best_t : was);
  cudaFree(snap);
  prof_ = prof_was;
  if (st != VXL_OK) return st;
  CU(cudaMemcpyAsync(ctl_h_, ctl_d_, sizeof(EngineCtl), cudaMemcpyDeviceToHost, stream_));
  st = finish();
  if (st != VXL_OK) return st;
  if (best) *best = best_t;
  if (best_ms) *best_ms = best_v;
  return VXL_OK;
}

uint32_t Engine::cells_last() {
  EngineCtl c;
  cudaMemcpyAsync(&c, ctl_d_, sizeof(EngineCtl), cudaMemcpyDeviceToHost, stream_);
  cudaStreamSynchronize(stream_);
  return c.cells;
}

uint32_t Engine::slow_gathers() {
  EngineCtl c;
  cudaMemcpyAsync(&c, ctl_d_, sizeof(EngineCtl), cudaMemcpyDeviceToHost, stream_);
  cudaStreamSynchronize(stream_);
  return c.slow_gathers;
}

}  // namespace vxl
