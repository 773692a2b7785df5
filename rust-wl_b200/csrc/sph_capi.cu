// C ABI of the WCSPH step (include/vxl_sph.h): the plain drop-in handle and its batched
// multi-scene form. A handle is an Engine (sph_engine.h); the plain form is an engine
// holding one scene.
//
// Reference seam: FluidStepper (crates/vxl-phys-core/src/interop.rs:293-316) as
// implemented by GpuFluidStepper (crates/vxl-phys-gpu/src/pipeline/stepper.rs:22-147).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "sph_engine.h"
#include "vxl_sph.h"
#include "vxl_sph_internal.h"

using vxl::Engine;
using vxl::set_error;

struct vxl_sph_handle {
  Engine* e = nullptr;
  std::vector<vxl_sph_reaction> last;  // reactions of the last synced tick
  uint32_t last_nspans = 0;            // spans of scene 0 in the last enqueued tick
};

namespace {

bool check_header(const vxl_block_header& hd, uint32_t size) {
  return hd.size == size && hd.version == VXL_SPH_ABI_VERSION;
}

vxl_status check_desc(const vxl_sph_desc* d) {
  if (!d) return set_error(VXL_NULL_POINTER, "desc is NULL");
  if (d->hdr.version != VXL_SPH_ABI_VERSION || d->params.hdr.version != VXL_SPH_ABI_VERSION)
    return set_error(VXL_VERSION_MISMATCH, "ABI version mismatch");
  if (!check_header(d->hdr, sizeof(vxl_sph_desc)) || !check_header(d->params.hdr, sizeof(vxl_sph_params)))
    return set_error(VXL_SIZE_MISMATCH, "struct size mismatch");
  if (d->n_fluid + d->n_boundary >= (1ull << 31)) return set_error(VXL_INVALID_ARGUMENT, "more than 2^31 particles");
  const uint32_t mb = d->params.max_bins ? d->params.max_bins : (1u << 21);
  if (mb > (1u << 21)) return set_error(VXL_INVALID_ARGUMENT, "max_bins above 2^21");
  if (!(d->params.particle_mass > 0.0f) || !(d->params.rest_density > 0.0f) || !(d->params.gamma_tait > 0.0f))
    return set_error(VXL_INVALID_ARGUMENT, "particle_mass, rest_density and gamma_tait must be positive");
  return VXL_OK;
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

#define HANDLE_OR_FAIL(h)                                                     \
  if (!(h) || !(h)->e) return set_error(VXL_NULL_POINTER, "handle is NULL"); \
  DeviceGuard dg_((h)->e->device())

vxl_status make_engine(const vxl_sph_desc* descs, uint32_t n, int32_t device, uint64_t cell_capacity,
                       vxl_sph_handle** out) {
  if (!out) return set_error(VXL_NULL_POINTER, "out is NULL");
  *out = nullptr;
  if (!descs || n == 0) return set_error(VXL_NULL_POINTER, "no scene descriptions");
  uint64_t slots = 0, cells = 0;
  for (uint32_t i = 0; i < n; ++i) {
    vxl_status s = check_desc(descs + i);
    if (s != VXL_OK) return s;
    slots += descs[i].n_fluid + descs[i].n_boundary;
    cells += (uint64_t)(descs[i].params.max_bins ? descs[i].params.max_bins : (1u << 21));
  }
  if (cell_capacity == 0) cell_capacity = std::min<uint64_t>(cells, 1ull << 28);
  Engine* e = nullptr;
  vxl_status s = Engine::create(device, slots, cell_capacity, n, &e);
  if (s != VXL_OK) return s;
  for (uint32_t i = 0; i < n; ++i) {
    const vxl_sph_desc& d = descs[i];
    s = e->add_scene(d.params, d.n_fluid, d.n_boundary, d.pos_xyz, d.vel_xyz, d.pmass, i, nullptr);
    if (s != VXL_OK) {
      delete e;
      return s;
    }
  }
  auto* h = new (std::nothrow) vxl_sph_handle();
  if (!h) {
    delete e;
    return set_error(VXL_OUT_OF_MEMORY, "host allocation failed");
  }
  h->e = e;
  *out = h;
  return VXL_OK;
}

}  // namespace

extern "C" {

uint32_t vxl_sph_abi_version(void) { return VXL_SPH_ABI_VERSION; }

const char* vxl_sph_last_error(void) { return vxl_get_last_error(); }

const char* vxl_sph_backend_name(void) { return "b200-cuda-wcsph"; }

int vxl_sph_backend_available(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return 0;
  }
  for (int d = 0; d < n; ++d) {
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, d) == cudaSuccess && p.major == 10) return 1;
  }
  return 0;
}

vxl_status vxl_sph_create(const vxl_sph_desc* desc, vxl_sph_handle** out) {
  try {
    if (!desc || !out) return set_error(VXL_NULL_POINTER, "desc or out is NULL");
    vxl_status s = check_desc(desc);
    if (s != VXL_OK) return s;
    const uint64_t mb = desc->params.max_bins ? desc->params.max_bins : (1u << 21);
    return make_engine(desc, 1, desc->device, mb, out);
  } catch (...) {
    return set_error(VXL_PANIC_CAUGHT, "exception in vxl_sph_create");
  }
}

vxl_status vxl_sph_create_batch(const vxl_sph_desc* descs, uint32_t n, int32_t device, uint64_t cell_capacity,
                                vxl_sph_handle** out) {
  try {
    return make_engine(descs, n, device, cell_capacity, out);
  } catch (...) {
    return set_error(VXL_PANIC_CAUGHT, "exception in vxl_sph_create_batch");
  }
}

vxl_status vxl_sph_destroy(vxl_sph_handle* h) {
  if (!h) return set_error(VXL_NULL_POINTER, "handle is NULL");
  delete h->e;
  delete h;
  return VXL_OK;
}

uint32_t vxl_sph_scene_count(vxl_sph_handle* h) { return (h && h->e) ? (uint32_t)h->e->scenes().size() : 0u; }

vxl_status vxl_sph_upload_boundary(vxl_sph_handle* h, uint64_t n_fluid, const float* pos_xyz, const float* vel_xyz,
                                   uint64_t nb) {
  HANDLE_OR_FAIL(h);
  if (h->e->scenes().empty()) return set_error(VXL_NOT_READY, "no scene");
  if (n_fluid != h->e->scenes()[0].nf)
    return set_error(VXL_SIZE_MISMATCH, "fluid prefix differs from the scene (rebuild the scene)");
  return h->e->upload_boundary(0, pos_xyz, vel_xyz, nb);
}

vxl_status vxl_sph_upload_boundary_scene(vxl_sph_handle* h, uint32_t scene, const float* pos_xyz,
                                         const float* vel_xyz, uint64_t nb) {
  HANDLE_OR_FAIL(h);
  return h->e->upload_boundary(scene, pos_xyz, vel_xyz, nb);
}

vxl_status vxl_sph_request_state(vxl_sph_handle* h) {
  HANDLE_OR_FAIL(h);
  try {
    return h->e->request_state();
  } catch (...) {
    return set_error(VXL_PANIC_CAUGHT, "exception in vxl_sph_request_state");
  }
}

vxl_status vxl_sph_take_state(vxl_sph_handle* h, float* pos_xyz, uint64_t n) {
  HANDLE_OR_FAIL(h);
  try {
    return h->e->take_state(pos_xyz, n);
  } catch (...) {
    return set_error(VXL_PANIC_CAUGHT, "exception in vxl_sph_take_state");
  }
}

vxl_status vxl_sph_set_rigid_bodies(vxl_sph_handle* h, uint32_t scene, const vxl_sph_rigid_body* bodies,
                                    uint32_t n) {
  HANDLE_OR_FAIL(h);
  try {
    return h->e->set_rigid_bodies(scene, bodies, n);
  } catch (...) {
    return set_error(VXL_PANIC_CAUGHT, "exception in vxl_sph_set_rigid_bodies");
  }
}

vxl_status vxl_sph_step_coupled(vxl_sph_handle* h, float dt_tick, uint32_t rigid_substeps, const float gravity[3],
                                float max_linear, float max_angular, vxl_sph_reaction* out_reactions,
                                uint32_t nspans) {
  HANDLE_OR_FAIL(h);
  if (nspans > 0 && !out_reactions) return set_error(VXL_NULL_POINTER, "out_reactions is NULL with nspans > 0");
  try {
    vxl_status s = h->e->step_coupled_async(dt_tick, rigid_substeps, gravity, max_linear, max_angular);
    if (s != VXL_OK) return s;
    s = h->e->sync(&h->last);
    if (s != VXL_OK) return s;
    if (nspans > h->last.size()) return set_error(VXL_SIZE_MISMATCH, "more reactions requested than spans stepped");
    for (uint32_t q = 0; q < nspans; ++q) out_reactions[q] = h->last[q];
    return VXL_OK;
  } catch (...) {
    return set_error(VXL_PANIC_CAUGHT, "exception in vxl_sph_step_coupled");
  }
}

vxl_status vxl_sph_read_rigid_bodies(vxl_sph_handle* h, uint32_t scene, vxl_sph_rigid_body* out, uint32_t n) {
  HANDLE_OR_FAIL(h);
  try {
    return h->e->read_rigid_bodies(scene, out, n);
  } catch (...) {
    return set_error(VXL_PANIC_CAUGHT, "exception in vxl_sph_read_rigid_bodies");
  }
}

vxl_status vxl_sph_set_providers(vxl_sph_handle* h, uint32_t scene, const vxl_sph_provider* providers,
                                 uint32_t nproviders, const vxl_sph_wall_plane* planes, uint32_t nplanes) {
  HANDLE_OR_FAIL(h);
  try {
    return h->e->set_providers(scene, providers, nproviders, planes, nplanes);
  } catch (...) {
    return set_error(VXL_PANIC_CAUGHT, "exception in vxl_sph_set_providers");
  }
}

vxl_status vxl_sph_set_wall_contacts(vxl_sph_handle* h, uint32_t scene, uint32_t side, const uint32_t* ids,
                                     const uint32_t* start, uint32_t n_entries, const float* planes,
                                     uint32_t n_planes) {
  HANDLE_OR_FAIL(h);
  try {
    return h->e->set_wall_contacts(scene, side, ids, start, n_entries, planes, n_planes);
  } catch (...) {
    return set_error(VXL_PANIC_CAUGHT, "exception in vxl_sph_set_wall_contacts");
  }
}

vxl_status vxl_sph_set_body_lattice(vxl_sph_handle* h, uint32_t scene, const float* local_xyz,
                                    const uint32_t* body_index, uint64_t nb, uint32_t nbodies) {
  HANDLE_OR_FAIL(h);
  try {
    return h->e->set_body_lattice(scene, local_xyz, body_index, nb, nbodies);
  } catch (...) {
    return set_error(VXL_PANIC_CAUGHT, "exception in vxl_sph_set_body_lattice");
  }
}

vxl_status vxl_sph_set_body_poses(vxl_sph_handle* h, uint32_t scene, const vxl_sph_body_pose* poses,
                                  uint32_t nbodies) {
  HANDLE_OR_FAIL(h);
  try {
    return h->e->set_body_poses(scene, poses, nbodies);
  } catch (...) {
    return set_error(VXL_PANIC_CAUGHT, "exception in vxl_sph_set_body_poses");
  }
}

vxl_status vxl_sph_set_spans_scene(vxl_sph_handle* h, uint32_t scene, const vxl_sph_span* spans, uint32_t nspans) {
  HANDLE_OR_FAIL(h);
  return h->e->set_spans(scene, spans, nspans);
}

vxl_status vxl_sph_step_tick_async(vxl_sph_handle* h, float dt_tick, const vxl_sph_span* spans, uint32_t nspans) {
  try {
    HANDLE_OR_FAIL(h);
    if (h->e->scenes().size() == 1) {
      vxl_status s = h->e->set_spans(0, spans, nspans);
      if (s != VXL_OK) return s;
    } else if (nspans > 0) {
      return set_error(VXL_INVALID_ARGUMENT, "batched handles take spans through vxl_sph_set_spans_scene");
    }
    h->last_nspans = nspans;
    return h->e->step_tick_async(dt_tick);
  } catch (...) {
    return set_error(VXL_PANIC_CAUGHT, "exception in vxl_sph_step_tick_async");
  }
}

vxl_status vxl_sph_sync(vxl_sph_handle* h, vxl_sph_reaction* out_reactions, uint32_t nspans) {
  HANDLE_OR_FAIL(h);
  if (nspans > 0 && !out_reactions) return set_error(VXL_NULL_POINTER, "out_reactions is NULL with nspans > 0");
  vxl_status s = h->e->sync(&h->last);
  if (s != VXL_OK) return s;
  if (nspans > h->last.size()) return set_error(VXL_SIZE_MISMATCH, "more reactions requested than spans stepped");
  for (uint32_t q = 0; q < nspans; ++q) out_reactions[q] = h->last[q];
  return VXL_OK;
}

vxl_status vxl_sph_step_tick(vxl_sph_handle* h, float dt_tick, const vxl_sph_span* spans, uint32_t nspans,
                             vxl_sph_reaction* out_reactions) {
  if (nspans > 0 && !out_reactions) return set_error(VXL_NULL_POINTER, "out_reactions is NULL with nspans > 0");
  vxl_status s = vxl_sph_step_tick_async(h, dt_tick, spans, nspans);
  if (s != VXL_OK) return s;
  return vxl_sph_sync(h, out_reactions, nspans);
}

vxl_status vxl_sph_reactions_all(vxl_sph_handle* h, vxl_sph_reaction* out, uint32_t cap, uint32_t* n) {
  HANDLE_OR_FAIL(h);
  if (!n) return set_error(VXL_NULL_POINTER, "n is NULL");
  *n = (uint32_t)h->last.size();
  if (out)
    for (uint32_t q = 0; q < cap && q < h->last.size(); ++q) out[q] = h->last[q];
  return VXL_OK;
}

vxl_status vxl_sph_substep(vxl_sph_handle* h, float dt) {
  HANDLE_OR_FAIL(h);
  if (!(dt > 0.0f)) return set_error(VXL_INVALID_ARGUMENT, "dt must be > 0");
  return h->e->substep(std::vector<float>(h->e->scenes().size(), dt));
}

vxl_status vxl_sph_bounds(vxl_sph_handle* h, float lo[3], float hi[3]) {
  HANDLE_OR_FAIL(h);
  if (!lo || !hi) return set_error(VXL_NULL_POINTER, "NULL argument");
  return h->e->bounds(0, lo, hi);
}

vxl_status vxl_sph_read_state(vxl_sph_handle* h, float* pos_xyz, float* vel_xyz) {
  HANDLE_OR_FAIL(h);
  if (h->e->scenes().empty()) return VXL_OK;
  return h->e->read_state(0, pos_xyz, vel_xyz);
}

vxl_status vxl_sph_read_state_scene(vxl_sph_handle* h, uint32_t scene, float* pos_xyz, float* vel_xyz) {
  HANDLE_OR_FAIL(h);
  return h->e->read_state(scene, pos_xyz, vel_xyz);
}

vxl_status vxl_sph_write_state(vxl_sph_handle* h, const float* pos_xyz, const float* vel_xyz) {
  HANDLE_OR_FAIL(h);
  if (h->e->scenes().empty()) return VXL_OK;
  return h->e->write_state(0, pos_xyz, vel_xyz);
}

vxl_status vxl_sph_write_state_scene(vxl_sph_handle* h, uint32_t scene, const float* pos_xyz, const float* vel_xyz) {
  HANDLE_OR_FAIL(h);
  return h->e->write_state(scene, pos_xyz, vel_xyz);
}

vxl_status vxl_sph_set_record(vxl_sph_handle* h, int on) {
  HANDLE_OR_FAIL(h);
  h->e->set_record(on != 0);
  return VXL_OK;
}

vxl_status vxl_sph_read_fields(vxl_sph_handle* h, float* dens, float* press, float* acc_xyz, float* xsph_xyz,
                               float* bforce_xyz) {
  HANDLE_OR_FAIL(h);
  return h->e->read_fields(0, dens, press, acc_xyz, xsph_xyz, bforce_xyz);
}

vxl_status vxl_sph_read_fields_scene(vxl_sph_handle* h, uint32_t scene, float* dens, float* press, float* acc_xyz,
                                     float* xsph_xyz, float* bforce_xyz) {
  HANDLE_OR_FAIL(h);
  return h->e->read_fields(scene, dens, press, acc_xyz, xsph_xyz, bforce_xyz);
}

vxl_status vxl_sph_export_grid(vxl_sph_handle* h, uint32_t* items, uint32_t* start, uint64_t start_cap,
                               uint32_t* bins, vxl_sph_grid_info* info) {
  HANDLE_OR_FAIL(h);
  if (info && !check_header(info->hdr, sizeof(vxl_sph_grid_info)))
    return set_error(VXL_SIZE_MISMATCH, "grid_info header");
  return h->e->export_grid(0, items, start, start_cap, bins, info);
}

vxl_status vxl_sph_export_grid_scene(vxl_sph_handle* h, uint32_t scene, uint32_t* items, uint32_t* start,
                                     uint64_t start_cap, uint32_t* bins, vxl_sph_grid_info* info) {
  HANDLE_OR_FAIL(h);
  if (info && !check_header(info->hdr, sizeof(vxl_sph_grid_info)))
    return set_error(VXL_SIZE_MISMATCH, "grid_info header");
  return h->e->export_grid(scene, items, start, start_cap, bins, info);
}

vxl_status vxl_sph_export_neighbors(vxl_sph_handle* h, uint64_t* offsets, uint64_t offsets_len, uint32_t* entries,
                                    uint64_t entries_cap, uint64_t* total) {
  HANDLE_OR_FAIL(h);
  return h->e->export_neighbors(0, offsets, offsets_len, entries, entries_cap, total);
}

vxl_status vxl_sph_get_stats(vxl_sph_handle* h, vxl_sph_stats* out) {
  HANDLE_OR_FAIL(h);
  if (!out) return set_error(VXL_NULL_POINTER, "NULL argument");
  if (!check_header(out->hdr, sizeof(vxl_sph_stats))) return set_error(VXL_SIZE_MISMATCH, "stats header");
  uint64_t nf = 0, nb = 0;
  for (auto& s : h->e->scenes()) {
    nf += s.nf;
    nb += s.nb;
  }
  out->n_fluid = nf;
  out->n_boundary = nb;
  out->cells = h->e->cells_last();
  out->launches_last_tick = h->e->launches_last_tick();
  out->device_bytes = h->e->device_bytes();
  out->last_tick_ms = 0.0f;
  return VXL_OK;
}

vxl_status vxl_sph_set_stream(vxl_sph_handle* h, void* cuda_stream) {
  HANDLE_OR_FAIL(h);
  h->e->set_stream((cudaStream_t)cuda_stream);
  return VXL_OK;
}

vxl_status vxl_sph_set_profile(vxl_sph_handle* h, int on) {
  HANDLE_OR_FAIL(h);
  return h->e->set_profile(on != 0);
}

vxl_status vxl_sph_profile_read(vxl_sph_handle* h, uint32_t k, const char** name, double* total_ms,
                                uint64_t* launches) {
  HANDLE_OR_FAIL(h);
  return h->e->profile_read(k, name, total_ms, launches);
}

vxl_status vxl_sph_set_tuning(vxl_sph_handle* h, const vxl_sph_tuning* t) {
  HANDLE_OR_FAIL(h);
  if (!t) return set_error(VXL_NULL_POINTER, "tuning is NULL");
  if (!check_header(t->hdr, sizeof(vxl_sph_tuning))) return set_error(VXL_SIZE_MISMATCH, "tuning header");
  if ((t->block != 128 && t->block != 256) || t->tile < t->block || t->tile % 128 != 0 || t->waves > 4 ||
      t->density > 1u)
    return set_error(VXL_INVALID_ARGUMENT,
                     "block must be 128/256, tile a multiple of 128 and >= block, waves 0..4, density 0/1");
  h->e->set_tuning(vxl::Tuning{t->block, t->tile, t->waves, t->density});
  return VXL_OK;
}

vxl_status vxl_sph_get_tuning(vxl_sph_handle* h, vxl_sph_tuning* t) {
  HANDLE_OR_FAIL(h);
  if (!t) return set_error(VXL_NULL_POINTER, "tuning is NULL");
  if (!check_header(t->hdr, sizeof(vxl_sph_tuning))) return set_error(VXL_SIZE_MISMATCH, "tuning header");
  t->block = h->e->tuning().block;
  t->tile = h->e->tuning().tile;
  t->waves = h->e->tuning().waves;
  t->density = h->e->tuning().density;
  return VXL_OK;
}

vxl_status vxl_sph_autotune(vxl_sph_handle* h, float dt_tick, uint32_t trials, vxl_sph_tuning* best) {
  HANDLE_OR_FAIL(h);
  if (best && !check_header(best->hdr, sizeof(vxl_sph_tuning))) return set_error(VXL_SIZE_MISMATCH, "tuning header");
  vxl::Tuning t;
  float ms = 0.f;
  vxl_status s = h->e->autotune(dt_tick, trials ? trials : 3, &t, &ms);
  if (s != VXL_OK) return s;
  if (best) {
    best->block = t.block;
    best->tile = t.tile;
    best->waves = t.waves;
    best->density = t.density;
    best->ms_per_substep = ms;
  }
  return VXL_OK;
}

}  // extern "C"
