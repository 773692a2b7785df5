// Served form of the WCSPH step: a request loop with continuous batching.
//
// Requests (a scene + a tick count) are queued on submit. Each vxl_sph_serve_step first
// retires the scenes that finished their ticks (their final state is copied to the host
// and their slots are compacted away), then admits queued requests, first fit in
// submission order, while their device footprint fits the budget (particle slots plus
// their grid's cell budget), and then advances every admitted scene by one substep of
// its own dt in one pass of the engine: requests that arrive while others are on the GPU
// join the batch at the next substep boundary. Scene state stays on the device from
// admission to retirement.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "sph_engine.h"
#include "vxl_sph.h"
#include "vxl_sph_internal.h"

using vxl::Engine;
using vxl::set_error;

namespace {

enum ReqState : uint32_t { kQueued = 0, kRunning = 1, kDone = 2, kRejected = 3 };

struct Request {
  uint64_t id = 0;
  vxl_sph_params params{};
  uint64_t nf = 0, nb = 0;
  std::vector<float> pos, vel, pmass;
  uint32_t ticks_total = 0, ticks_done = 0, sub_in_tick = 0;
  uint32_t state = kQueued;
  double submit_s = 0, admit_s = 0, done_s = 0, tick_start_s = 0;
  std::vector<double> tick_ms;
  uint64_t slot_bytes = 0, cells = 0;
};

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double idx = q * (double)(v.size() - 1);
  const size_t lo = (size_t)idx;
  const size_t hi = std::min(v.size() - 1, lo + 1);
  const double f = idx - (double)lo;
  return v[lo] * (1.0 - f) + v[hi] * f;
}

}  // namespace

struct vxl_sph_server {
  Engine* e = nullptr;
  uint64_t budget = 0, slot_cap = 0, cell_cap = 0;
  uint64_t used_slots = 0, used_cells = 0;
  std::map<uint64_t, Request> req;
  std::deque<uint64_t> queue;
  std::vector<uint64_t> active;  // request id of each engine scene, in scene order
  uint64_t active_fluid = 0;     // fluid particles of the admitted scenes
  uint64_t batch_cap = 0;        // admission stops at this many fluid particles per substep (0: none)
  uint64_t next_id = 1;
  std::chrono::steady_clock::time_point t0;

  double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

extern "C" {

vxl_status vxl_sph_serve_create(int32_t device, uint64_t budget_bytes, uint32_t max_scenes, vxl_sph_server** out) {
  if (!out) return set_error(VXL_NULL_POINTER, "out is NULL");
  *out = nullptr;
  if (budget_bytes < (64ull << 20)) return set_error(VXL_INVALID_ARGUMENT, "budget below 64 MiB");
  if (max_scenes == 0) max_scenes = 4096;
  // split the budget: 85% particle slots, 15% cells
  const uint64_t per_slot = Engine::bytes_per_slot(64);
  uint64_t slots = (budget_bytes / 100 * 85) / per_slot;
  uint64_t cells = (budget_bytes / 100 * 15) / Engine::bytes_per_cell();
  slots = std::min<uint64_t>(slots, (1ull << 31) - 1);
  cells = std::min<uint64_t>(cells, (1ull << 31) - 2);
  Engine* e = nullptr;
  vxl_status s = Engine::create(device, slots, cells, max_scenes, &e);
  if (s != VXL_OK) return s;
  auto* sv = new (std::nothrow) vxl_sph_server();
  if (!sv) {
    delete e;
    return set_error(VXL_OUT_OF_MEMORY, "host allocation failed");
  }
  sv->e = e;
  sv->budget = budget_bytes;
  sv->slot_cap = slots;
  sv->cell_cap = cells;
  sv->t0 = std::chrono::steady_clock::now();
  *out = sv;
  return VXL_OK;
}

vxl_status vxl_sph_serve_destroy(vxl_sph_server* s) {
  if (!s) return set_error(VXL_NULL_POINTER, "server is NULL");
  delete s->e;
  delete s;
  return VXL_OK;
}

vxl_status vxl_sph_serve_submit(vxl_sph_server* s, const vxl_sph_desc* d, uint32_t ticks, uint64_t* out_id) {
  if (!s || !d || !out_id) return set_error(VXL_NULL_POINTER, "NULL argument");
  if (d->hdr.version != VXL_SPH_ABI_VERSION || d->params.hdr.version != VXL_SPH_ABI_VERSION)
    return set_error(VXL_VERSION_MISMATCH, "ABI version mismatch");
  if (d->hdr.size != sizeof(vxl_sph_desc) || d->params.hdr.size != sizeof(vxl_sph_params))
    return set_error(VXL_SIZE_MISMATCH, "struct size mismatch");
  const uint64_t nt = d->n_fluid + d->n_boundary;
  if (nt == 0 || !d->pos_xyz || !d->vel_xyz || (d->n_boundary && !d->pmass))
    return set_error(VXL_NULL_POINTER, "empty scene or NULL arrays");
  if (ticks == 0) return set_error(VXL_INVALID_ARGUMENT, "ticks must be > 0");
  Request r;
  r.id = s->next_id++;
  r.params = d->params;
  if (!r.params.substeps) r.params.substeps = 1;
  r.nf = d->n_fluid;
  r.nb = d->n_boundary;
  r.pos.assign(d->pos_xyz, d->pos_xyz + 3 * nt);
  r.vel.assign(d->vel_xyz, d->vel_xyz + 3 * nt);
  r.pmass.assign(nt, d->params.particle_mass);
  if (d->pmass) r.pmass.assign(d->pmass, d->pmass + nt);
  r.ticks_total = ticks;
  r.submit_s = s->now();
  r.cells = d->params.max_bins ? d->params.max_bins : (1u << 21);
  *out_id = r.id;
  if (nt > s->slot_cap || r.cells > s->cell_cap) {
    r.state = kRejected;
    s->req[r.id] = std::move(r);
    return set_error(VXL_OUT_OF_MEMORY, "request can never fit the budget");
  }
  s->queue.push_back(r.id);
  s->req[r.id] = std::move(r);
  return VXL_OK;
}

vxl_status vxl_sph_serve_step(vxl_sph_server* s, float dt_tick, vxl_sph_serve_report* rep) {
  if (!s) return set_error(VXL_NULL_POINTER, "server is NULL");
  if (!(dt_tick > 0.0f)) return set_error(VXL_INVALID_ARGUMENT, "dt_tick must be > 0");
  if (rep && (rep->hdr.size != sizeof(vxl_sph_serve_report) || rep->hdr.version != VXL_SPH_ABI_VERSION))
    return set_error(VXL_SIZE_MISMATCH, "report header");
  cudaSetDevice(s->e->device());
  uint32_t retired = 0, admitted = 0;
  // 1. retire finished scenes (copy their state out), compact. Every finished scene's
  // state is read first; requests and budget counters change only once all reads and the
  // compaction have succeeded, so a failed call can be repeated without counting twice.
  std::vector<uint32_t> drop;
  std::vector<std::vector<float>> out_pos, out_vel;
  for (uint32_t q = 0; q < s->active.size(); ++q) {
    const Request& r = s->req[s->active[q]];
    if (r.ticks_done >= r.ticks_total) {
      out_pos.emplace_back((size_t)3 * (r.nf + r.nb));
      out_vel.emplace_back((size_t)3 * (r.nf + r.nb));
      vxl_status st = s->e->read_state(q, out_pos.back().data(), out_vel.back().data());
      if (st != VXL_OK) return st;
      drop.push_back(q);
    }
  }
  if (!drop.empty()) {
    vxl_status st = s->e->remove_scenes(drop);
    if (st != VXL_OK) return st;
    const double t = s->now();
    for (size_t k = 0; k < drop.size(); ++k) {
      Request& r = s->req[s->active[drop[k]]];
      r.pos.swap(out_pos[k]);
      r.vel.swap(out_vel[k]);
      r.state = kDone;
      r.done_s = t;
      s->used_slots -= r.nf + r.nb;
      s->used_cells -= r.cells;
      s->active_fluid -= r.nf;
    }
    std::vector<uint64_t> keep;
    for (uint32_t q = 0; q < s->active.size(); ++q)
      if (std::find(drop.begin(), drop.end(), q) == drop.end()) keep.push_back(s->active[q]);
    s->active.swap(keep);
    retired = (uint32_t)drop.size();
  }
  // 2. admit queued requests that fit (first fit, in submission order)
  for (auto it = s->queue.begin(); it != s->queue.end();) {
    Request& r = s->req[*it];
    const uint64_t nt = r.nf + r.nb;
    // the batch cap (vxl_sph_serve_set_batch_cap) bounds the fluid particles stepped per
    // substep; a request larger than the cap is admitted alone
    const bool under_cap = s->batch_cap == 0 || s->active.empty() || s->active_fluid + r.nf <= s->batch_cap;
    if (s->used_slots + nt <= s->slot_cap && s->used_cells + r.cells <= s->cell_cap &&
        s->e->scenes().size() < 0xffffffu && under_cap) {
      vxl_sph_params p = r.params;
      vxl_status st = s->e->add_scene(p, r.nf, r.nb, r.pos.data(), r.vel.data(), r.pmass.data(), r.id, nullptr);
      if (st == VXL_OUT_OF_MEMORY) {  // scene table full: wait
        ++it;
        continue;
      }
      if (st != VXL_OK) {
        r.state = kRejected;
        it = s->queue.erase(it);
        continue;
      }
      r.state = kRunning;
      r.admit_s = s->now();
      r.tick_start_s = r.admit_s;
      s->used_slots += nt;
      s->used_cells += r.cells;
      s->active_fluid += r.nf;
      s->active.push_back(r.id);
      ++admitted;
      it = s->queue.erase(it);
    } else {
      ++it;
    }
  }
  // 3. one substep of every admitted scene, each with its own dt
  uint64_t particles = 0;
  if (!s->active.empty()) {
    std::vector<float> dt(s->active.size());
    for (uint32_t q = 0; q < s->active.size(); ++q) {
      const Request& r = s->req[s->active[q]];
      dt[q] = dt_tick / (float)r.params.substeps;
      particles += r.nf;
    }
    vxl_status st = s->e->substep(dt);
    if (st != VXL_OK) return st;
    const double t = s->now();
    for (uint32_t q = 0; q < s->active.size(); ++q) {
      Request& r = s->req[s->active[q]];
      if (++r.sub_in_tick >= r.params.substeps) {
        r.sub_in_tick = 0;
        ++r.ticks_done;
        r.tick_ms.push_back((t - r.tick_start_s) * 1e3);
        r.tick_start_s = t;
      }
    }
  }
  if (rep) {
    rep->active = (uint32_t)s->active.size();
    rep->queued = (uint32_t)s->queue.size();
    rep->admitted = admitted;
    rep->retired = retired;
    rep->particles = particles;
    rep->device_bytes_in_use = s->used_slots * Engine::bytes_per_slot(64) + s->used_cells * Engine::bytes_per_cell();
  }
  return VXL_OK;
}

vxl_status vxl_sph_serve_set_batch_cap(vxl_sph_server* s, uint64_t max_fluid_particles) {
  if (!s) return set_error(VXL_NULL_POINTER, "server is NULL");
  s->batch_cap = max_fluid_particles;
  return VXL_OK;
}

vxl_status vxl_sph_serve_poll(vxl_sph_server* s, uint64_t id, vxl_sph_request_status* out) {
  if (!s || !out) return set_error(VXL_NULL_POINTER, "NULL argument");
  if (out->hdr.size != sizeof(vxl_sph_request_status) || out->hdr.version != VXL_SPH_ABI_VERSION)
    return set_error(VXL_SIZE_MISMATCH, "status header");
  auto it = s->req.find(id);
  if (it == s->req.end()) return set_error(VXL_INVALID_ARGUMENT, "unknown request id");
  const Request& r = it->second;
  out->state = r.state;
  out->ticks_done = r.ticks_done;
  out->ticks_total = r.ticks_total;
  out->submit_s = r.submit_s;
  out->admit_s = r.admit_s;
  out->done_s = r.done_s;
  out->tick_p50_ms = percentile(r.tick_ms, 0.50);
  out->tick_p99_ms = percentile(r.tick_ms, 0.99);
  return VXL_OK;
}

vxl_status vxl_sph_serve_read(vxl_sph_server* s, uint64_t id, float* pos_xyz, float* vel_xyz) {
  if (!s) return set_error(VXL_NULL_POINTER, "server is NULL");
  auto it = s->req.find(id);
  if (it == s->req.end()) return set_error(VXL_INVALID_ARGUMENT, "unknown request id");
  Request& r = it->second;
  const uint64_t nt = r.nf + r.nb;
  if (r.state == kRunning) {
    for (uint32_t q = 0; q < s->active.size(); ++q)
      if (s->active[q] == id) return s->e->read_state(q, pos_xyz, vel_xyz);
    return set_error(VXL_NOT_READY, "request not resident");
  }
  if (r.state == kDone || r.state == kQueued) {
    if (pos_xyz) std::memcpy(pos_xyz, r.pos.data(), nt * 12);
    if (vel_xyz) std::memcpy(vel_xyz, r.vel.data(), nt * 12);
    return VXL_OK;
  }
  return set_error(VXL_NOT_READY, "request was rejected");
}

vxl_status vxl_sph_serve_tick_times(vxl_sph_server* s, uint64_t id, double* out_ms, uint32_t cap, uint32_t* n) {
  if (!s || !n) return set_error(VXL_NULL_POINTER, "NULL argument");
  if (cap > 0 && !out_ms) return set_error(VXL_NULL_POINTER, "out_ms is NULL with cap > 0");
  auto it = s->req.find(id);
  if (it == s->req.end()) return set_error(VXL_INVALID_ARGUMENT, "unknown request id");
  const std::vector<double>& t = it->second.tick_ms;
  *n = (uint32_t)t.size();
  for (uint32_t q = 0; q < cap && q < t.size(); ++q) out_ms[q] = t[q];
  return VXL_OK;
}

}  // extern "C"
