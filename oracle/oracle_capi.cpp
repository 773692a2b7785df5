// C entry points over the WCSPH oracle — TEST INFRASTRUCTURE ONLY.
//
// tests/ (through ctypes), __graft_entry__.smoke() and bench.py's cpu_baseline leg load
// this library as the checker. The shipped library never links it.
//
// Each handle holds an f32 restatement (bit-identical to the reference's Rust CPU path)
// or its FP64 twin (same formulas and constants in double precision).
#include <chrono>
#include <cstring>
#include <memory>
#include <type_traits>

#include "wcsph_oracle.hpp"

using namespace oracle;

extern "C" {

struct orc_cfg {
  float rest_density;
  float smoothing_radius;
  float xsph_viscosity;
  uint32_t tensile_instability_suppression;
  float sound_speed;
  float gamma_tait;
  uint32_t substeps;
  uint32_t threads;
  uint32_t boundary_layers;
  float gravity[3];
  float max_speed_frac;
  float artificial_viscosity;
  uint64_t max_bins;
};

struct orc_body {
  uint32_t id;
  uint32_t shape;   // 0 = box (half), 1 = sphere (radius)
  float half[3];
  float radius;
  float pos[3];
  float rot[4];     // x, y, z, w
  float linvel[3];
  float angvel[3];
};

struct orc_span {
  uint32_t body;
  float origin[3];
  uint32_t start, end;
};

struct orc_reaction {
  uint32_t body;
  float force[3];
  float torque[3];
};

// Provider walls: kind 0 = axis-aligned faces (axis, d = plane, sign), 1 = convex
// half-space set (normal, d); planes [first, first + count) of the plane array.
struct orc_wall_plane {
  float normal[3];
  float d;
  uint32_t axis;
  float sign;
};

struct orc_provider {
  uint32_t kind;
  uint32_t first, count;
  uint32_t has_bounds;
  float bmin[3], bmax[3];
};
}

namespace {

template <class R>
FluidConfig<R> to_cfg(const orc_cfg* c) {
  FluidConfig<R> f;
  f.rest_density = (R)c->rest_density;
  f.smoothing_radius = (R)c->smoothing_radius;
  f.xsph_viscosity = (R)c->xsph_viscosity;
  f.tensile_instability_suppression = c->tensile_instability_suppression != 0;
  f.sound_speed = (R)c->sound_speed;
  f.gamma_tait = (R)c->gamma_tait;
  f.substeps = c->substeps;
  f.threads = c->threads;
  f.boundary_layers = c->boundary_layers;
  f.gravity = V3<R>((R)c->gravity[0], (R)c->gravity[1], (R)c->gravity[2]);
  f.max_speed_frac = (R)c->max_speed_frac;
  f.artificial_viscosity = (R)c->artificial_viscosity;
  f.max_bins = c->max_bins ? c->max_bins : GRID_MAX_BINS;
  return f;
}

struct Handle {
  std::unique_ptr<FluidSystem<float>> f;
  std::unique_ptr<FluidSystem<double>> d;
};

template <class R, class Fn>
void with(Handle* h, Fn&& fn) {
  if (h->f) fn(*h->f);
  else fn(*h->d);
}

template <class R>
Body<R> to_body(const orc_body& b) {
  Body<R> o;
  o.id = b.id;
  o.shape.kind = b.shape == 1 ? ShapeKind::Sphere : ShapeKind::Box;
  o.shape.half = V3<R>(b.half[0], b.half[1], b.half[2]);
  o.shape.radius = b.radius;
  o.pose.pos = V3<R>(b.pos[0], b.pos[1], b.pos[2]);
  o.pose.rot = Quat<R>(b.rot[0], b.rot[1], b.rot[2], b.rot[3]);
  o.pose.linvel = V3<R>(b.linvel[0], b.linvel[1], b.linvel[2]);
  o.pose.angvel = V3<R>(b.angvel[0], b.angvel[1], b.angvel[2]);
  return o;
}

}  // namespace

extern "C" {

void* orc_create(const orc_cfg* cfg, const float origin[3], const uint64_t dims[3], float spacing,
                 int fp64) {
  auto* h = new Handle();
  size_t d[3] = {(size_t)dims[0], (size_t)dims[1], (size_t)dims[2]};
  if (fp64)
    h->d.reset(new FluidSystem<double>(to_cfg<double>(cfg), V3<double>(origin[0], origin[1], origin[2]), d,
                                       (double)spacing));
  else
    h->f.reset(new FluidSystem<float>(to_cfg<float>(cfg), V3<float>(origin[0], origin[1], origin[2]), d,
                                      spacing));
  return h;
}

void orc_destroy(void* p) { delete (Handle*)p; }

uint64_t orc_n_total(void* p) {
  uint64_t n = 0;
  with<float>((Handle*)p, [&](auto& s) { n = s.n_total(); });
  return n;
}
uint64_t orc_n_fluid(void* p) {
  uint64_t n = 0;
  with<float>((Handle*)p, [&](auto& s) { n = s.n_fluid; });
  return n;
}
double orc_mass(void* p) {
  double m = 0;
  with<float>((Handle*)p, [&](auto& s) { m = (double)s.mass; });
  return m;
}
// The system's kernel constants (fluid_access.rs:7-13): h, h2, k6, ks, w0, skin.
void orc_consts(void* p, double out[6]) {
  with<float>((Handle*)p, [&](auto& s) {
    out[0] = (double)s.h;
    out[1] = (double)s.h2;
    out[2] = (double)s.k6;
    out[3] = (double)s.ks;
    out[4] = (double)s.w0;
    out[5] = (double)s.skin;
  });
}
void orc_set_threads(void* p, uint32_t t) {
  with<float>((Handle*)p, [&](auto& s) { s.cfg.threads = t; });
}

// Override the fluid particle mass (and the fluid prefix's pmass), e.g. to give the FP64
// twin exactly the f32 system's calibrated mass.
void orc_set_mass(void* p, double m) {
  with<float>((Handle*)p, [&](auto& s) {
    using R = std::decay_t<decltype(s.h)>;
    s.mass = (R)m;
    for (size_t i = 0; i < s.n_fluid; ++i) s.pmass[i] = (R)m;
  });
}

// Lattice mass calibration without building a system (crates/vxl-phys-fluid/src/fluid_access.rs:27-42).
float orc_lattice_mass(const orc_cfg* cfg, float spacing) {
  return FluidSystem<float>::lattice_mass(to_cfg<float>(cfg), spacing);
}

// Overwrite positions/velocities of all n_total particles (harness-only: the reference
// has no position setter; seeded jitter is applied through this after construction).
int orc_set_state(void* p, const float* pos, const float* vel, uint64_t n) {
  int rc = 0;
  with<float>((Handle*)p, [&](auto& s) {
    using R = std::decay_t<decltype(s.h)>;
    if (n != s.n_total()) { rc = 3; return; }
    for (size_t i = 0; i < n; ++i) {
      if (pos) s.pos[i] = V3<R>(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
      if (vel) s.vel[i] = V3<R>(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
    }
  });
  return rc;
}

// set_boundary_particles (crates/vxl-phys-fluid/src/fluid_step.rs:13-53); returns N_b.
uint64_t orc_set_bodies(void* p, const orc_body* bodies, uint32_t n) {
  uint64_t nb = 0;
  with<float>((Handle*)p, [&](auto& s) {
    using R = std::decay_t<decltype(s.h)>;
    std::vector<Body<R>> v;
    for (uint32_t i = 0; i < n; ++i) v.push_back(to_body<R>(bodies[i]));
    nb = s.set_boundary_particles(v);
  });
  return nb;
}

// Register the fluid's boundary providers, in order (FluidSystem::set_boundaries,
// crates/vxl-phys-fluid/src/fluid_access.rs:184-186, with the providers themselves).
void orc_set_providers(void* p, const orc_provider* pr, uint32_t n, const orc_wall_plane* planes) {
  with<float>((Handle*)p, [&](auto& s) {
    using R = std::decay_t<decltype(s.h)>;
    s.providers.clear();
    for (uint32_t i = 0; i < n; ++i) {
      Provider<R> q;
      q.kind = pr[i].kind;
      q.has_bounds = pr[i].has_bounds != 0;
      q.bmin = V3<R>(pr[i].bmin[0], pr[i].bmin[1], pr[i].bmin[2]);
      q.bmax = V3<R>(pr[i].bmax[0], pr[i].bmax[1], pr[i].bmax[2]);
      for (uint32_t k = pr[i].first; k < pr[i].first + pr[i].count; ++k) {
        WallPlane<R> w;
        w.n = V3<R>(planes[k].normal[0], planes[k].normal[1], planes[k].normal[2]);
        w.d = planes[k].d;
        w.axis = planes[k].axis;
        w.sign = planes[k].sign;
        q.planes.push_back(w);
      }
      s.providers.push_back(q);
    }
  });
}

// Contact table of one side (0: mirror, 1: projection) as the GPU tier uploads it
// (WallStage::upload, crates/vxl-phys-gpu/src/pipeline/walls.rs:100-121): entries e with
// particle ids[e] (fluid, ascending) and planes [start[e], start[e + 1]) of `planes`
// (point xyz, outward normal xyz). n_entries = 0 removes the table.
void orc_set_wall_contacts(void* p, uint32_t side, const uint32_t* ids, const uint32_t* start, uint32_t n_entries,
                           const float* planes) {
  with<float>((Handle*)p, [&](auto& s) {
    using R = std::decay_t<decltype(s.h)>;
    auto& t = s.ctab[side & 1u];
    t.off.clear();
    t.pt.clear();
    t.n.clear();
    if (n_entries == 0) return;
    t.off.assign(s.n_fluid + 1, 0);
    std::vector<uint32_t> cnt(s.n_fluid, 0);
    for (uint32_t e = 0; e < n_entries; ++e) cnt[ids[e]] = start[e + 1] - start[e];
    for (size_t i = 0; i < s.n_fluid; ++i) t.off[i + 1] = t.off[i] + cnt[i];
    t.pt.resize(t.off[s.n_fluid]);
    t.n.resize(t.off[s.n_fluid]);
    for (uint32_t e = 0; e < n_entries; ++e) {
      uint32_t o = t.off[ids[e]];
      for (uint32_t k = start[e]; k < start[e + 1]; ++k, ++o) {
        const float* q = planes + 6 * (size_t)k;
        t.pt[o] = V3<R>(q[0], q[1], q[2]);
        t.n[o] = V3<R>(q[3], q[4], q[5]);
      }
    }
  });
}

// Replace the boundary suffix with explicit particles (the FluidStepper view: the
// facade hands over pos/vel/pmass of the boundary segment plus the span table).
int orc_set_boundary_raw(void* p, uint64_t nb, const float* pos, const float* vel, const float* pm,
                         const orc_span* spans, uint32_t nspans) {
  with<float>((Handle*)p, [&](auto& s) {
    using R = std::decay_t<decltype(s.h)>;
    s.truncate_to_fluid();
    for (size_t k = 0; k < nb; ++k) {
      s.pos.push_back(V3<R>(pos[3 * k], pos[3 * k + 1], pos[3 * k + 2]));
      s.vel.push_back(V3<R>(vel[3 * k], vel[3 * k + 1], vel[3 * k + 2]));
      s.pmass.push_back((R)pm[k]);
      s.dens.push_back(R(0));
      s.press.push_back(R(0));
      s.acc.push_back(V3<R>());
      s.xsph.push_back(V3<R>());
    }
    for (uint32_t q = 0; q < nspans; ++q)
      s.spans.push_back(Span<R>{spans[q].body, V3<R>(spans[q].origin[0], spans[q].origin[1], spans[q].origin[2]),
                                spans[q].start, spans[q].end});
    s.bforce.resize(s.pos.size(), V3<R>());
    s.breact.clear();
  });
  return 0;
}

void orc_step(void* p, float dt_tick) {
  with<float>((Handle*)p, [&](auto& s) { s.step((decltype(s.h))dt_tick); });
}
void orc_substep(void* p, float dt) {
  with<float>((Handle*)p, [&](auto& s) { s.substep((decltype(s.h))dt); });
}

// Timed ticks for the CPU baseline: returns wall seconds.
double orc_run_ticks(void* p, float dt_tick, uint32_t ticks) {
  auto t0 = std::chrono::steady_clock::now();
  for (uint32_t t = 0; t < ticks; ++t) orc_step(p, dt_tick);
  auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

// Read any subset of the per-particle arrays (all n_total long; xyz arrays 3*n).
// Values are converted to double so the FP64 twin loses nothing.
void orc_read(void* p, double* pos, double* vel, double* dens, double* press, double* acc, double* xsph,
              double* bforce, double* pmass) {
  with<float>((Handle*)p, [&](auto& s) {
    size_t n = s.n_total();
    for (size_t i = 0; i < n; ++i) {
      if (pos) { pos[3 * i] = s.pos[i].x; pos[3 * i + 1] = s.pos[i].y; pos[3 * i + 2] = s.pos[i].z; }
      if (vel) { vel[3 * i] = s.vel[i].x; vel[3 * i + 1] = s.vel[i].y; vel[3 * i + 2] = s.vel[i].z; }
      if (acc) { acc[3 * i] = s.acc[i].x; acc[3 * i + 1] = s.acc[i].y; acc[3 * i + 2] = s.acc[i].z; }
      if (xsph) { xsph[3 * i] = s.xsph[i].x; xsph[3 * i + 1] = s.xsph[i].y; xsph[3 * i + 2] = s.xsph[i].z; }
      if (bforce) { bforce[3 * i] = s.bforce[i].x; bforce[3 * i + 1] = s.bforce[i].y; bforce[3 * i + 2] = s.bforce[i].z; }
      if (dens) dens[i] = s.dens[i];
      if (press) press[i] = s.press[i];
      if (pmass) pmass[i] = s.pmass[i];
    }
  });
}

// Same as orc_read for f32 handles, without conversion (bit patterns preserved).
void orc_read_f32(void* p, float* pos, float* vel, float* dens, float* press, float* acc, float* xsph,
                  float* bforce, float* pmass) {
  auto* h = (Handle*)p;
  if (!h->f) return;
  auto& s = *h->f;
  size_t n = s.n_total();
  for (size_t i = 0; i < n; ++i) {
    if (pos) std::memcpy(pos + 3 * i, &s.pos[i], 12);
    if (vel) std::memcpy(vel + 3 * i, &s.vel[i], 12);
    if (acc) std::memcpy(acc + 3 * i, &s.acc[i], 12);
    if (xsph) std::memcpy(xsph + 3 * i, &s.xsph[i], 12);
    if (bforce) std::memcpy(bforce + 3 * i, &s.bforce[i], 12);
    if (dens) dens[i] = s.dens[i];
    if (press) press[i] = s.press[i];
    if (pmass) pmass[i] = s.pmass[i];
  }
}

// Grid table of the last substep (the reference's neighbor_grid()). Returns the
// number of cells; start must hold cells+1 entries, items n_total entries.
uint64_t orc_grid(void* p, uint32_t* start, uint64_t start_cap, uint32_t* items, float* min3, float* inv_bin,
                  uint32_t* dims3) {
  auto* h = (Handle*)p;
  if (!h->f) return 0;
  auto& g = h->f->grid;
  uint64_t total = (uint64_t)g.nx * g.ny * g.nz;
  if (dims3) { dims3[0] = g.nx; dims3[1] = g.ny; dims3[2] = g.nz; }
  if (min3) { min3[0] = g.min.x; min3[1] = g.min.y; min3[2] = g.min.z; }
  if (inv_bin) { inv_bin[0] = g.inv; inv_bin[1] = g.bin; }
  if (start && start_cap >= total + 1) std::memcpy(start, g.start.data(), (total + 1) * 4);
  if (items) std::memcpy(items, g.items.data(), g.items.size() * 4);
  return total;
}

// The neighbour lists of the next substep, the lists its density pass walks: the grid is
// rebuilt from the current positions exactly as FluidSystem::substep does
// (crates/vxl-phys-fluid/src/fluid_step.rs:96-100, grid.rs:29-76), and for every particle
// i the neighbours j of UniformGrid::for_neighbors_in (grid.rs:115-155) are listed in its
// walk order — all of them for a fluid particle, the fluid ones for a boundary particle
// (fluid_density.rs:59-69). CSR in particle order: offsets[0..n], entries[offsets[i]..
// offsets[i + 1]]. Returns the entry count; entries are written only if cap holds them.
uint64_t orc_neighbors(void* p, uint64_t* offsets, uint32_t* entries, uint64_t cap) {
  auto* hd = (Handle*)p;
  if (!hd->f) return 0;
  auto& s = *hd->f;
  UniformGrid<float> g;
  g.rebuild(s.pos, s.h, s.cfg.max_bins);
  const size_t n = s.pos.size(), nf = s.n_fluid;
  uint64_t total = 0;
  for (size_t i = 0; i < n; ++i) {
    if (offsets) offsets[i] = total;
    const bool fluid_i = i < nf;
    g.for_neighbors_in(s.pos, s.h2, i, [&](size_t j, const V3<float>&, float) {
      if (!fluid_i && j >= nf) return;
      if (entries && total < cap) entries[total] = (uint32_t)j;
      ++total;
    });
  }
  if (offsets) offsets[n] = total;
  return total;
}

uint32_t orc_reactions(void* p, orc_reaction* out, uint32_t cap) {
  uint32_t n = 0;
  with<float>((Handle*)p, [&](auto& s) {
    n = (uint32_t)s.breact.size();
    for (uint32_t k = 0; k < n && k < cap; ++k) {
      out[k].body = s.breact[k].body;
      out[k].force[0] = (float)s.breact[k].force.x;
      out[k].force[1] = (float)s.breact[k].force.y;
      out[k].force[2] = (float)s.breact[k].force.z;
      out[k].torque[0] = (float)s.breact[k].torque.x;
      out[k].torque[1] = (float)s.breact[k].torque.y;
      out[k].torque[2] = (float)s.breact[k].torque.z;
    }
  });
  return n;
}

// Run the aggregation alone on a given bforce suffix (the reference's C2 reaction
// test drives aggregate_reactions directly: crates/vxl-phys-fluid/src/tests.rs:667-712).
void orc_aggregate_with(void* p, const float* bforce_suffix, int clear) {
  auto* h = (Handle*)p;
  if (!h->f) return;
  auto& s = *h->f;
  if (clear) s.breact.clear();
  for (size_t k = s.n_fluid; k < s.n_total(); ++k) {
    size_t q = k - s.n_fluid;
    s.bforce[k] = V3<float>(bforce_suffix[3 * q], bforce_suffix[3 * q + 1], bforce_suffix[3 * q + 2]);
  }
  s.aggregate_reactions();
}
void orc_scale_reactions(void* p, float inv) {
  auto* h = (Handle*)p;
  if (!h->f) return;
  for (auto& e : h->f->breact) { e.force *= inv; e.torque *= inv; }
}

uint32_t orc_spans(void* p, orc_span* out, uint32_t cap) {
  uint32_t n = 0;
  with<float>((Handle*)p, [&](auto& s) {
    n = (uint32_t)s.spans.size();
    for (uint32_t k = 0; k < n && k < cap; ++k) {
      out[k].body = s.spans[k].body;
      out[k].origin[0] = (float)s.spans[k].origin.x;
      out[k].origin[1] = (float)s.spans[k].origin.y;
      out[k].origin[2] = (float)s.spans[k].origin.z;
      out[k].start = s.spans[k].start;
      out[k].end = s.spans[k].end;
    }
  });
  return n;
}

// grid_box alone (crates/vxl-phys-core/src/grid.rs:34-50).
void orc_grid_box(const float lo[3], const float hi[3], float h, uint64_t max_bins, float* min3, float* bin,
                  uint32_t* dims3) {
  GridBox<float> g = grid_box(V3<float>(lo[0], lo[1], lo[2]), V3<float>(hi[0], hi[1], hi[2]), h, max_bins);
  min3[0] = g.min.x; min3[1] = g.min.y; min3[2] = g.min.z;
  *bin = g.bin;
  dims3[0] = g.dims[0]; dims3[1] = g.dims[1]; dims3[2] = g.dims[2];
}

// Grid rebuild alone over arbitrary positions (n points, xyz).
uint64_t orc_rebuild_grid(const float* pos, uint64_t n, float h, uint64_t max_bins, uint32_t* start,
                          uint64_t start_cap, uint32_t* items, uint32_t* dims3) {
  std::vector<V3<float>> v(n);
  for (size_t i = 0; i < n; ++i) v[i] = V3<float>(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
  UniformGrid<float> g;
  g.rebuild(v, h, max_bins);
  uint64_t total = (uint64_t)g.nx * g.ny * g.nz;
  if (dims3) { dims3[0] = g.nx; dims3[1] = g.ny; dims3[2] = g.nz; }
  if (start && start_cap >= total + 1) std::memcpy(start, g.start.data(), (total + 1) * 4);
  if (items) std::memcpy(items, g.items.data(), n * 4);
  return total;
}

// Boundary lattice of one shape (crates/vxl-phys-fluid/src/boundary.rs:67-88).
// Returns the particle count; fills pts (3*cap floats) when cap suffices.
uint64_t orc_lattice(uint32_t shape, const float half[3], float radius, float s, float h, uint32_t layers,
                     float* pts, uint64_t cap, float* volume, uint64_t* n0) {
  Shape<float> sh;
  sh.kind = shape == 1 ? ShapeKind::Sphere : ShapeKind::Box;
  sh.half = V3<float>(half[0], half[1], half[2]);
  sh.radius = radius;
  BoundaryLattice<float> l = lattice(sh, s, h, layers);
  if (volume) *volume = l.volume;
  if (n0) *n0 = l.n0;
  if (pts && cap >= l.pts.size())
    for (size_t i = 0; i < l.pts.size(); ++i) std::memcpy(pts + 3 * i, &l.pts[i], 12);
  return l.pts.size();
}

// Self-sum used by the volume calibration (boundary.rs:104-129), for the
// calibration-consistency test (boundary.rs:367-372).
float orc_boundary_self_sum(const float* pts, uint64_t n, float h) {
  std::vector<V3<float>> v(n);
  for (size_t i = 0; i < n; ++i) v[i] = V3<float>(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
  return boundary_self_sum(v, h);
}

// The reference grid probe scene (crates/vxl-phys-gpu/examples/gpu_grid_probe.rs:181-226):
// n^3 lattice at spacing 0.05, origin (-n*s/2, 0.5, -n*s/2), default FluidConfig, no
// providers; 5 ticks, snapshot, 1 more tick; FNV hash of the last substep's table.
uint64_t orc_grid_probe_hash(uint64_t n, uint64_t max_bins, uint32_t threads) {
  float spacing = 0.05f;
  FluidConfig<float> cfg;
  cfg.threads = threads;
  cfg.max_bins = max_bins ? max_bins : GRID_MAX_BINS;
  float nf = (float)n;
  V3<float> origin(-nf * spacing * 0.5f, 0.5f, -nf * spacing * 0.5f);
  size_t dims[3] = {(size_t)n, (size_t)n, (size_t)n};
  FluidSystem<float> f(cfg, origin, dims, spacing);
  for (int t = 0; t < 5; ++t) f.step(1.0f / 60.0f);
  size_t np = f.n_fluid;
  f.step(1.0f / 60.0f);
  auto& g = f.grid;
  size_t total = (size_t)g.nx * g.ny * g.nz;
  return table_hash(g.start, g.items, total, np);
}

// Rigid bodies of the coupling loop (no contacts), float32: `substeps` rigid substeps of
// dt each, every body receiving its reaction (force, torque; 6 floats per body) each
// substep. bodies: pos[3], rot[4], linvel[3], angvel[3], inv_mass, local_inv_inertia[3],
// dynamic (as a float 0/1) — 18 floats per body, updated in place.
void orc_rigid_step(float* bodies, uint32_t n, const float* reactions, const float g[3], float dt, uint32_t substeps,
                    float max_linear, float max_angular) {
  for (uint32_t i = 0; i < n; ++i) {
    float* b = bodies + 18 * i;
    RigidBody<float> rb;
    rb.pos = V3<float>(b[0], b[1], b[2]);
    rb.rot = Quat<float>(b[3], b[4], b[5], b[6]);
    rb.linvel = V3<float>(b[7], b[8], b[9]);
    rb.angvel = V3<float>(b[10], b[11], b[12]);
    rb.inv_mass = b[13];
    rb.local_inv_inertia = V3<float>(b[14], b[15], b[16]);
    rb.dynamic = b[17] != 0.0f;
    const float* r = reactions + 6 * i;
    for (uint32_t k = 0; k < substeps; ++k)
      rigid_substep(rb, V3<float>(g[0], g[1], g[2]), V3<float>(r[0], r[1], r[2]), V3<float>(r[3], r[4], r[5]), dt,
                    max_linear, max_angular);
    const float out[17] = {rb.pos.x, rb.pos.y, rb.pos.z, rb.rot.x, rb.rot.y, rb.rot.z, rb.rot.w,
                           rb.linvel.x, rb.linvel.y, rb.linvel.z, rb.angvel.x, rb.angvel.y, rb.angvel.z,
                           rb.inv_mass, rb.local_inv_inertia.x, rb.local_inv_inertia.y, rb.local_inv_inertia.z};
    for (int k = 0; k < 17; ++k) b[k] = out[k];
  }
}

void orc_box_mass_props(const float half[3], float density, float* inv_mass, float local_inv_inertia[3]) {
  V3<float> d;
  box_mass_props(V3<float>(half[0], half[1], half[2]), density, *inv_mass, d);
  local_inv_inertia[0] = d.x;
  local_inv_inertia[1] = d.y;
  local_inv_inertia[2] = d.z;
}

}  // extern "C"
