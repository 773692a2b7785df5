// WCSPH oracle — TEST INFRASTRUCTURE ONLY.
//
// A CPU restatement of the reference's Rust WCSPH fluid step (crate `vxl-phys-fluid`
// of bfxh/RUST-WL), used by tests/, by __graft_entry__.smoke() and by bench.py's
// cpu_baseline leg as the checker. Nothing in the shipped library links or calls it.
//
// Every function cites the reference file:line it follows (paths are relative to the
// reference project root). Arithmetic is written in the reference's exact evaluation
// order: Rust never contracts a*b+c into an FMA and evaluates left to right, so this
// file must be compiled with -ffp-contract=off and without fast-math on x86-64 (SSE
// scalar float). Under those flags the f32 instantiation is bit-identical to the Rust
// code; it is pinned against the reference's own published CPU grid-table hashes
// (tests/golden/grid_hashes.json).
//
// Templated on the scalar type: R = float is the f32 restatement, R = double is the
// FP64 twin used to state the error of both the oracle and the CUDA path.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <limits>
#include <thread>
#include <vector>

namespace oracle {

// ---------------------------------------------------------------- math
// crates/vxl-phys-core/src/math.rs:8-75 (Vec3: component-wise ops, dot is
// ((x*ox + y*oy) + z*oz), cross as written there).
template <class R>
struct V3 {
  R x, y, z;
  V3() : x(0), y(0), z(0) {}
  V3(R a, R b, R c) : x(a), y(b), z(c) {}
  V3 operator+(const V3& o) const { return V3(x + o.x, y + o.y, z + o.z); }
  V3 operator-(const V3& o) const { return V3(x - o.x, y - o.y, z - o.z); }
  V3 operator*(R s) const { return V3(x * s, y * s, z * s); }
  V3& operator+=(const V3& o) { *this = *this + o; return *this; }
  V3& operator-=(const V3& o) { *this = *this - o; return *this; }
  V3& operator*=(R s) { *this = *this * s; return *this; }
  R dot(const V3& o) const { return x * o.x + y * o.y + z * o.z; }
  V3 cross(const V3& o) const {
    return V3(y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x);
  }
  R length_squared() const { return dot(*this); }
  R length() const { return std::sqrt(length_squared()); }
  // f32::min / f32::max are IEEE minNum/maxNum (NaN-ignoring) == fmin/fmax.
  V3 vmin(const V3& o) const { return V3(std::fmin(x, o.x), std::fmin(y, o.y), std::fmin(z, o.z)); }
  V3 vmax(const V3& o) const { return V3(std::fmax(x, o.x), std::fmax(y, o.y), std::fmax(z, o.z)); }
  R axis(int a) const { return a == 0 ? x : (a == 1 ? y : z); }
  void set_axis(int a, R v) {  // crates/vxl-phys-fluid/src/boundary.rs:198-204
    if (a == 0) x = v; else if (a == 1) y = v; else z = v;
  }
};

// crates/vxl-phys-core/src/math.rs (Quat::rotate_vec3): t = 2 (q x v); v + q x t + w t.
template <class R>
struct Quat {
  R x, y, z, w;
  Quat() : x(0), y(0), z(0), w(1) {}
  Quat(R a, R b, R c, R d) : x(a), y(b), z(c), w(d) {}
  V3<R> rotate(const V3<R>& v) const {
    V3<R> qv(x, y, z);
    V3<R> t = qv.cross(v) * R(2);
    return v + qv.cross(t) + t * w;
  }
};

// ---------------------------------------------------------------- rigid bodies (coupling loop)
// A dynamic body of the facade's coupling loop without contacts: pose, velocities and mass
// properties (crates/vxl-phys-core/src/body.rs).
template <class R>
struct RigidBody {
  V3<R> pos;
  Quat<R> rot;
  V3<R> linvel, angvel;
  R inv_mass;
  V3<R> local_inv_inertia;
  bool dynamic;
};

// crates/vxl-phys-core/src/mass.rs:35-48 (Shape::Box): m = rho ex ey ez, I = m/12 (..).
template <class R>
inline void box_mass_props(const V3<R>& half, R density, R& inv_mass, V3<R>& local_inv_inertia) {
  if (!(density > R(0))) density = R(1);
  R ex = R(2) * half.x, ey = R(2) * half.y, ez = R(2) * half.z;
  R m = density * ex * ey * ez;
  R ix = m / R(12) * (ey * ey + ez * ez);
  R iy = m / R(12) * (ex * ex + ez * ez);
  R iz = m / R(12) * (ex * ex + ey * ey);
  inv_mass = R(1) / m;
  local_inv_inertia = V3<R>(R(1) / ix, R(1) / iy, R(1) / iz);
}

// crates/vxl-phys-core/src/math.rs:241-252 (Hamilton product a * b).
template <class R>
inline Quat<R> qmul(const Quat<R>& a, const Quat<R>& b) {
  return Quat<R>(a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
                 a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z);
}

// crates/vxl-phys-core/src/math.rs:216-238 (normalize; integrate_angular with world w).
template <class R>
inline Quat<R> integrate_angular(const Quat<R>& q, const V3<R>& w, R dt) {
  Quat<R> dq = qmul(Quat<R>(w.x, w.y, w.z, R(0)), q);
  R hd = R(0.5) * dt;
  Quat<R> r(q.x + dq.x * hd, q.y + dq.y * hd, q.z + dq.z * hd, q.w + dq.w * hd);
  R len2 = r.x * r.x + r.y * r.y + r.z * r.z + r.w * r.w;
  if (len2 > R(1e-16)) {
    R inv = R(1) / std::sqrt(len2);
    return Quat<R>(r.x * inv, r.y * inv, r.z * inv, r.w * inv);
  }
  return Quat<R>();
}

// crates/vxl-phys-core/src/body.rs:172-176 with Mat3::from_quat / transpose_mul_vec3 /
// mul_vec3 (math.rs:275-311): R diag(d) R^T l.
template <class R>
inline V3<R> world_inv_inertia(const Quat<R>& q, const V3<R>& d, const V3<R>& l) {
  R xx = q.x * q.x, yy = q.y * q.y, zz = q.z * q.z;
  R xy = q.x * q.y, xz = q.x * q.z, yz = q.y * q.z;
  R wx = q.w * q.x, wy = q.w * q.y, wz = q.w * q.z;
  R m[3][3] = {{R(1) - R(2) * (yy + zz), R(2) * (xy - wz), R(2) * (xz + wy)},
               {R(2) * (xy + wz), R(1) - R(2) * (xx + zz), R(2) * (yz - wx)},
               {R(2) * (xz - wy), R(2) * (yz + wx), R(1) - R(2) * (xx + yy)}};
  V3<R> lt(m[0][0] * l.x + m[1][0] * l.y + m[2][0] * l.z, m[0][1] * l.x + m[1][1] * l.y + m[2][1] * l.z,
           m[0][2] * l.x + m[1][2] * l.y + m[2][2] * l.z);
  V3<R> v(lt.x * d.x, lt.y * d.y, lt.z * d.z);
  return V3<R>(m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z, m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z,
               m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z);
}

// One rigid substep of a dynamic, awake body with no contacts, as the facade runs it
// (crates/vxl-phys/src/world_step.rs:240-330): the gravity field adds g * (1 / inv_mass)
// (crates/vxl-phys-field/src/lib.rs:22-31), the fluid reaction pass adds the tick-averaged
// reaction (world_step.rs:235-255, coupling.rs:52-57), Integrator::integrate_velocities with
// gravity ZERO and its clamps, then integrate_positions (crates/vxl-phys-integrate/src/lib.rs:18-60).
template <class R>
inline void rigid_substep(RigidBody<R>& b, const V3<R>& g, const V3<R>& rf, const V3<R>& rt, R dt, R max_linear,
                          R max_angular) {
  if (!b.dynamic) return;
  V3<R> force = V3<R>() + g * (R(1) / b.inv_mass);
  V3<R> torque;
  force += rf;
  torque += rt;
  V3<R> accel = V3<R>() + force * b.inv_mass;
  b.linvel += accel * dt;
  V3<R> ang = world_inv_inertia(b.rot, b.local_inv_inertia, torque);
  b.angvel = b.angvel + ang * dt;
  R sp = b.linvel.length();
  if (sp > max_linear) b.linvel = b.linvel * (max_linear / sp);
  R ws = b.angvel.length();
  if (ws > max_angular) b.angvel = b.angvel * (max_angular / ws);
  b.pos = b.pos + b.linvel * dt;
  b.rot = integrate_angular(b.rot, b.angvel, dt);
}

// Rust `f32::powi` lowers to repeated squaring (LLVM ExpandPowI / compiler-rt
// __powisf2); both give r = a^(bits) multiplied in this order.
template <class R>
inline R powi(R a, int b) {
  bool recip = b < 0;
  R r = 1;
  for (;;) {
    if (b & 1) r *= a;
    b /= 2;
    if (b == 0) break;
    a *= a;
  }
  return recip ? R(1) / r : r;
}

template <class R> inline R pi_v();
template <> inline float pi_v<float>() { return 3.14159265358979323846f; }
template <> inline double pi_v<double>() { return 3.14159265358979323846; }

// Rust `x as u32` / `x as usize` from float: saturating, NaN -> 0.
template <class R>
inline uint64_t sat_u64(R v) {
  if (!(v > R(0))) return 0;  // NaN, negatives, -0
  if (v >= R(18446744073709551616.0)) return UINT64_MAX;
  return (uint64_t)v;
}
template <class R>
inline uint32_t sat_u32(R v) {
  if (!(v > R(0))) return 0;
  if (v >= R(4294967296.0)) return UINT32_MAX;
  return (uint32_t)v;
}

// ---------------------------------------------------------------- grid rule
// crates/vxl-phys-core/src/grid.rs:8,20
constexpr uint32_t GRID_DIM_MAX = 1u << 14;
constexpr uint64_t GRID_MAX_BINS = 1ull << 21;

template <class R>
struct GridBox {
  V3<R> min;
  R bin;
  uint32_t dims[3];
};

// crates/vxl-phys-core/src/grid.rs:34-50 (grid_box)
template <class R>
GridBox<R> grid_box(V3<R> lo, V3<R> hi, R h, uint64_t max_bins) {
  GridBox<R> g;
  R bin = std::fmax(h, R(1e-6f));
  V3<R> ext = hi - lo;
  R exts[3] = {ext.x, ext.y, ext.z};
  uint32_t dims[3] = {1, 1, 1};
  for (;;) {
    for (int a = 0; a < 3; ++a) {
      // ((ext/bin).floor() as usize + 1).clamp(1, GRID_DIM_MAX); `+ 1` wraps in release.
      uint64_t d = sat_u64(std::floor(exts[a] / bin)) + 1u;
      if (d < 1) d = 1;
      if (d > GRID_DIM_MAX) d = GRID_DIM_MAX;
      dims[a] = (uint32_t)d;
    }
    if ((uint64_t)dims[0] * dims[1] * dims[2] <= max_bins) break;
    bin *= R(2);
  }
  g.min = lo;
  g.bin = bin;
  g.dims[0] = dims[0]; g.dims[1] = dims[1]; g.dims[2] = dims[2];
  return g;
}

// crates/vxl-phys-fluid/src/grid.rs:12-155 (UniformGrid: counting sort + 27-cell walk)
template <class R>
struct UniformGrid {
  R bin = 0, inv = 0;
  V3<R> min;
  uint32_t nx = 0, ny = 0, nz = 0;
  std::vector<uint32_t> items, start, counts;

  // crates/vxl-phys-fluid/src/grid.rs:29-76
  void rebuild(const std::vector<V3<R>>& pos, R h, uint64_t max_bins) {
    size_t n = pos.size();
    if (n == 0) {
      nx = ny = nz = 0;
      items.clear();
      start.assign(1, 0);
      return;
    }
    V3<R> lo = pos[0], hi = pos[0];
    for (size_t i = 1; i < n; ++i) { lo = lo.vmin(pos[i]); hi = hi.vmax(pos[i]); }
    GridBox<R> g = grid_box(lo, hi, h, max_bins);
    bin = g.bin;
    inv = R(1) / bin;
    min = g.min;
    nx = g.dims[0]; ny = g.dims[1]; nz = g.dims[2];
    size_t total = (size_t)nx * ny * nz;
    counts.assign(total + 1, 0);
    for (size_t i = 0; i < n; ++i) counts[bin_index_of(pos[i], total) + 1] += 1;
    for (size_t c = 0; c < total; ++c) counts[c + 1] += counts[c];
    start = counts;
    items.assign(n, 0);
    for (size_t i = 0; i < n; ++i) {
      size_t c = bin_index_of(pos[i], total);
      items[counts[c]] = (uint32_t)i;
      counts[c] += 1;
    }
  }

  // crates/vxl-phys-fluid/src/grid.rs:79-100
  uint32_t axis_bin(R o, R v, uint32_t n) const {
    uint32_t b = sat_u32(std::fmax(std::floor((v - o) * inv), R(0)));
    return std::min(b, n - 1);
  }
  size_t bin_index_of(const V3<R>& p, size_t total) const {
    uint32_t idx = (axis_bin(min.x, p.x, nx) * ny + axis_bin(min.y, p.y, ny)) * nz +
                   axis_bin(min.z, p.z, nz);
    size_t cap = total == 0 ? 0 : total - 1;
    return std::min((size_t)idx, cap);
  }
  void bin_of(const V3<R>& p, uint32_t& cx, uint32_t& cy, uint32_t& cz) const {
    cx = axis_bin(min.x, p.x, nx);
    cy = axis_bin(min.y, p.y, ny);
    cz = axis_bin(min.z, p.z, nz);
  }

  // crates/vxl-phys-fluid/src/grid.rs:115-155 (dz outer, dy, dx inner; ascending items;
  // skip j == i; accept r2 <= h2 with r2 = |p_i - p_j|^2)
  template <class F>
  void for_neighbors_in(const std::vector<V3<R>>& pos, R h2, size_t i, F&& f) const {
    V3<R> pi = pos[i];
    uint32_t cx, cy, cz;
    bin_of(pi, cx, cy, cz);
    for (int dz = -1; dz <= 1; ++dz) {
      int z = (int)cz + dz;
      if (z < 0 || z >= (int)nz) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        int y = (int)cy + dy;
        if (y < 0 || y >= (int)ny) continue;
        for (int dx = -1; dx <= 1; ++dx) {
          int x = (int)cx + dx;
          if (x < 0 || x >= (int)nx) continue;
          size_t idx = ((size_t)x * ny + (size_t)y) * nz + (size_t)z;
          for (uint32_t k = start[idx]; k < start[idx + 1]; ++k) {
            size_t j = items[k];
            if (j == i) continue;
            V3<R> d = pi - pos[j];
            R r2 = d.length_squared();
            if (r2 <= h2) f(j, d, r2);
          }
        }
      }
    }
  }
};

// ---------------------------------------------------------------- config
// crates/vxl-phys-fluid/src/config.rs:6-68 (FluidConfig + Default)
template <class R>
struct FluidConfig {
  R rest_density = R(1000.0f);
  R smoothing_radius = R(0.1f);
  R xsph_viscosity = R(0.1f);
  bool tensile_instability_suppression = true;
  R sound_speed = R(10.0f);
  R gamma_tait = R(7.0f);
  uint32_t substeps = 4;
  uint32_t threads = 1;
  uint32_t boundary_layers = 2;
  V3<R> gravity = V3<R>(R(0), R(-9.81f), R(0));
  R max_speed_frac = R(0.4f);
  R artificial_viscosity = R(1.0f);
  uint64_t max_bins = GRID_MAX_BINS;  // crates/vxl-phys-core/src/grid.rs:20
};

// ---------------------------------------------------------------- boundary lattice
// crates/vxl-phys-fluid/src/boundary.rs (box family and sphere; the configs use boxes)
enum class ShapeKind : int { Box = 0, Sphere = 1 };

template <class R>
struct Shape {
  ShapeKind kind = ShapeKind::Box;
  V3<R> half;   // Box
  R radius = 0;  // Sphere
  bool operator==(const Shape& o) const {
    return kind == o.kind && half.x == o.half.x && half.y == o.half.y && half.z == o.half.z &&
           radius == o.radius;
  }
};

template <class R>
struct BoundaryLattice {
  std::vector<V3<R>> pts;
  size_t n0 = 0;
  R volume = 0;
};

// crates/vxl-phys-fluid/src/boundary.rs:190-194 (round half away from zero, >= 1)
template <class R>
inline size_t lattice_count(R len, R s) {
  double v = (double)std::round(len / s);
  int64_t c = (int64_t)v;
  return (size_t)std::max<int64_t>(c, 1);
}

// crates/vxl-phys-fluid/src/boundary.rs:208-232 (box_faces)
template <class R>
void box_faces(V3<R> half, R s, std::vector<V3<R>>& pts, std::vector<V3<R>>& nrm) {
  R h[3] = {half.x, half.y, half.z};
  for (int a = 0; a < 3; ++a) {
    int b = (a + 1) % 3, c = (a + 2) % 3;
    R hb = h[b], hc = h[c];
    size_t nb = lattice_count(R(2) * hb, s);
    size_t nc = lattice_count(R(2) * hc, s);
    R db = R(2) * hb / (R)nb;
    R dc = R(2) * hc / (R)nc;
    const R signs[2] = {R(1), R(-1)};
    for (R sign : signs) {
      for (size_t i = 0; i < nb; ++i) {
        for (size_t j = 0; j < nc; ++j) {
          V3<R> p, n;
          p.set_axis(a, sign * h[a]);
          n.set_axis(a, sign);
          p.set_axis(b, -hb + ((R)i + R(0.5f)) * db);
          p.set_axis(c, -hc + ((R)j + R(0.5f)) * dc);
          pts.push_back(p);
          nrm.push_back(n);
        }
      }
    }
  }
}

// crates/vxl-phys-fluid/src/boundary.rs:237-258 (sphere_shell, golden-angle spiral)
template <class R>
void sphere_shell(V3<R> center, R radius, R s, int hemi, std::vector<V3<R>>& pts,
                  std::vector<V3<R>>& nrm) {
  R area = (hemi == 0 ? R(4) : R(2)) * pi_v<R>() * radius * radius;
  size_t n = lattice_count(area, s * s);
  R ga = pi_v<R>() * (R(3) - std::sqrt(R(5)));
  for (size_t k = 0; k < n; ++k) {
    R y = R(1) - R(2) * ((R)k + R(0.5f)) / (R)n;
    bool keep = hemi == 0 ? true : (hemi == 1 ? y >= R(0) : y < R(0));
    if (!keep) continue;
    R r = std::sqrt(std::fmax(R(1) - y * y, R(0)));
    R th = ga * (R)k;
    R sn = std::sin(th), cs = std::cos(th);
    V3<R> nr(r * cs, y, r * sn);
    pts.push_back(center + nr * radius);
    nrm.push_back(nr);
  }
}

// crates/vxl-phys-fluid/src/boundary.rs:145-165 (min_half_extent)
template <class R>
R min_half_extent(const Shape<R>& sh) {
  if (sh.kind == ShapeKind::Box) return std::fmin(std::fmin(sh.half.x, sh.half.y), sh.half.z);
  return sh.radius;
}

// crates/vxl-phys-fluid/src/boundary.rs:104-129 (boundary_self_sum). The reference
// loops over all j in index order; only r2 <= h2 terms contribute, so summing the
// accepted j in ascending index order (found through a cell walk) is the same sum.
template <class R>
R boundary_self_sum(const std::vector<V3<R>>& pts, R h) {
  if (pts.empty()) return R(0);
  R h2 = h * h;
  R k6 = R(315.0f) / (R(64.0f) * pi_v<R>() * powi(h, 9));
  R w0 = k6 * h2 * h2 * h2;
  // cell walk for candidate collection (cell side h)
  V3<R> lo = pts[0], hi = pts[0];
  for (auto& p : pts) { lo = lo.vmin(p); hi = hi.vmax(p); }
  auto cell = [&](R v, R o, int64_t n) {
    int64_t c = (int64_t)std::floor((double)((v - o) / h));
    return std::min<int64_t>(std::max<int64_t>(c, 0), n - 1);
  };
  int64_t nx = std::max<int64_t>(1, (int64_t)std::floor((double)((hi.x - lo.x) / h)) + 1);
  int64_t ny = std::max<int64_t>(1, (int64_t)std::floor((double)((hi.y - lo.y) / h)) + 1);
  int64_t nz = std::max<int64_t>(1, (int64_t)std::floor((double)((hi.z - lo.z) / h)) + 1);
  std::vector<std::vector<uint32_t>> cells((size_t)(nx * ny * nz));
  for (size_t j = 0; j < pts.size(); ++j) {
    int64_t cx = cell(pts[j].x, lo.x, nx), cy = cell(pts[j].y, lo.y, ny), cz = cell(pts[j].z, lo.z, nz);
    cells[(size_t)((cx * ny + cy) * nz + cz)].push_back((uint32_t)j);
  }
  std::vector<R> per(pts.size());
  auto worker = [&](size_t b, size_t e) {
    std::vector<uint32_t> cand;
    for (size_t i = b; i < e; ++i) {
      const V3<R> pi = pts[i];
      int64_t cx = cell(pi.x, lo.x, nx), cy = cell(pi.y, lo.y, ny), cz = cell(pi.z, lo.z, nz);
      cand.clear();
      for (int64_t x = cx - 1; x <= cx + 1; ++x)
        for (int64_t y = cy - 1; y <= cy + 1; ++y)
          for (int64_t z = cz - 1; z <= cz + 1; ++z) {
            if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) continue;
            for (uint32_t j : cells[(size_t)((x * ny + y) * nz + z)]) cand.push_back(j);
          }
      std::sort(cand.begin(), cand.end());
      R sum = w0;
      for (uint32_t j : cand) {
        if (j == i) continue;
        R r2 = (pi - pts[j]).length_squared();
        if (r2 <= h2) {
          R t = h2 - r2;
          sum += k6 * t * t * t;
        }
      }
      per[i] = sum;
    }
  };
  size_t nthr = std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), 16));
  if (pts.size() < 4096) nthr = 1;
  std::vector<std::thread> th;
  size_t chunk = (pts.size() + nthr - 1) / nthr;
  for (size_t t = 0; t < nthr; ++t) {
    size_t b = t * chunk, e = std::min(pts.size(), b + chunk);
    if (b < e) th.emplace_back(worker, b, e);
  }
  for (auto& t : th) t.join();
  R acc = 0;
  for (size_t i = 0; i < pts.size(); ++i) acc += per[i];
  return acc / (R)pts.size();
}

// crates/vxl-phys-fluid/src/boundary.rs:95-102
template <class R>
R volume_from_self_sum(const std::vector<V3<R>>& pts, R h) {
  R sum = boundary_self_sum(pts, h);
  return sum > R(1e-12f) ? R(1) / sum : R(1);
}

// crates/vxl-phys-fluid/src/boundary.rs:67-88 (lattice)
template <class R>
BoundaryLattice<R> lattice(const Shape<R>& shape, R s, R h, uint32_t layers_in) {
  s = std::fmax(s, R(1e-6f));
  size_t layers = std::max<uint32_t>(layers_in, 1);
  std::vector<V3<R>> sp, sn;
  if (shape.kind == ShapeKind::Box) box_faces(shape.half, s, sp, sn);
  else sphere_shell(V3<R>(), shape.radius, s, 0, sp, sn);
  BoundaryLattice<R> out;
  out.n0 = sp.size();
  R hm = min_half_extent(shape);
  out.pts.reserve(out.n0 * layers);
  for (size_t k = 0; k < layers; ++k) {
    R want = ((R)k + R(0.5f)) * s;
    R cap = (R(0.45f) + R(0.45f) * (R)k) * hm;
    R d = std::fmax(std::fmin(std::fmin(want, cap), R(0.95f) * hm), R(1e-6f));
    for (size_t q = 0; q < sp.size(); ++q) out.pts.push_back(sp[q] - sn[q] * d);
  }
  out.volume = volume_from_self_sum(out.pts, std::fmax(h, s));
  return out;
}

template <class R>
struct BodyPose {
  V3<R> pos;
  Quat<R> rot;
  V3<R> linvel, angvel;
};

template <class R>
struct Body {
  uint32_t id;
  Shape<R> shape;
  BodyPose<R> pose;
};

template <class R>
struct Span {
  uint32_t body;
  V3<R> origin;
  uint32_t start, end;
};

template <class R>
struct Reaction {
  uint32_t body;
  V3<R> force, torque;
};

// ---------------------------------------------------------------- provider walls
// Analytic boundary providers (ProviderColliders, crates/vxl-phys-core/src/interop.rs:162-222)
// of two kinds, each restated from the reference implementation it follows:
//  - kFaces: independent axis-aligned half-space faces (the fluid crate's test providers
//    FloorY / Tank, crates/vxl-phys-fluid/src/tests.rs:9-110): a face (axis, plane, sign)
//    reports a contact when sdf = (p[axis] - plane) * sign <= 2 probe, at p with its axis
//    coordinate set to the plane, normal sign along the axis, depth probe - sdf.
//  - kConvex: a convex solid as an intersection of half-spaces n.x <= d (HalfSpaceSet,
//    crates/vxl-phys-terrain/src/plane_set.rs:60-76, 166-181): the decisive plane k maximises
//    s = n.x - d; a contact is reported when depth = -s >= -probe, at x - n (n.x - d).
// contacts_point_boundary is contacts_point for both (interop.rs:214-222).
template <class R>
struct Contact {
  V3<R> point, normal;
  R depth;
};

template <class R>
struct WallPlane {
  V3<R> n;       // kConvex: outward normal
  R d;           // kConvex: offset; kFaces: plane coordinate
  uint32_t axis; // kFaces
  R sign;        // kFaces: +1 / -1
};

template <class R>
struct Provider {
  enum : uint32_t { kFaces = 0, kConvex = 1 };
  uint32_t kind = kFaces;
  bool has_bounds = false;
  V3<R> bmin, bmax;
  std::vector<WallPlane<R>> planes;

  void contacts_point(const V3<R>& p, R probe, std::vector<Contact<R>>& out) const {
    if (kind == kFaces) {
      for (const auto& f : planes) {  // tests.rs:81-110
        R comp = p.axis((int)f.axis);
        R sdf = (comp - f.d) * f.sign;
        if (sdf > R(2) * probe) continue;
        V3<R> point = p;
        point.set_axis((int)f.axis, f.d);
        V3<R> normal;
        normal.set_axis((int)f.axis, f.sign);
        out.push_back(Contact<R>{point, normal, probe - sdf});
      }
      return;
    }
    if (planes.empty()) return;  // plane_set.rs:166-169
    R best = -std::numeric_limits<R>::infinity();
    size_t k = 0;
    for (size_t i = 0; i < planes.size(); ++i) {  // plane_set.rs:60-71 (signed)
      R s = planes[i].n.dot(p) - planes[i].d;
      if (s > best) { best = s; k = i; }
    }
    R depth = -best;
    if (depth < -probe) return;
    const auto& pl = planes[k];
    V3<R> point = p - pl.n * (pl.n.dot(p) - pl.d);  // plane_set.rs:74-76 (project)
    out.push_back(Contact<R>{point, pl.n, depth});
  }

  // Prefilter of the fluid passes: a provider with bounds is skipped when p lies outside
  // them expanded by m (fluid_density.rs:90-101, fluid_boundary.rs:60-71).
  bool outside(const V3<R>& p, R m) const {
    return has_bounds && (p.x < bmin.x - m || p.x > bmax.x + m || p.y < bmin.y - m || p.y > bmax.y + m ||
                          p.z < bmin.z - m || p.z > bmax.z + m);
  }
};

// Contact tables of the GPU tier's provider walls (crates/vxl-phys-gpu/src/pipeline/walls.rs:
// 143-215, WallStage::upload :100-121): the host gathers, once per tick, for each fluid
// particle the contacts of every ProviderColliders — of any kind, voxel, mesh or SDF —
// as (point, outward normal) planes, one table for the mirror ghosts (contacts_point,
// 0 < sdf < h) and one for the projection (contacts_point_boundary, sdf < h), at most 8
// per particle; the substeps of that tick read the tables instead of querying providers.
// Here a table acts as one more provider after the registered ones, queried by particle
// index: its contacts for particle i are the table's planes of i (no bounds prefilter).
template <class R>
struct ContactTable {
  std::vector<uint32_t> off;   // n_fluid + 1 offsets into pt / n (empty: no table)
  std::vector<V3<R>> pt, n;
  void contacts(size_t i, std::vector<Contact<R>>& out) const {
    if (off.empty() || i + 1 >= off.size()) return;
    for (uint32_t k = off[i]; k < off[i + 1]; ++k) out.push_back(Contact<R>{pt[k], n[k], R(0)});
  }
};

// ---------------------------------------------------------------- fluid system
// crates/vxl-phys-fluid/src/system.rs:5-51 (fields) and fluid_access.rs:7-76 (new)
template <class R>
struct FluidSystem {
  FluidConfig<R> cfg;
  R h, h2, k6, ks, w0, b_tait, mass, spacing;
  std::vector<V3<R>> pos, vel, acc, xsph, bforce;
  std::vector<R> dens, press, pmass;
  size_t n_fluid = 0;
  std::vector<Span<R>> spans;
  std::vector<Reaction<R>> breact;
  UniformGrid<R> grid;
  std::vector<std::pair<Shape<R>, BoundaryLattice<R>>> lattice_cache;
  std::vector<Provider<R>> providers;  // the registered boundaries, in order
  ContactTable<R> ctab[2];             // contact tables: [0] mirror, [1] projection
  bool walls() const { return !providers.empty() || !ctab[0].off.empty() || !ctab[1].off.empty(); }
  R skin;                              // fluid_access.rs:47 (0.15 h)

  // crates/vxl-phys-fluid/src/fluid_access.rs:7-76
  FluidSystem(const FluidConfig<R>& c, V3<R> origin, const size_t dims[3], R sp) : cfg(c) {
    h = std::fmax(cfg.smoothing_radius, R(1e-5f));
    h2 = h * h;
    k6 = R(315.0f) / (R(64.0f) * pi_v<R>() * powi(h, 9));
    ks = R(45.0f) / (pi_v<R>() * powi(h, 6));
    w0 = k6 * h2 * h2 * h2;
    b_tait = cfg.sound_speed * cfg.sound_speed * cfg.rest_density / cfg.gamma_tait;
    skin = R(0.15f) * h;
    size_t n = dims[0] * dims[1] * dims[2];
    pos.reserve(n);
    for (size_t i = 0; i < dims[0]; ++i)
      for (size_t j = 0; j < dims[1]; ++j)
        for (size_t k = 0; k < dims[2]; ++k)
          pos.push_back(V3<R>(origin.x + ((R)i + R(0.5f)) * sp, origin.y + ((R)j + R(0.5f)) * sp,
                              origin.z + ((R)k + R(0.5f)) * sp));
    mass = lattice_mass(cfg, sp);
    spacing = sp;
    n_fluid = n;
    vel.assign(n, V3<R>());
    dens.assign(n, R(0));
    press.assign(n, R(0));
    acc.assign(n, V3<R>());
    xsph.assign(n, V3<R>());
    pmass.assign(n, mass);
    bforce.assign(n, V3<R>());
  }

  // crates/vxl-phys-fluid/src/fluid_access.rs:27-42 (lattice mass calibration)
  static R lattice_mass(const FluidConfig<R>& c, R sp) {
    R hh = std::fmax(c.smoothing_radius, R(1e-5f));
    R hh2 = hh * hh;
    R kk6 = R(315.0f) / (R(64.0f) * pi_v<R>() * powi(hh, 9));
    R wsum = 0;
    int side = (int)std::ceil(hh / std::fmax(sp, R(1e-6f)));
    for (int i = -side; i <= side; ++i)
      for (int j = -side; j <= side; ++j)
        for (int k = -side; k <= side; ++k) {
          V3<R> d((R)i * sp, (R)j * sp, (R)k * sp);
          R r2 = d.length_squared();
          if (r2 <= hh2) {
            R t = hh2 - r2;
            wsum += kk6 * t * t * t;
          }
        }
    return c.rest_density / wsum;
  }

  size_t n_total() const { return pos.size(); }

  // crates/vxl-phys-fluid/src/fluid_step.rs:60-73 (truncate_to_fluid)
  void truncate_to_fluid() {
    size_t nf = n_fluid;
    pos.resize(nf); vel.resize(nf); dens.resize(nf); press.resize(nf);
    acc.resize(nf); xsph.resize(nf); pmass.resize(nf); bforce.resize(nf);
    spans.clear();
    breact.clear();
  }

  // crates/vxl-phys-fluid/src/fluid_step.rs:13-53 (set_boundary_particles)
  size_t set_boundary_particles(const std::vector<Body<R>>& bodies) {
    truncate_to_fluid();
    for (const auto& b : bodies) {
      int idx = -1;
      for (size_t q = 0; q < lattice_cache.size(); ++q)
        if (lattice_cache[q].first == b.shape) { idx = (int)q; break; }
      if (idx < 0) {
        BoundaryLattice<R> lat = lattice(b.shape, spacing, h, cfg.boundary_layers);
        if (lat.pts.empty()) continue;
        lattice_cache.emplace_back(b.shape, std::move(lat));
        idx = (int)lattice_cache.size() - 1;
      }
      const BoundaryLattice<R>& lat = lattice_cache[(size_t)idx].second;
      uint32_t st = (uint32_t)pos.size();
      for (const auto& lp : lat.pts) {
        V3<R> wp = b.pose.pos + b.pose.rot.rotate(lp);
        pos.push_back(wp);
        vel.push_back(b.pose.linvel + b.pose.angvel.cross(wp - b.pose.pos));
        pmass.push_back(cfg.rest_density * lat.volume);
        dens.push_back(R(0));
        press.push_back(R(0));
        acc.push_back(V3<R>());
        xsph.push_back(V3<R>());
      }
      uint32_t en = (uint32_t)pos.size();
      if (en > st) spans.push_back(Span<R>{b.id, b.pose.pos, st, en});
    }
    bforce.resize(pos.size(), V3<R>());
    breact.clear();
    return pos.size() - n_fluid;
  }

  // crates/vxl-phys-fluid/src/fluid_step.rs:75-89 (step: C2 tick-average reactions)
  void step(R dt_tick) {
    uint32_t sub = std::max<uint32_t>(cfg.substeps, 1);
    R dt = dt_tick / (R)sub;
    breact.clear();
    for (uint32_t s = 0; s < sub; ++s) substep(dt);
    if (sub > 1) {
      R inv = R(1) / (R)sub;
      for (auto& e : breact) { e.force *= inv; e.torque *= inv; }
    }
  }

  // crates/vxl-phys-fluid/src/fluid_step.rs:91-127 (substep)
  void substep(R dt) {
    size_t nf = n_fluid;
    if (nf == 0) return;
    grid.rebuild(pos, h, cfg.max_bins);
    density_pass();
    pressure_pass();
    force_pass();
    integrate(dt);
    boundary_pass();
  }

  // crates/vxl-phys-fluid/src/fluid_density.rs:76-118 (wall_planes_in): the provider
  // planes within h of a fluid particle (contact point + outward normal, 0 < sdf < h), <= 8.
  size_t wall_planes(size_t i, const V3<R>& pi, V3<R> pl_pt[8], V3<R> pl_n[8]) const {
    size_t np = 0;
    std::vector<Contact<R>> scratch;
    auto take = [&]() {
      for (const auto& c : scratch) {
        R sdf = (pi - c.point).dot(c.normal);
        if (sdf > R(0) && sdf < h && np < 8) {
          pl_pt[np] = c.point;
          pl_n[np] = c.normal;
          ++np;
        }
      }
    };
    for (const auto& pr : providers) {
      if (pr.outside(pi, h)) continue;
      scratch.clear();
      pr.contacts_point(pi, h, scratch);
      take();
    }
    scratch.clear();
    ctab[0].contacts(i, scratch);  // the mirror table (contacts_point, gathered per tick)
    take();
    return np;
  }

  // crates/vxl-phys-fluid/src/fluid_boundary.rs:45-101 (boundary_pass): fluid particles
  // inside a provider are pushed out along each contact normal by min(pen + skin, h), their
  // inward normal velocity removed; the pushed ones then go through separate_coincident.
  void boundary_pass() {
    if (providers.empty() && ctab[1].off.empty()) return;
    std::vector<std::pair<size_t, V3<R>>> pushed;
    std::vector<Contact<R>> contacts;
    for (size_t i = 0; i < n_fluid; ++i) {
      V3<R> pi = pos[i];
      V3<R> p = pi, v = vel[i], n_sum;
      bool hit = false;
      auto apply = [&]() {
        for (const auto& c : contacts) {
          R sdf = (pi - c.point).dot(c.normal);
          R pen = -sdf;
          if (pen <= R(0)) continue;
          p += c.normal * std::fmin(pen + skin, h);
          n_sum += c.normal;
          hit = true;
          R vn = v.dot(c.normal);
          if (vn < R(0)) v -= c.normal * vn;
        }
        pos[i] = p;
        vel[i] = v;
      };
      for (const auto& pr : providers) {
        if (pr.outside(pi, h)) continue;
        contacts.clear();
        pr.contacts_point(pi, skin, contacts);  // contacts_point_boundary
        apply();
      }
      if (!ctab[1].off.empty()) {  // the projection table (contacts_point_boundary, gathered per tick)
        contacts.clear();
        ctab[1].contacts(i, contacts);
        apply();
      }
      if (hit) pushed.emplace_back(i, n_sum);
    }
    separate_coincident(pushed);
  }

  // crates/vxl-phys-fluid/src/fluid_boundary.rs:103-128: among the particles pushed this
  // substep, in ascending index, each one closer than 0.2 h to an earlier one moves along
  // its normal sum until r_min apart.
  void separate_coincident(const std::vector<std::pair<size_t, V3<R>>>& pushed) {
    R r_min = R(0.2f) * h;
    for (size_t a = 0; a < pushed.size(); ++a) {
      size_t ia = pushed[a].first;
      V3<R> na = pushed[a].second;
      R nl = na.length();
      if (nl <= R(1e-9f)) continue;
      V3<R> dir = na * (R(1) / nl);
      V3<R> pa = pos[ia];
      for (size_t b = 0; b < a; ++b) {
        V3<R> d = pa - pos[pushed[b].first];
        R r2 = d.length_squared();
        if (r2 < r_min * r_min) {
          R r = std::sqrt(r2);
          pa += dir * (r_min - r);
        }
      }
      pos[ia] = pa;
    }
  }

  // crates/vxl-phys-fluid/src/fluid_step.rs:112-123
  void integrate(R dt) {
    size_t nf = n_fluid;
    R vmax = cfg.max_speed_frac * h / dt;
    R vmax2 = vmax * vmax;
    R eps = cfg.xsph_viscosity;
    for (size_t i = 0; i < nf; ++i) {
      V3<R> v = vel[i] + acc[i] * dt + xsph[i] * eps;
      R s2 = v.length_squared();
      if (s2 > vmax2) v *= vmax / std::sqrt(s2);
      vel[i] = v;
      pos[i] += v * dt;
    }
  }

  template <class F>
  void for_neighbors(size_t i, F&& f) const {
    grid.for_neighbors_in(pos, h2, i, f);
  }

  template <class Fn>
  void parallel_for(size_t b, size_t e, Fn&& fn) const {
    size_t threads = std::max<uint32_t>(cfg.threads, 1);
    if (threads <= 1 || e - b < 2) { fn(b, e); return; }
    // crates/vxl-phys-fluid/src/fluid_density.rs:141 (per = n.div_ceil(threads).max(1))
    size_t n = e - b;
    size_t per = std::max<size_t>((n + threads - 1) / threads, 1);
    std::vector<std::thread> th;
    for (size_t s = b; s < e; s += per) th.emplace_back(fn, s, std::min(e, s + per));
    for (auto& t : th) t.join();
  }

  // crates/vxl-phys-fluid/src/fluid_density.rs:17-70 (serial) and :123-233 (parallel;
  // bit-identical since each particle's walk order is unchanged). Each neighbour's term is
  // followed by its mirror ghosts in the particle's provider planes (fluid_density.rs:38-47).
  void density_pass() {
    size_t nf = n_fluid, nt = pos.size();
    parallel_for(0, nf, [&](size_t b, size_t e) {
      V3<R> pl_pt[8], pl_n[8];
      for (size_t i = b; i < e; ++i) {
        V3<R> pi = pos[i];
        size_t np = walls() ? wall_planes(i, pi, pl_pt, pl_n) : 0;
        R sum = w0, sum_b = R(0);
        for_neighbors(i, [&](size_t j, const V3<R>& d, R r2) {
          R t = h2 - r2;
          R w = k6 * t * t * t;
          if (j < nf) sum += w;
          else sum_b += pmass[j] * w;
          for (size_t k = 0; k < np; ++k) {
            V3<R> pj = pi - d;
            R dn = (pj - pl_pt[k]).dot(pl_n[k]);
            V3<R> g = pj - pl_n[k] * (R(2) * dn);
            R rg2 = (pi - g).length_squared();
            if (rg2 <= h2) {
              R tg = h2 - rg2;
              sum += k6 * tg * tg * tg;
            }
          }
        });
        dens[i] = mass * sum + sum_b;
      }
    });
    parallel_for(nf, nt, [&](size_t b, size_t e) {
      for (size_t i = b; i < e; ++i) {
        R sum = R(0);
        for_neighbors(i, [&](size_t j, const V3<R>&, R r2) {
          if (j >= nf) return;
          R t = h2 - r2;
          sum += pmass[j] * (k6 * t * t * t);
        });
        dens[i] = pmass[i] * w0 + sum;
      }
    });
  }

  // crates/vxl-phys-fluid/src/fluid_force.rs:11-29 (Tait EOS; gamma == 7 expands q^7)
  static R tait(R dens, R rho0, R g, R b_tait, bool clamp) {
    R q = dens / rho0;
    R p;
    if (std::fabs(g - R(7.0f)) < R(1e-6f)) {
      R q2 = q * q;
      R q4 = q2 * q2;
      p = b_tait * (q * q2 * q4 - R(1));
    } else {
      p = b_tait * (std::pow(q, g) - R(1));
    }
    if (clamp && p < R(0)) p = R(0);
    return p;
  }
  void pressure_pass() {
    for (size_t i = 0; i < pos.size(); ++i)
      press[i] = tait(dens[i], cfg.rest_density, cfg.gamma_tait, b_tait,
                      cfg.tensile_instability_suppression);
  }

  // crates/vxl-phys-fluid/src/fluid_force.rs:165-217 (serial) and :52-162 (parallel;
  // acc/xsph per particle, bforce by a serial make-up pass in the same order)
  void force_pass() {
    size_t nf = n_fluid, nt = pos.size();
    V3<R> g = cfg.gravity;
    R alpha_c = cfg.artificial_viscosity * cfg.sound_speed;
    for (size_t j = nf; j < nt; ++j) bforce[j] = V3<R>();
    bool serial_bforce = cfg.threads <= 1;
    parallel_for(0, nf, [&](size_t b, size_t e) {
      for (size_t i = b; i < e; ++i) {
        V3<R> vi = vel[i];
        R rho_i = dens[i];
        R ci2 = press[i] / (rho_i * rho_i);
        R mi = pmass[i];
        V3<R> a = g, xs;
        for_neighbors(i, [&](size_t j, const V3<R>& d, R r2) {
          R rho_j = dens[j];
          R cj2 = press[j] / (rho_j * rho_j);
          R r = std::sqrt(r2);
          R t = h - r;
          R mj = pmass[j];
          R coef = mj * (ks * t * t) * (ci2 + cj2);
          R denom = std::fmax(r, R(1e-9f));
          a += d * (coef / denom);
          V3<R> vij = vi - vel[j];
          R vdn = -vij.dot(d);
          R cv = R(0);
          if (vdn > R(0)) {
            R mu = vdn * h / (r2 + R(0.01f) * h2);
            R c = mj * (alpha_c * mu / (R(0.5f) * (rho_i + rho_j))) * (ks * t * t);
            a += d * (c / denom);
            cv = c;
          }
          if (serial_bforce && j >= nf) bforce[j] -= d * (mi * (coef + cv) / denom);
          R tt = h2 - r2;
          R w = k6 * tt * tt * tt;
          xs += (vel[j] - vi) * (mj * R(2.0f) / (rho_i + rho_j) * w);
        });
        acc[i] = a;
        xsph[i] = xs;
      }
    });
    if (!serial_bforce && nt > nf) {
      for (size_t i = 0; i < nf; ++i) {
        V3<R> vi = vel[i];
        R rho_i = dens[i];
        R ci2 = press[i] / (rho_i * rho_i);
        R mi = pmass[i];
        for_neighbors(i, [&](size_t j, const V3<R>& d, R r2) {
          if (j < nf) return;
          R rho_j = dens[j];
          R cj2 = press[j] / (rho_j * rho_j);
          R r = std::sqrt(r2);
          R t = h - r;
          R mj = pmass[j];
          R coef = mj * (ks * t * t) * (ci2 + cj2);
          R denom = std::fmax(r, R(1e-9f));
          R cv = R(0);
          V3<R> vij = vi - vel[j];
          R vdn = -vij.dot(d);
          if (vdn > R(0)) {
            R mu = vdn * h / (r2 + R(0.01f) * h2);
            cv = mj * (alpha_c * mu / (R(0.5f) * (rho_i + rho_j))) * (ks * t * t);
          }
          bforce[j] -= d * (mi * (coef + cv) / denom);
        });
      }
    }
    aggregate_reactions();
  }

  // crates/vxl-phys-fluid/src/fluid_boundary.rs:10-28 (per-span F and torque about the
  // body origin, summed in index order, accumulated into the tick accumulator)
  void aggregate_reactions() {
    for (size_t si = 0; si < spans.size(); ++si) {
      const Span<R>& sp = spans[si];
      V3<R> f, tau;
      for (uint32_t k = sp.start; k < sp.end; ++k) {
        V3<R> fk = bforce[k];
        f += fk;
        tau += (pos[k] - sp.origin).cross(fk);
      }
      if (si < breact.size()) {
        if (breact[si].body == sp.body) { breact[si].force += f; breact[si].torque += tau; }
        else breact[si] = Reaction<R>{sp.body, f, tau};
      } else {
        breact.push_back(Reaction<R>{sp.body, f, tau});
      }
    }
  }
};

// FNV-1a table hash used by the reference's grid probe
// (crates/vxl-phys-gpu/examples/gpu_grid_probe.rs:50-67): start, 0xffffffff, items,
// 0xffffffff, per-particle bin recovered from the table (bins_from_table, :37-46).
inline uint64_t table_hash(const std::vector<uint32_t>& start, const std::vector<uint32_t>& items,
                           size_t total, size_t np) {
  std::vector<uint32_t> bins(np, UINT32_MAX);
  for (size_t c = 0; c < total; ++c)
    for (uint32_t k = start[c]; k < start[c + 1]; ++k) bins[items[k]] = (uint32_t)c;
  uint64_t h = 0xcbf29ce484222325ull;
  auto fnv = [&](uint32_t v) { h ^= (uint64_t)v; h *= 0x00000100000001b3ull; };
  for (uint32_t v : start) fnv(v);
  fnv(0xffffffffu);
  for (uint32_t v : items) fnv(v);
  fnv(0xffffffffu);
  for (uint32_t v : bins) fnv(v);
  return h;
}

}  // namespace oracle
