// Host-side set-up of a WCSPH scene: the fluid particle mass calibration and the
// Akinci boundary-particle lattice of a body shape. These run once per scene (or once
// per shape, the reference caches lattices per shape: crates/vxl-phys-fluid/src/
// fluid_step.rs:33-47), not per substep.
//
// f32 arithmetic follows the reference's operation order; the file is compiled with
// -ffp-contract=off so every product is rounded before its sum, as in Rust.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

#include "vxl_sph.h"
#include "vxl_sph_internal.h"

namespace {

constexpr float kPi = 3.14159265358979323846f;

struct P3 {
  float v[3];
};

inline float len2(float x, float y, float z) { return x * x + y * y + z * z; }

// poly6 normalisation 315 / (64 pi h^9): crates/vxl-phys-fluid/src/fluid_access.rs:10.
inline float poly6_norm(float h) { return 315.0f / (64.0f * kPi * vxl_powi(h, 9)); }

// Cells per face edge: round(len / s) clamped to >= 1
// (crates/vxl-phys-fluid/src/boundary.rs:190-194).
inline int64_t edge_cells(float len, float s) {
  int64_t c = (int64_t)std::round(len / s);
  return c < 1 ? 1 : c;
}

// Six faces, each a grid of cell centres, outward normals
// (crates/vxl-phys-fluid/src/boundary.rs:208-232): face order a = x, y, z; sign +, -.
void box_surface(const float half[3], float s, std::vector<P3>& pts, std::vector<P3>& nrm) {
  for (int a = 0; a < 3; ++a) {
    const int b = (a + 1) % 3, c = (a + 2) % 3;
    const int64_t nb = edge_cells(2.0f * half[b], s), nc = edge_cells(2.0f * half[c], s);
    const float db = 2.0f * half[b] / (float)nb, dc = 2.0f * half[c] / (float)nc;
    for (float sign : {1.0f, -1.0f}) {
      for (int64_t i = 0; i < nb; ++i) {
        const float pb = -half[b] + ((float)i + 0.5f) * db;
        for (int64_t j = 0; j < nc; ++j) {
          P3 p{{0.0f, 0.0f, 0.0f}}, n{{0.0f, 0.0f, 0.0f}};
          p.v[a] = sign * half[a];
          n.v[a] = sign;
          p.v[b] = pb;
          p.v[c] = -half[c] + ((float)j + 0.5f) * dc;
          pts.push_back(p);
          nrm.push_back(n);
        }
      }
    }
  }
}

// Golden-angle sphere (crates/vxl-phys-fluid/src/boundary.rs:237-258), whole sphere.
void sphere_surface(float radius, float s, std::vector<P3>& pts, std::vector<P3>& nrm) {
  const float area = 4.0f * kPi * radius * radius;
  const int64_t n = edge_cells(area, s * s);
  const float ga = kPi * (3.0f - std::sqrt(5.0f));
  for (int64_t k = 0; k < n; ++k) {
    const float y = 1.0f - 2.0f * ((float)k + 0.5f) / (float)n;
    const float r = std::sqrt(std::fmax(1.0f - y * y, 0.0f));
    const float th = ga * (float)k;
    const float sn = std::sin(th), cs = std::cos(th);
    P3 nr{{r * cs, y, r * sn}};
    // centre (origin) + normal * radius, kept as an explicit add so signed zeros match
    pts.push_back(P3{{0.0f + nr.v[0] * radius, 0.0f + nr.v[1] * radius, 0.0f + nr.v[2] * radius}});
    nrm.push_back(nr);
  }
}

// Mean over particles of (W(0) + sum_{j != i, r <= h} W(r_ij)), each inner sum in
// ascending j (crates/vxl-phys-fluid/src/boundary.rs:104-129). Candidates come from a
// bucket grid and are visited in ascending index, so the sum is the same as the
// reference's all-pairs loop (pairs beyond h add nothing).
float self_sum(const std::vector<P3>& pts, float h) {
  const size_t n = pts.size();
  if (n == 0) return 0.0f;
  const float h2 = h * h;
  const float k6 = poly6_norm(h);
  const float w0 = k6 * h2 * h2 * h2;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (const P3& p : pts)
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], (double)p.v[a]);
      hi[a] = std::max(hi[a], (double)p.v[a]);
    }
  const double side = (double)h * 1.0001;  // a pair within h never skips a bucket
  int64_t dim[3];
  for (int a = 0; a < 3; ++a) dim[a] = std::max<int64_t>(1, (int64_t)std::floor((hi[a] - lo[a]) / side) + 1);
  auto bucket_of = [&](const P3& p, int64_t c[3]) {
    for (int a = 0; a < 3; ++a) {
      int64_t q = (int64_t)std::floor(((double)p.v[a] - lo[a]) / side);
      c[a] = std::min(std::max<int64_t>(q, 0), dim[a] - 1);
    }
  };
  // bucket -> ascending particle indices (counting sort)
  const size_t nbk = (size_t)(dim[0] * dim[1] * dim[2]);
  std::vector<uint32_t> first(nbk + 1, 0), ids(n);
  std::vector<uint32_t> key(n);
  for (size_t i = 0; i < n; ++i) {
    int64_t c[3];
    bucket_of(pts[i], c);
    key[i] = (uint32_t)((c[0] * dim[1] + c[1]) * dim[2] + c[2]);
    first[key[i] + 1]++;
  }
  for (size_t b = 0; b < nbk; ++b) first[b + 1] += first[b];
  {
    std::vector<uint32_t> cur(first.begin(), first.end() - 1);
    for (size_t i = 0; i < n; ++i) ids[cur[key[i]]++] = (uint32_t)i;
  }
  std::vector<float> row(n);
  auto work = [&](size_t b0, size_t b1) {
    std::vector<uint32_t> cand;
    for (size_t i = b0; i < b1; ++i) {
      int64_t c[3];
      bucket_of(pts[i], c);
      cand.clear();
      for (int64_t x = std::max<int64_t>(c[0] - 1, 0); x <= std::min(c[0] + 1, dim[0] - 1); ++x)
        for (int64_t y = std::max<int64_t>(c[1] - 1, 0); y <= std::min(c[1] + 1, dim[1] - 1); ++y)
          for (int64_t z = std::max<int64_t>(c[2] - 1, 0); z <= std::min(c[2] + 1, dim[2] - 1); ++z) {
            size_t bk = (size_t)((x * dim[1] + y) * dim[2] + z);
            cand.insert(cand.end(), ids.begin() + first[bk], ids.begin() + first[bk + 1]);
          }
      std::sort(cand.begin(), cand.end());
      float sum = w0;
      const P3& pi = pts[i];
      for (uint32_t j : cand) {
        if (j == i) continue;
        const P3& pj = pts[j];
        float r2 = len2(pi.v[0] - pj.v[0], pi.v[1] - pj.v[1], pi.v[2] - pj.v[2]);
        if (r2 <= h2) {
          float t = h2 - r2;
          sum += k6 * t * t * t;
        }
      }
      row[i] = sum;
    }
  };
  unsigned nth = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  if (n < 2048) nth = 1;
  std::vector<std::thread> pool;
  const size_t chunk = (n + nth - 1) / nth;
  for (unsigned t = 0; t < nth; ++t) {
    size_t b0 = t * chunk, b1 = std::min(n, b0 + chunk);
    if (b0 < b1) pool.emplace_back(work, b0, b1);
  }
  for (auto& t : pool) t.join();
  float acc = 0.0f;
  for (size_t i = 0; i < n; ++i) acc += row[i];
  return acc / (float)n;
}

}  // namespace

extern "C" {

// crates/vxl-phys-fluid/src/fluid_access.rs:27-42.
vxl_status vxl_sph_lattice_mass(const vxl_sph_params* params, float spacing, float* out_mass) {
  if (!params || !out_mass) return VXL_NULL_POINTER;
  const float h = std::fmax(params->smoothing_radius, 1e-5f);
  const float h2 = h * h;
  const float k6 = poly6_norm(h);
  const int side = (int)std::ceil(h / std::fmax(spacing, 1e-6f));
  float wsum = 0.0f;
  for (int i = -side; i <= side; ++i)
    for (int j = -side; j <= side; ++j)
      for (int k = -side; k <= side; ++k) {
        const float r2 = len2((float)i * spacing, (float)j * spacing, (float)k * spacing);
        if (r2 <= h2) {
          const float t = h2 - r2;
          wsum += k6 * t * t * t;
        }
      }
  *out_mass = params->rest_density / wsum;
  return VXL_OK;
}

// crates/vxl-phys-fluid/src/boundary.rs:67-88 (lattice): surface samples moved inward
// along the normal by d_k = max(min((k+1/2)s, (0.45+0.45k) half_min, 0.95 half_min), 1e-6)
// per layer, layer-major; per-particle volume 1 / mean self sum at radius max(h, s).
vxl_status vxl_sph_boundary_lattice(uint32_t shape, const float half[3], float radius, float spacing, float h,
                                    uint32_t layers, float* out_pts_xyz, uint64_t cap, uint64_t* out_count,
                                    float* out_volume) {
  if (!out_count) return VXL_NULL_POINTER;
  if (shape > 1) return VXL_INVALID_ARGUMENT;
  if (shape == 0 && !half) return VXL_NULL_POINTER;
  const float s = std::fmax(spacing, 1e-6f);
  const uint32_t nl = layers < 1 ? 1 : layers;
  std::vector<P3> sp, sn;
  float half_min;
  if (shape == 0) {
    box_surface(half, s, sp, sn);
    half_min = std::fmin(std::fmin(half[0], half[1]), half[2]);
  } else {
    sphere_surface(radius, s, sp, sn);
    half_min = radius;
  }
  std::vector<P3> pts;
  pts.reserve(sp.size() * nl);
  for (uint32_t k = 0; k < nl; ++k) {
    const float want = ((float)k + 0.5f) * s;
    const float cap_k = (0.45f + 0.45f * (float)k) * half_min;
    const float d = std::fmax(std::fmin(std::fmin(want, cap_k), 0.95f * half_min), 1e-6f);
    for (size_t q = 0; q < sp.size(); ++q)
      pts.push_back(P3{{sp[q].v[0] - sn[q].v[0] * d, sp[q].v[1] - sn[q].v[1] * d, sp[q].v[2] - sn[q].v[2] * d}});
  }
  *out_count = pts.size();
  if (out_volume) {
    const float sum = self_sum(pts, std::fmax(h, s));
    *out_volume = sum > 1e-12f ? 1.0f / sum : 1.0f;
  }
  if (out_pts_xyz && cap >= pts.size())
    for (size_t i = 0; i < pts.size(); ++i)
      for (int a = 0; a < 3; ++a) out_pts_xyz[3 * i + a] = pts[i].v[a];
  return VXL_OK;
}

}  // extern "C"
