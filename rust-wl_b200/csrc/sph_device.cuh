// Device-side building blocks of the WCSPH step for sm_100a.
//
// Arithmetic contract: this file is compiled with -fmad=false (no FMA contraction),
// IEEE division and square root (-prec-div=true -prec-sqrt=true) and no flush to zero,
// and every expression keeps the reference's evaluation order, so results are
// bit-identical to the reference's Rust f32 CPU path
// (crates/vxl-phys-fluid/src/fluid_density.rs, fluid_force.rs, fluid_step.rs).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace vxl {

constexpr uint32_t kGridDimMax = 1u << 14;   // crates/vxl-phys-core/src/grid.rs:8
constexpr uint32_t kErrGridLoop = 1u << 0;    // grid-box doubling loop did not settle
constexpr uint32_t kErrCanonLarge = 1u << 2;  // a cell above the shared-memory sort size (info)

// Grid box of one substep: crates/vxl-phys-core/src/grid.rs:34-50 (min, bin, dims)
// plus inv = 1 / bin (crates/vxl-phys-fluid/src/grid.rs:50).
struct GridBox {
  float minx, miny, minz, inv;
  float bin;
  uint32_t nx, ny, nz;
  uint32_t total;
  uint32_t pad[3];
};

// Constants of one scene, computed on the host exactly as FluidSystem::new does
// (crates/vxl-phys-fluid/src/fluid_access.rs:8-13).
struct SphConst {
  float h, h2, k6, ks, w0, b_tait, mass, rho0;
  float gamma, eps, alpha_c, h001;  // h001 = 0.01 * h2 (fluid_force.rs:197)
  float gx, gy, gz;
  uint32_t clamp_p, gamma7;
  uint32_t n_fluid, n_total, max_bins;
};

// Ordered-uint encoding of floats: monotone, so atomicMin/atomicMax on the code give
// exact float min/max independent of order.
__device__ __forceinline__ uint32_t f2o(float f) {
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t o) {
  uint32_t u = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
  return __uint_as_float(u);
}

// `((v - o) * inv).floor().max(0.0) as u32).min(n - 1)`: crates/vxl-phys-fluid/src/grid.rs:79-100.
__device__ __forceinline__ uint32_t axis_bin(float o, float v, float inv, uint32_t n) {
  float f = fmaxf(floorf((v - o) * inv), 0.0f);
  uint32_t b = (f >= 4294967296.0f) ? 0xffffffffu : (uint32_t)f;
  return min(b, n - 1u);
}

__device__ __forceinline__ void bin_of(const GridBox& g, float x, float y, float z, uint32_t& cx,
                                       uint32_t& cy, uint32_t& cz) {
  cx = axis_bin(g.minx, x, g.inv, g.nx);
  cy = axis_bin(g.miny, y, g.inv, g.ny);
  cz = axis_bin(g.minz, z, g.inv, g.nz);
}

__device__ __forceinline__ uint32_t cell_index(const GridBox& g, float x, float y, float z) {
  uint32_t cx, cy, cz;
  bin_of(g, x, y, z, cx, cy, cz);
  uint32_t idx = (cx * g.ny + cy) * g.nz + cz;
  return min(idx, g.total - 1u);
}

// Tait EOS with the free-surface clamp: crates/vxl-phys-fluid/src/fluid_force.rs:11-29.
__device__ __forceinline__ float tait(const SphConst& k, float rho) {
  float q = rho / k.rho0;
  float p;
  if (k.gamma7) {
    float q2 = q * q;
    float q4 = q2 * q2;
    p = k.b_tait * (q * q2 * q4 - 1.0f);
  } else {
    p = k.b_tait * (powf(q, k.gamma) - 1.0f);
  }
  if (k.clamp_p && p < 0.0f) p = 0.0f;
  return p;
}

// crates/vxl-phys-core/src/grid.rs:34-50 on the device (same f32 operations).
__device__ inline bool grid_box(float lox, float loy, float loz, float hix, float hiy, float hiz, float h,
                                uint32_t max_bins, GridBox& g) {
  float bin = fmaxf(h, 1e-6f);
  float ext[3] = {hix - lox, hiy - loy, hiz - loz};
  uint32_t dims[3] = {1, 1, 1};
  bool ok = false;
  for (int it = 0; it < 512; ++it) {
    for (int a = 0; a < 3; ++a) {
      float f = floorf(ext[a] / bin);
      unsigned long long d;
      if (!(f > 0.0f)) d = 0ull;
      else if (f >= 18446744073709551616.0f) d = ~0ull;
      else d = (unsigned long long)f;
      d += 1ull;  // wraps like the reference's release build
      if (d < 1ull) d = 1ull;
      if (d > kGridDimMax) d = kGridDimMax;
      dims[a] = (uint32_t)d;
    }
    if ((unsigned long long)dims[0] * dims[1] * dims[2] <= (unsigned long long)max_bins) {
      ok = true;
      break;
    }
    bin *= 2.0f;
  }
  g.minx = lox;
  g.miny = loy;
  g.minz = loz;
  g.bin = bin;
  g.inv = 1.0f / bin;
  g.nx = dims[0];
  g.ny = dims[1];
  g.nz = dims[2];
  g.total = dims[0] * dims[1] * dims[2];
  return ok;
}

}  // namespace vxl
