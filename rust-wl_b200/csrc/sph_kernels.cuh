// Kernels of one WCSPH substep on a resident, cell-sorted particle set (sm_100a).
//
// Resident layout (structure of arrays, one entry per particle slot):
//   pos[s]  float4 (x, y, z, m)   m = +particle mass for fluid, -pmass for boundary
//   vel[s]  float4 (vx, vy, vz, 0)
//   orig[s] reference index of the particle in slot s; slot_of[orig[s]] == s
// Slots are ordered by (cell, reference index) after every sort, which is exactly the
// reference's counting-sort table order (crates/vxl-phys-fluid/src/grid.rs:29-76):
// cell c holds slots [start[c], start[c+1]) in ascending reference index. Walking the
// 27 cells in the reference's (dz, dy, dx) order over these slot ranges therefore
// visits neighbours in the same order as UniformGrid::for_neighbors_in
// (grid.rs:115-155), and every per-particle sum matches the CPU bit for bit.
//
// Per substep: gridbox -> keys -> scan (3 kernels) -> place -> canon (sort + gather
// into the second buffer) -> density+EOS -> force+XSPH+integrate (back into the first
// buffer) -> boundary reaction gather -> per-span reduction.
#pragma once

#include "sph_device.cuh"

namespace vxl {
namespace {

constexpr int kScanTile = 2048;   // cells per scan block (256 threads x 8)
constexpr int kScanThreads = 256;
constexpr int kCanonSmem = 1024;  // per-warp shared keys for cells of <= 1024 particles
constexpr int kBGatherCap = 64;   // fluid neighbours a boundary particle sorts in registers/local

// Block-level ordered-uint min/max of (x, y, z) then one atomic per component.
__device__ __forceinline__ void block_bbox_accumulate(uint32_t* acc, float x, float y, float z, bool valid) {
  uint32_t mn[3], mx[3];
  float v[3] = {x, y, z};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    bool ok = valid && (v[a] == v[a]);  // NaN never wins (Rust f32::min/max ignore NaN)
    mn[a] = ok ? f2o(v[a]) : 0xffffffffu;
    mx[a] = ok ? f2o(v[a]) : 0u;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      mn[a] = min(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], off));
      mx[a] = max(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], off));
    }
  }
  __shared__ uint32_t s_mn[3][32], s_mx[3][32];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if (lane == 0) {
#pragma unroll
    for (int a = 0; a < 3; ++a) { s_mn[a][wid] = mn[a]; s_mx[a][wid] = mx[a]; }
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      mn[a] = lane < nw ? s_mn[a][lane] : 0xffffffffu;
      mx[a] = lane < nw ? s_mx[a][lane] : 0u;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        mn[a] = min(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], off));
        mx[a] = max(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], off));
      }
    }
    if (lane == 0) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        if (mn[a] != 0xffffffffu) atomicMin(&acc[a], mn[a]);
        if (mx[a] != 0u) atomicMax(&acc[3 + a], mx[a]);
      }
    }
  }
}

// ---------------------------------------------------------------- set-up kernels

// Scatter host-order input (xyz triples) into slots in reference order.
__global__ void k_init_state(const float* __restrict__ pin, const float* __restrict__ vin,
                             const float* __restrict__ pm, float4* __restrict__ pos, float4* __restrict__ vel,
                             uint32_t* __restrict__ orig, uint32_t* __restrict__ slot_of,
                             float4* __restrict__ bpos, SphConst k) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= k.n_total) return;
  float x = pin[3 * i], y = pin[3 * i + 1], z = pin[3 * i + 2];
  bool fluid = i < k.n_fluid;
  float m = fluid ? k.mass : -pm[i];
  pos[i] = make_float4(x, y, z, m);
  vel[i] = make_float4(vin[3 * i], vin[3 * i + 1], vin[3 * i + 2], 0.0f);
  orig[i] = i;
  slot_of[i] = i;
  if (!fluid) bpos[i - k.n_fluid] = make_float4(x, y, z, 0.0f);
}

// Overwrite positions/velocities (reference order input) keeping the current slot order.
__global__ void k_write_state(const float* __restrict__ pin, const float* __restrict__ vin,
                              float4* __restrict__ pos, float4* __restrict__ vel,
                              const uint32_t* __restrict__ orig, float4* __restrict__ bpos, SphConst k) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= k.n_total) return;
  uint32_t o = orig[s];
  float4 p = pos[s];
  if (pin) {
    p.x = pin[3 * o]; p.y = pin[3 * o + 1]; p.z = pin[3 * o + 2];
    pos[s] = p;
    if (o >= k.n_fluid) bpos[o - k.n_fluid] = make_float4(p.x, p.y, p.z, 0.0f);
  }
  if (vin) vel[s] = make_float4(vin[3 * o], vin[3 * o + 1], vin[3 * o + 2], 0.0f);
}

// Boundary segment re-upload (crates/vxl-phys-gpu/src/pipeline/coupling.rs:20-50):
// boundary particle k sits in slot slot_of[n_fluid + k].
__global__ void k_upload_boundary(const float* __restrict__ pin, const float* __restrict__ vin,
                                  float4* __restrict__ pos, float4* __restrict__ vel,
                                  const uint32_t* __restrict__ slot_of, float4* __restrict__ bpos,
                                  uint32_t* __restrict__ bbox_acc, SphConst k) {
  uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t nb = k.n_total - k.n_fluid;
  bool valid = q < nb;
  float x = 0, y = 0, z = 0;
  if (valid) {
    uint32_t s = slot_of[k.n_fluid + q];
    x = pin[3 * q]; y = pin[3 * q + 1]; z = pin[3 * q + 2];
    float4 p = pos[s];
    p.x = x; p.y = y; p.z = z;
    pos[s] = p;
    vel[s] = make_float4(vin[3 * q], vin[3 * q + 1], vin[3 * q + 2], 0.0f);
    bpos[q] = make_float4(x, y, z, 0.0f);
  }
  block_bbox_accumulate(bbox_acc, x, y, z, valid);
}

// AABB of fluid (pos.w > 0) or boundary (pos.w < 0) slots into acc.
__global__ void k_bbox(const float4* __restrict__ pos, uint32_t n, int want_fluid, uint32_t* __restrict__ acc) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  float4 p = make_float4(0, 0, 0, 0);
  bool valid = false;
  if (s < n) {
    p = pos[s];
    valid = want_fluid ? (p.w > 0.0f) : (p.w < 0.0f);
  }
  block_bbox_accumulate(acc, p.x, p.y, p.z, valid);
}

// ---------------------------------------------------------------- substep kernels

// Grid box of this substep from the AABB of all particles
// (crates/vxl-phys-fluid/src/grid.rs:37-44 -> crates/vxl-phys-core/src/grid.rs:34-50),
// then reset the fluid accumulator for the force kernel's epilogue.
__global__ void k_gridbox(Ctl* ctl, float h, uint32_t max_bins) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  float lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = fminf(o2f(ctl->fbox[a]), o2f(ctl->bbox[a]));
    hi[a] = fmaxf(o2f(ctl->fbox[3 + a]), o2f(ctl->bbox[3 + a]));
  }
  GridBox g;
  if (!grid_box(lo[0], lo[1], lo[2], hi[0], hi[1], hi[2], h, max_bins, g)) atomicOr(&ctl->err, kErrGridLoop);
  ctl->grid = g;
  for (int a = 0; a < 3; ++a) {
    ctl->fbox[a] = 0xffffffffu;
    ctl->fbox[3 + a] = 0u;
  }
}

// Cell key + arrival rank per slot. Lanes with equal keys are merged into one atomic
// (warp-aggregated); the rank is only a placement ticket — canon makes the final order
// deterministic.
__global__ void k_keys(const float4* __restrict__ pos, const Ctl* __restrict__ ctl, uint32_t* __restrict__ counts,
                       uint2* __restrict__ cellrank, uint32_t n) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  const GridBox g = ctl->grid;
  bool valid = s < n;
  uint32_t c = 0xffffffffu;
  if (valid) {
    float4 p = pos[s];
    c = cell_index(g, p.x, p.y, p.z);
  }
  uint32_t active = __ballot_sync(0xffffffffu, valid);
  if (!valid) return;
  uint32_t peers = __match_any_sync(active, c);
  int lane = threadIdx.x & 31;
  int leader = __ffs(peers) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(&counts[c], (uint32_t)__popc(peers));
  base = __shfl_sync(peers, base, leader);
  uint32_t rank = base + __popc(peers & ((1u << lane) - 1u));
  cellrank[s] = make_uint2(c, rank);
}

// Exclusive scan counts -> start, phase 1: per-tile sums.
__global__ void k_scan_partial(const uint32_t* __restrict__ counts, const Ctl* __restrict__ ctl,
                               uint32_t* __restrict__ partial) {
  uint32_t total = ctl->grid.total;
  uint32_t base = blockIdx.x * kScanTile;
  if (base >= total) return;
  uint32_t sum = 0;
  for (uint32_t i = base + threadIdx.x; i < min(base + kScanTile, total); i += kScanThreads) sum += counts[i];
  for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off);
  __shared__ uint32_t ws[kScanThreads / 32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < kScanThreads / 32; ++w) t += ws[w];
    partial[blockIdx.x] = t;
  }
}

// Phase 2: one block scans the tile sums (<= 1024 tiles: max_bins <= 2^21).
__global__ void k_scan_top(uint32_t* __restrict__ partial, const Ctl* __restrict__ ctl, uint32_t* __restrict__ start) {
  uint32_t total = ctl->grid.total;
  uint32_t ntiles = (total + kScanTile - 1) / kScanTile;
  __shared__ uint32_t sh[1024];
  uint32_t t = threadIdx.x;
  uint32_t v = t < ntiles ? partial[t] : 0u;
  sh[t] = v;
  __syncthreads();
  for (uint32_t off = 1; off < 1024; off <<= 1) {
    uint32_t add = t >= off ? sh[t - off] : 0u;
    __syncthreads();
    sh[t] += add;
    __syncthreads();
  }
  if (t < ntiles) partial[t] = sh[t] - v;  // exclusive
  if (t == 1023) start[total] = sh[1023];
}

// Phase 3: per-tile exclusive scan + tile offset -> start; zero counts for the next substep.
__global__ void k_scan_final(uint32_t* __restrict__ counts, const Ctl* __restrict__ ctl,
                             const uint32_t* __restrict__ partial, uint32_t* __restrict__ start) {
  uint32_t total = ctl->grid.total;
  uint32_t base = blockIdx.x * kScanTile;
  if (base >= total) return;
  constexpr int kPer = kScanTile / kScanThreads;  // 8 consecutive cells per thread
  uint32_t v[kPer];
  uint32_t i0 = base + threadIdx.x * kPer;
  uint32_t local = 0;
#pragma unroll
  for (int q = 0; q < kPer; ++q) {
    uint32_t i = i0 + q;
    v[q] = i < total ? counts[i] : 0u;
    local += v[q];
  }
  // block exclusive scan of `local`
  uint32_t incl = local;
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += y;
  }
  __shared__ uint32_t ws[kScanThreads / 32];
  if (lane == 31) ws[wid] = incl;
  __syncthreads();
  uint32_t woff = 0;
  for (int w = 0; w < wid; ++w) woff += ws[w];
  uint32_t run = partial[blockIdx.x] + woff + incl - local;
#pragma unroll
  for (int q = 0; q < kPer; ++q) {
    uint32_t i = i0 + q;
    if (i < total) {
      start[i] = run;
      counts[i] = 0u;
    }
    run += v[q];
  }
}

// Place each slot's (reference index, old slot) at start[cell] + rank.
__global__ void k_place(const uint2* __restrict__ cellrank, const uint32_t* __restrict__ start,
                        const uint32_t* __restrict__ orig, uint2* __restrict__ items, uint32_t n) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint2 cr = cellrank[s];
  items[start[cr.x] + cr.y] = make_uint2(orig[s], s);
}

// Per cell: order the placed entries by reference index (the reference's index-ascending
// table, grid.rs:56-62) and gather position/velocity into the sorted buffer.
// A warp scans 32 consecutive cells at a time and handles each non-empty one
// cooperatively. Rank of an entry = number of entries in the cell with a smaller
// reference index (indices are unique).
__device__ __forceinline__ void canon_cell(uint32_t b, uint32_t n, int lane, uint32_t* skeys, Ctl* ctl,
                                           const uint2* __restrict__ items, const float4* __restrict__ pos_in,
                                           const float4* __restrict__ vel_in, float4* __restrict__ pos_out,
                                           float4* __restrict__ vel_out, uint32_t* __restrict__ orig,
                                           uint32_t* __restrict__ slot_of) {
  if (n <= 32) {
    uint2 it = make_uint2(0xffffffffu, 0u);
    if ((uint32_t)lane < n) it = items[b + lane];
    uint32_t rank = 0;
    for (uint32_t j = 0; j < n; ++j) {
      uint32_t kj = __shfl_sync(0xffffffffu, it.x, j);
      rank += (kj < it.x) ? 1u : 0u;
    }
    if ((uint32_t)lane < n) {
      uint32_t dst = b + rank;
      pos_out[dst] = pos_in[it.y];
      vel_out[dst] = vel_in[it.y];
      orig[dst] = it.x;
      slot_of[it.x] = dst;
    }
  } else if (n <= (uint32_t)kCanonSmem) {
    for (uint32_t e = lane; e < n; e += 32) skeys[e] = items[b + e].x;
    __syncwarp();
    for (uint32_t e = lane; e < n; e += 32) {
      uint2 it = items[b + e];
      uint32_t rank = 0;
      for (uint32_t j = 0; j < n; ++j) rank += (skeys[j] < it.x) ? 1u : 0u;
      uint32_t dst = b + rank;
      pos_out[dst] = pos_in[it.y];
      vel_out[dst] = vel_in[it.y];
      orig[dst] = it.x;
      slot_of[it.x] = dst;
    }
    __syncwarp();
  } else {
    if (lane == 0) atomicOr(&ctl->err, kErrCanonLarge);
    for (uint32_t e = lane; e < n; e += 32) {
      uint2 it = items[b + e];
      uint32_t rank = 0;
      for (uint32_t j = 0; j < n; ++j) rank += (items[b + j].x < it.x) ? 1u : 0u;
      uint32_t dst = b + rank;
      pos_out[dst] = pos_in[it.y];
      vel_out[dst] = vel_in[it.y];
      orig[dst] = it.x;
      slot_of[it.x] = dst;
    }
  }
}

__global__ void k_canon(const uint2* __restrict__ items, const uint32_t* __restrict__ start, Ctl* ctl,
                        const float4* __restrict__ pos_in, const float4* __restrict__ vel_in,
                        float4* __restrict__ pos_out, float4* __restrict__ vel_out, uint32_t* __restrict__ orig,
                        uint32_t* __restrict__ slot_of) {
  __shared__ uint32_t skeys[8][kCanonSmem];
  const uint32_t total = ctl->grid.total;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32u; base < total; base += warps * 32u) {
    uint32_t c = base + lane;
    uint32_t b = 0, n = 0;
    if (c < total) {
      b = start[c];
      n = start[c + 1] - b;
    }
    uint32_t mask = __ballot_sync(0xffffffffu, n > 0);
    while (mask) {
      int l = __ffs(mask) - 1;
      mask &= mask - 1;
      uint32_t cb = __shfl_sync(0xffffffffu, b, l);
      uint32_t cn = __shfl_sync(0xffffffffu, n, l);
      canon_cell(cb, cn, lane, skeys[wib], ctl, items, pos_in, vel_in, pos_out, vel_out, orig, slot_of);
    }
  }
}

// Walk the 27 cells around position p (cell (cx, cy, cz)) in the reference order
// (dz outer, dy, dx inner; crates/vxl-phys-fluid/src/grid.rs:123-153), calling f(j) for
// every slot j in them — except cells whose nominal box lies farther than h from p.
// Such a cell holds no particle with r2 <= h2, so skipping it changes neither the set nor
// the order of accepted neighbours. The test is conservative: per-axis gaps to the
// neighbouring cell faces are clamped at 0 and compared with (h + bin/1024)^2, a margin
// far above the f32 rounding of cell faces and bin assignment.
template <class F>
__device__ __forceinline__ void walk27(const GridBox& g, const uint32_t* __restrict__ start, float px, float py,
                                       float pz, uint32_t cx, uint32_t cy, uint32_t cz, float h, F&& f) {
  const float lx = g.minx + (float)cx * g.bin, ly = g.miny + (float)cy * g.bin, lz = g.minz + (float)cz * g.bin;
  const float gxl = fmaxf(px - lx, 0.0f), gxr = fmaxf(lx + g.bin - px, 0.0f);
  const float gyl = fmaxf(py - ly, 0.0f), gyr = fmaxf(ly + g.bin - py, 0.0f);
  const float gzl = fmaxf(pz - lz, 0.0f), gzr = fmaxf(lz + g.bin - pz, 0.0f);
  const float reach = h + g.bin * (1.0f / 1024.0f);
  const float reach2 = reach * reach;
  for (int dz = -1; dz <= 1; ++dz) {
    const int z = (int)cz + dz;
    if (z < 0 || z >= (int)g.nz) continue;
    const float gz = dz < 0 ? gzl : (dz > 0 ? gzr : 0.0f);
    const float dz2 = gz * gz;
    for (int dy = -1; dy <= 1; ++dy) {
      const int y = (int)cy + dy;
      if (y < 0 || y >= (int)g.ny) continue;
      const float gy = dy < 0 ? gyl : (dy > 0 ? gyr : 0.0f);
      const float dyz2 = dz2 + gy * gy;
      for (int dx = -1; dx <= 1; ++dx) {
        const int x = (int)cx + dx;
        if (x < 0 || x >= (int)g.nx) continue;
        const float gx = dx < 0 ? gxl : (dx > 0 ? gxr : 0.0f);
        if (dyz2 + gx * gx > reach2) continue;
        const uint32_t idx = ((uint32_t)x * g.ny + (uint32_t)y) * g.nz + (uint32_t)z;
        const uint32_t j1 = start[idx + 1];
        for (uint32_t j = start[idx]; j < j1; ++j) f(j);
      }
    }
  }
}

// Density (poly6 with self term) + Tait EOS, one thread per slot.
// Fluid: rho = mass * (w0 + sum_fluid W) + sum_boundary pmass_j W
// (crates/vxl-phys-fluid/src/fluid_density.rs:24-51); boundary: rho = pmass_i w0 +
// sum_fluid pmass_j W (fluid_density.rs:59-69). Writes (rho, p / rho^2) for the force
// pass (the reference recomputes press/(rho*rho) per pair: same value).
// Also records, in walk order, the slots of the neighbours that contributed (all of
// them for fluid, fluid ones for boundary particles): nbr[k * n_total + s], k < cap,
// and the full count in nbr_n[s] (a count above cap sends the consumers back to the walk).
__global__ void __launch_bounds__(256, 6) k_density(const float4* __restrict__ pos, const uint32_t* __restrict__ start,
                                                 const Ctl* __restrict__ ctl, float2* __restrict__ rc,
                                                 float* __restrict__ press_out, uint32_t* __restrict__ nbr,
                                                 uint32_t* __restrict__ nbr_n, uint32_t cap, SphConst k) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= k.n_total) return;
  const GridBox g = ctl->grid;
  const uint32_t nt = k.n_total;
  float4 pi = pos[s];
  bool fluid_i = pi.w > 0.0f;
  uint32_t cx, cy, cz;
  bin_of(g, pi.x, pi.y, pi.z, cx, cy, cz);
  float sum = fluid_i ? k.w0 : 0.0f;
  float sum_b = 0.0f;
  uint32_t cnt = 0;
  const float h2 = k.h2, k6 = k.k6;
  walk27(g, start, pi.x, pi.y, pi.z, cx, cy, cz, k.h, [&](uint32_t j) {
    if (j == s) return;
    float4 pj = pos[j];
    float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
    float r2 = dx * dx + dy * dy + dz * dz;
    if (r2 <= h2) {
      float t = h2 - r2;
      float w = k6 * t * t * t;
      bool rec = true;
      if (fluid_i) {
        if (pj.w > 0.0f) sum += w;
        else sum_b += (-pj.w) * w;
      } else if (pj.w > 0.0f) {
        sum += pj.w * w;
      } else {
        rec = false;
      }
      if (rec) {
        if (cnt < cap) nbr[(size_t)cnt * nt + s] = j;
        ++cnt;
      }
    }
  });
  nbr_n[s] = cnt;
  float rho = fluid_i ? (k.mass * sum + sum_b) : ((-pi.w) * k.w0 + sum);
  float p = tait(k, rho);
  rc[s] = make_float2(rho, p / (rho * rho));
  if (press_out) press_out[s] = p;
}

// Force (gravity + spiky pressure + Monaghan viscosity + XSPH, fluid_force.rs:165-214)
// fused with integration (semi-implicit Euler + CFL clamp, fluid_step.rs:112-123) for
// fluid slots; boundary slots are copied unchanged (kinematic within the tick).
// Neighbours come from the density pass's list (same walk order, so the same sums);
// a particle whose list overflowed walks the 27 cells again.
// Reads the sorted buffer (pos, vel) and writes the integrated state to (pos_out, vel_out)
// in the same slot order; accumulates the fluid AABB for the next substep's grid box.
__global__ void __launch_bounds__(256) k_force(const float4* __restrict__ pos, const float4* __restrict__ vel,
                                               const float2* __restrict__ rc, const uint32_t* __restrict__ start,
                                               const uint32_t* __restrict__ nbr, const uint32_t* __restrict__ nbr_n,
                                               uint32_t cap, Ctl* ctl, float4* __restrict__ pos_out,
                                               float4* __restrict__ vel_out, float4* __restrict__ acc_out,
                                               float4* __restrict__ xsph_out, SphConst k, StepConst st) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  bool valid = s < k.n_total;
  float nx = 0, ny = 0, nz = 0;
  bool fluid_i = false;
  if (valid) {
    float4 pi = pos[s];
    float4 vi = vel[s];
    fluid_i = pi.w > 0.0f;
    if (!fluid_i) {
      pos_out[s] = pi;
      vel_out[s] = vi;
    } else {
      float2 rci = rc[s];
      const float rho_i = rci.x, ci2 = rci.y;
      const float h = k.h, h2 = k.h2, ks = k.ks, k6 = k.k6, alpha_c = k.alpha_c, h001 = k.h001;
      float ax = k.gx, ay = k.gy, az = k.gz;
      float xx = 0.0f, xy = 0.0f, xz = 0.0f;
      auto pair = [&](uint32_t j, float4 pj, float dx, float dy, float dz, float r2) {
        float2 rcj = rc[j];
        float4 vj = vel[j];
        const float rho_j = rcj.x, cj2 = rcj.y;
        const float mj = fabsf(pj.w);
        float r = sqrtf(r2);
        float t = h - r;
        float coef = mj * (ks * t * t) * (ci2 + cj2);
        float denom = fmaxf(r, 1e-9f);
        float q = coef / denom;
        ax = ax + dx * q;
        ay = ay + dy * q;
        az = az + dz * q;
        float vx = vi.x - vj.x, vy = vi.y - vj.y, vz = vi.z - vj.z;
        float vdn = -(vx * dx + vy * dy + vz * dz);
        if (vdn > 0.0f) {
          float mu = vdn * h / (r2 + h001);
          float c = mj * (alpha_c * mu / (0.5f * (rho_i + rho_j))) * (ks * t * t);
          float q2 = c / denom;
          ax = ax + dx * q2;
          ay = ay + dy * q2;
          az = az + dz * q2;
        }
        float tt = h2 - r2;
        float w = k6 * tt * tt * tt;
        float f = mj * 2.0f / (rho_i + rho_j) * w;
        xx = xx + (vj.x - vi.x) * f;
        xy = xy + (vj.y - vi.y) * f;
        xz = xz + (vj.z - vi.z) * f;
      };
      const uint32_t cnt = nbr_n[s];
      if (cnt <= cap) {
        const uint32_t nt = k.n_total;
        for (uint32_t q = 0; q < cnt; ++q) {
          uint32_t j = nbr[(size_t)q * nt + s];
          float4 pj = pos[j];
          float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
          float r2 = dx * dx + dy * dy + dz * dz;
          pair(j, pj, dx, dy, dz, r2);
        }
      } else {
        const GridBox g = ctl->grid;
        uint32_t cx, cy, cz;
        bin_of(g, pi.x, pi.y, pi.z, cx, cy, cz);
        walk27(g, start, pi.x, pi.y, pi.z, cx, cy, cz, k.h, [&](uint32_t j) {
          if (j == s) return;
          float4 pj = pos[j];
          float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
          float r2 = dx * dx + dy * dy + dz * dz;
          if (r2 <= h2) pair(j, pj, dx, dy, dz, r2);
        });
      }
      if (acc_out) {
        acc_out[s] = make_float4(ax, ay, az, 0.0f);
        xsph_out[s] = make_float4(xx, xy, xz, 0.0f);
      }
      float dt = st.dt, eps = k.eps;
      float ux = vi.x + ax * dt + xx * eps;
      float uy = vi.y + ay * dt + xy * eps;
      float uz = vi.z + az * dt + xz * eps;
      float s2 = ux * ux + uy * uy + uz * uz;
      if (s2 > st.vmax2) {
        float sc = st.vmax / sqrtf(s2);
        ux = ux * sc;
        uy = uy * sc;
        uz = uz * sc;
      }
      nx = pi.x + ux * dt;
      ny = pi.y + uy * dt;
      nz = pi.z + uz * dt;
      pos_out[s] = make_float4(nx, ny, nz, pi.w);
      vel_out[s] = make_float4(ux, uy, uz, 0.0f);
    }
  }
  block_bbox_accumulate(ctl->fbox, nx, ny, nz, valid && fluid_i);
}

// Pair term of the boundary reaction for fluid i on boundary j, from i's side of the
// reference loop (crates/vxl-phys-fluid/src/fluid_force.rs:182-207): returns
// q = m_i (coef + cv) / denom, with d = p_i - p_j; the caller applies bforce -= d * q.
__device__ __forceinline__ float bforce_pair(const SphConst& k, float r2, float dx, float dy, float dz,
                                             float rho_i, float ci2, float mi, float4 vi, float rho_j, float cj2,
                                             float mj, float4 vj) {
  float r = sqrtf(r2);
  float t = k.h - r;
  float coef = mj * (k.ks * t * t) * (ci2 + cj2);
  float denom = fmaxf(r, 1e-9f);
  float cv = 0.0f;
  float vx = vi.x - vj.x, vy = vi.y - vj.y, vz = vi.z - vj.z;
  float vdn = -(vx * dx + vy * dy + vz * dz);
  if (vdn > 0.0f) {
    float mu = vdn * k.h / (r2 + k.h001);
    cv = mj * (k.alpha_c * mu / (0.5f * (rho_i + rho_j))) * (k.ks * t * t);
  }
  return mi * (coef + cv) / denom;
}

// Reaction on each boundary particle j: the reference accumulates bforce[j] -= F_ij over
// fluid i in ascending reference index (the outer loop of force_pass_serial). Here the
// boundary particle takes its fluid neighbours (recorded by the density pass, or found by
// walking the 27 cells when that list overflowed), orders them by reference index and
// sums in that order, so the result is the same sum. Output in boundary order
// (bforce[k], k = reference index - n_fluid).
__global__ void __launch_bounds__(128) k_bforce(const float4* __restrict__ pos, const float4* __restrict__ vel,
                                                const float2* __restrict__ rc, const uint32_t* __restrict__ start,
                                                const uint32_t* __restrict__ orig, const uint32_t* __restrict__ nbr,
                                                const uint32_t* __restrict__ nbr_n, uint32_t cap, Ctl* ctl,
                                                float4* __restrict__ bforce, SphConst k) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= k.n_total) return;
  float4 pj = pos[s];
  if (pj.w > 0.0f) return;  // fluid slot
  const GridBox g = ctl->grid;
  const float h2 = k.h2;
  float4 vj = vel[s];
  float2 rcj = rc[s];
  const float mj = -pj.w;
  uint32_t cx, cy, cz;
  bin_of(g, pj.x, pj.y, pj.z, cx, cy, cz);
  uint32_t key[kBGatherCap];
  uint32_t slot[kBGatherCap];
  int n = 0;
  bool overflow = false;
  auto insert = [&](uint32_t i) {
    if (n < kBGatherCap) {
      uint32_t o = orig[i];
      int q = n++;
      while (q > 0 && key[q - 1] > o) {
        key[q] = key[q - 1];
        slot[q] = slot[q - 1];
        --q;
      }
      key[q] = o;
      slot[q] = i;
    } else {
      overflow = true;
    }
  };
  const uint32_t cnt = nbr_n[s];
  if (cnt <= cap) {
    for (uint32_t q = 0; q < cnt; ++q) insert(nbr[(size_t)q * k.n_total + s]);
  } else {
    walk27(g, start, pj.x, pj.y, pj.z, cx, cy, cz, k.h, [&](uint32_t i) {
      float4 p = pos[i];
      if (!(p.w > 0.0f)) return;
      float dx = p.x - pj.x, dy = p.y - pj.y, dz = p.z - pj.z;
      float r2 = dx * dx + dy * dy + dz * dz;
      if (!(r2 <= h2)) return;
      insert(i);
    });
  }
  float bx = 0.0f, by = 0.0f, bz = 0.0f;
  auto apply = [&](uint32_t i) {
    float4 p = pos[i];
    float dx = p.x - pj.x, dy = p.y - pj.y, dz = p.z - pj.z;
    float r2 = dx * dx + dy * dy + dz * dz;
    float2 rci = rc[i];
    float q = bforce_pair(k, r2, dx, dy, dz, rci.x, rci.y, p.w, vel[i], rcj.x, rcj.y, mj, vj);
    bx = bx - dx * q;
    by = by - dy * q;
    bz = bz - dz * q;
  };
  if (!overflow) {
    for (int q = 0; q < n; ++q) apply(slot[q]);
  } else {
    // Slow path: visit fluid neighbours in ascending reference index by repeated
    // minimum search (O(neighbours x candidates)); counted in ctl->slow_gathers.
    atomicAdd(&ctl->slow_gathers, 1u);
    uint32_t last = 0;
    bool first = true;
    for (;;) {
      uint32_t best = 0xffffffffu, best_slot = 0;
      walk27(g, start, pj.x, pj.y, pj.z, cx, cy, cz, k.h, [&](uint32_t i) {
        float4 p = pos[i];
        if (!(p.w > 0.0f)) return;
        uint32_t o = orig[i];
        if (!first && o <= last) return;
        if (o >= best) return;
        float dx = p.x - pj.x, dy = p.y - pj.y, dz = p.z - pj.z;
        float r2 = dx * dx + dy * dy + dz * dz;
        if (!(r2 <= h2)) return;
        best = o;
        best_slot = i;
      });
      if (best == 0xffffffffu) break;
      apply(best_slot);
      last = best;
      first = false;
    }
  }
  bforce[orig[s] - k.n_fluid] = make_float4(bx, by, bz, 0.0f);
}

// Per-span force and torque about the body origin (fluid_boundary.rs:10-28), added to
// the tick accumulator. Fixed-shape two-level reduction, deterministic run to run:
// level 1, one block per chunk of <= kReactChunk consecutive particles of a span
// (thread t sums t, t + blockDim, ... in order, then a fixed tree); level 2, one thread
// per span adds its chunk partials in chunk order.
struct SpanDev {
  uint32_t body;
  float ox, oy, oz;
  uint32_t start, end;
};

struct SpanChunk {
  uint32_t span, begin, end, pad;
};

constexpr uint32_t kReactChunk = 4096;
constexpr int kReactThreads = 256;

__global__ void __launch_bounds__(kReactThreads) k_react_chunks(const float4* __restrict__ bforce,
                                                                const float4* __restrict__ bpos,
                                                                const SpanDev* __restrict__ spans,
                                                                const SpanChunk* __restrict__ chunks,
                                                                float* __restrict__ partial, uint32_t n_fluid) {
  const SpanChunk ch = chunks[blockIdx.x];
  const SpanDev sp = spans[ch.span];
  float f[6] = {0, 0, 0, 0, 0, 0};
  for (uint32_t kk = ch.begin + threadIdx.x; kk < ch.end; kk += kReactThreads) {
    float4 fk = bforce[kk - n_fluid];
    float4 p = bpos[kk - n_fluid];
    float rx = p.x - sp.ox, ry = p.y - sp.oy, rz = p.z - sp.oz;
    f[0] = f[0] + fk.x;
    f[1] = f[1] + fk.y;
    f[2] = f[2] + fk.z;
    f[3] = f[3] + (ry * fk.z - rz * fk.y);
    f[4] = f[4] + (rz * fk.x - rx * fk.z);
    f[5] = f[5] + (rx * fk.y - ry * fk.x);
  }
  __shared__ float sh[6][kReactThreads];
  for (int a = 0; a < 6; ++a) sh[a][threadIdx.x] = f[a];
  __syncthreads();
  for (uint32_t w = kReactThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int a = 0; a < 6; ++a) sh[a][threadIdx.x] = sh[a][threadIdx.x] + sh[a][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 6) partial[6 * blockIdx.x + threadIdx.x] = sh[threadIdx.x][0];
}

// chunk_first[q] .. chunk_first[q + 1]: the chunks of span q (in order).
__global__ void k_react_spans(const float* __restrict__ partial, const uint32_t* __restrict__ chunk_first,
                              float* __restrict__ breact, uint32_t nspans) {
  uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nspans) return;
  float f[6] = {0, 0, 0, 0, 0, 0};
  for (uint32_t c = chunk_first[q]; c < chunk_first[q + 1]; ++c)
    for (int a = 0; a < 6; ++a) f[a] = f[a] + partial[6 * c + a];
  for (int a = 0; a < 6; ++a) breact[6 * q + a] = breact[6 * q + a] + f[a];
}

// Tick average (fluid_step.rs:84-88): e *= 1 / substeps.
__global__ void k_scale(float* __restrict__ breact, uint32_t n, float inv) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) breact[i] = breact[i] * inv;
}

// ---------------------------------------------------------------- export kernels

__global__ void k_read_state(const float4* __restrict__ pos, const float4* __restrict__ vel,
                             const uint32_t* __restrict__ orig, float* __restrict__ pout, float* __restrict__ vout,
                             uint32_t n) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t o = orig[s];
  if (pout) {
    float4 p = pos[s];
    pout[3 * o] = p.x; pout[3 * o + 1] = p.y; pout[3 * o + 2] = p.z;
  }
  if (vout) {
    float4 v = vel[s];
    vout[3 * o] = v.x; vout[3 * o + 1] = v.y; vout[3 * o + 2] = v.z;
  }
}

__global__ void k_read_fields(const float2* __restrict__ rc, const float* __restrict__ press,
                              const float4* __restrict__ acc, const float4* __restrict__ xsph,
                              const uint32_t* __restrict__ orig, float* __restrict__ dout, float* __restrict__ pout,
                              float* __restrict__ aout, float* __restrict__ xout, uint32_t n) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t o = orig[s];
  if (dout) dout[o] = rc[s].x;
  if (pout) pout[o] = press[s];
  if (aout) { float4 a = acc[s]; aout[3 * o] = a.x; aout[3 * o + 1] = a.y; aout[3 * o + 2] = a.z; }
  if (xout) { float4 x = xsph[s]; xout[3 * o] = x.x; xout[3 * o + 1] = x.y; xout[3 * o + 2] = x.z; }
}

__global__ void k_export_bins(const uint32_t* __restrict__ start, const uint32_t* __restrict__ orig,
                              const Ctl* __restrict__ ctl, uint32_t* __restrict__ bins) {
  uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ctl->grid.total) return;
  for (uint32_t q = start[c]; q < start[c + 1]; ++q) bins[orig[q]] = c;
}

}  // namespace
}  // namespace vxl
