// Multi-scene WCSPH engine: the device kernels of one substep for any number of
// resident scenes (sm_100a). One scene is the plain drop-in; many scenes are the
// batched and served forms.
//
// Layout. All scenes share one pool of particle slots, packed without gaps in scene
// order: scene q owns slots [base_q, base_q + n_q) and its particles never leave that
// range. Per slot (structure of arrays):
//   pos[s]  float4 (x, y, z, m)   m = +particle mass for fluid, -pmass for boundary
//   vel[s]  float4 (vx, vy, vz, 0)
//   orig[s] global reference index (base_q + the particle's index in its scene);
//           slot_of[orig[s]] == s
// Each substep every scene gets its own grid (the reference's grid rule on its own
// AABB, crates/vxl-phys-core/src/grid.rs:34-50) and a range of a global cell space
// [cell_off_q, cell_off_q + cells_q), assigned in scene order. A particle's key is
// cell_off_q + its cell, so one counting sort over the global cells is a segmented sort
// that keeps each scene inside its slot range, and inside every cell the slots ascend by
// reference index: the reference's table (crates/vxl-phys-fluid/src/grid.rs:29-76).
// Walking a scene's 27 cells in the reference's (dz, dy, dx) order over those ranges
// visits neighbours in the order of UniformGrid::for_neighbors_in (grid.rs:115-155),
// so every per-particle sum matches the reference's CPU path bit for bit.
//
// Work list. The particle kernels run persistent blocks over a list of tiles
// (scene, first slot, count): a block takes the next tile from an atomic counter, so the
// scene of a tile is uniform and scenes of very different sizes balance across SMs.
//
// Substep: gridbox (per scene) -> cell offsets -> keys -> scan -> place -> canon ->
// density + EOS (+ neighbour lists) -> force + XSPH + integrate -> boundary reactions ->
// per-span reduction.
#pragma once

#include "sph_device.cuh"

// Resident threads per SM the density and force passes are compiled for (register
// budget = 65536 / this).
#ifndef VXL_DENSITY_THREADS_PER_SM
#define VXL_DENSITY_THREADS_PER_SM 2048
#endif
#ifndef VXL_FORCE_THREADS_PER_SM
#define VXL_FORCE_THREADS_PER_SM 1280
#endif
#ifndef VXL_DENSITY_SEG_THREADS_PER_SM
#define VXL_DENSITY_SEG_THREADS_PER_SM 1024  // 64 registers, no spills: 11.4 vs 15.0 ms at 1536 on dam10m
#endif


namespace vxl {

constexpr uint32_t kErrCellCap = 1u << 3;  // the scenes' cells exceed the cell capacity

// Per-scene device record (one per scene of the engine). The fields up to `g` are
// written by the host (constants, substep dt, slot range); the rest by the kernels.
struct SceneDev {
  SphConst k;
  float dt, vmax, vmax2, pad0;
  uint32_t base;        // first slot
  uint32_t count;       // slots (fluid + boundary)
  uint32_t prov_first;  // the scene's providers in the engine's provider array
  uint32_t prov_count;  // 0: no provider walls
  GridBox g;            // this substep's grid
  uint32_t cell_off;    // first global cell this substep
  uint32_t cells;       // cells this substep
  uint32_t fbox[6];     // fluid AABB accumulator (ordered uint)
  uint32_t bbox[6];     // boundary AABB (fixed within a tick)
};

// Per-body pose of the device-side boundary rebuild.
struct BodyPoseDev {
  float px, py, pz;
  float qx, qy, qz, qw;
  float vx, vy, vz;
  float wx, wy, wz;
};

// A rigid body of the device-side coupling loop: pose and velocities (the BodyPoseDev
// fields, same names), mass properties, and the global index of the span whose reaction
// drives it (~0u: none).
struct RigidBodyDev {
  float px, py, pz;
  float qx, qy, qz, qw;
  float vx, vy, vz;
  float wx, wy, wz;
  float inv_mass, iix, iiy, iiz;
  uint32_t dynamic, span;
};

struct TileDev {
  uint32_t scene, first, count, pad;
};

// Body span (global reference indices [start, end)) and its reduction chunks.
struct SpanDev {
  uint32_t body;
  float ox, oy, oz;
  uint32_t start, end;
  uint32_t rigid;  // coupled rigid body whose position is the torque origin (~0u: use ox, oy, oz)
};

struct LongSpan {  // a span above kReactExactSpan, summed by a block of its own
  uint32_t span, begin, end, pad;
};

// Spans of at most this many particles (bodies) are summed by one warp each; larger ones
// (tank walls) by one block each. Both add the terms in index order: the reference's sum,
// bit for bit.
constexpr uint32_t kReactExactSpan = 8192;
constexpr uint32_t kReactBatch = 1024;  // terms a block stages per step of a long span
constexpr int kReactThreads = 256;
constexpr int kReactSpanWarps = 2;  // spans per block of k_react_spans (one warp each)

// Engine-wide control block.
constexpr int kWorkSlots = 16;  // persistent-kernel work counters per substep
struct EngineCtl {
  uint32_t cells;  // sum of the scenes' cells this substep
  uint32_t err;
  uint32_t slow_gathers;
  uint32_t doubled;  // some scene's bins are at least 2h this substep (half-cell masks needed)
  uint32_t epoch;    // substep counter: wet[c] == epoch marks cells holding fluid this substep
  uint32_t work[kWorkSlots];
};

// Work counter indices (zeroed at the start of every substep). The provider-wall passes
// keep their per-substep results in slots 4-6: pushed particles, "some pushed pair is
// closer than 0.2 h", "the separation moved a particle".
enum WorkId : int {
  kWorkDensity = 0, kWorkForce = 1, kWorkBforce = 2, kWorkScan = 3,
  kWorkPushed = 4, kWorkTrigger = 5, kWorkMoved = 6, kWorkSegs = 7
};

// Provider walls (analytic ProviderColliders queried on the device). A plane of a FACES
// provider is (axis, d = plane coordinate, sign); of a CONVEX provider (n, d).
struct WallPlaneDev {
  float nx, ny, nz, d;
  uint32_t axis;
  float sign;
  uint32_t pad0, pad1;
};

// One side (mirror or projection) of the contact tables: ent[global reference index] =
// entry + 1 (0: no planes), entry e owning planes [start[e], start[e + 1]), each plane two
// float4 (contact point, outward normal).
struct ContactTableDev {
  const uint32_t* ent;
  const uint32_t* start;
  const float4* planes;
};

struct ProviderDev {
  uint32_t kind, first, count, has_bounds;
  float bminx, bminy, bminz, bmaxx, bmaxy, bmaxz;
  uint32_t pad0, pad1;
};

constexpr uint32_t kProviderFaces = 0u, kProviderConvex = 1u;
// A contact table (any ProviderColliders, gathered on the host once per tick, as the
// reference's GPU tier does: crates/vxl-phys-gpu/src/pipeline/walls.rs:143-215) is one more
// provider of the scene, after its analytic ones, queried by particle.
constexpr uint32_t kProviderTable = 2u;
constexpr uint32_t kMaxWallPlanes = 8;     // mirror planes per particle (fluid_density.rs:110)
constexpr uint32_t kPushedChunk = 4096;    // reference indices per block of the pushed-list passes

namespace {

constexpr int kScanTile = 2048;
constexpr int kScanThreads = 256;
constexpr int kCanonSmem = 1024;
constexpr int kCanonWindow = kCanonSmem / 2;  // window path: keys + segment table in one warp's buffer
constexpr int kBGatherCap = 64;
constexpr uint32_t kListPrefetch = 4;  // force pass: list entries fetched into L2 this far ahead

// Block-level ordered-uint min/max of (x, y, z), one atomic per component into acc.
__device__ __forceinline__ void block_bbox_accumulate(uint32_t* acc, float x, float y, float z, bool valid) {
  uint32_t mn[3], mx[3];
  const float v[3] = {x, y, z};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const bool ok = valid && (v[a] == v[a]);  // NaN never wins (Rust f32::min/max ignore NaN)
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
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if (lane == 0) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      s_mn[a][wid] = mn[a];
      s_mx[a][wid] = mx[a];
    }
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
  __syncthreads();
}

// Next tile of a persistent kernel (block-uniform); >= ntiles means done.
__device__ __forceinline__ uint32_t next_tile(uint32_t* counter) {
  __shared__ uint32_t s_tile;
  if (threadIdx.x == 0) s_tile = atomicAdd(counter, 1u);
  __syncthreads();
  const uint32_t t = s_tile;
  __syncthreads();
  return t;
}

// Tile scheduling of the particle passes. A grid of at least ntiles blocks runs one
// block per tile (the hardware block scheduler balances); a smaller grid is persistent
// and its blocks draw tiles from the atomic counter until the list is exhausted.
__device__ __forceinline__ uint32_t first_tile(uint32_t* counter, uint32_t ntiles) {
  return gridDim.x >= ntiles ? blockIdx.x : next_tile(counter);
}
__device__ __forceinline__ uint32_t following_tile(uint32_t* counter, uint32_t ntiles) {
  return gridDim.x >= ntiles ? ntiles : next_tile(counter);
}

// ---------------------------------------------------------------- set-up kernels

// Scatter one scene's host-order input (xyz triples, scene-local index) into its slots
// [base, base + n) in reference order.
__global__ void k_e_init_scene(const float* __restrict__ pin, const float* __restrict__ vin,
                               const float* __restrict__ pm, float4* __restrict__ pos, float4* __restrict__ vel,
                               uint32_t* __restrict__ orig, uint32_t* __restrict__ slot_of,
                               float4* __restrict__ bpos, uint32_t base, uint32_t n, uint32_t nf, float mass) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float x = pin[3 * i], y = pin[3 * i + 1], z = pin[3 * i + 2];
  const bool fluid = i < nf;
  const uint32_t g = base + i;
  pos[g] = make_float4(x, y, z, fluid ? mass : -pm[i]);
  vel[g] = make_float4(vin[3 * i], vin[3 * i + 1], vin[3 * i + 2], 0.0f);
  orig[g] = g;
  slot_of[g] = g;
  if (!fluid) bpos[g] = make_float4(x, y, z, 0.0f);
}

// Overwrite one scene's positions/velocities (scene-local reference order input),
// keeping its current slot order.
__global__ void k_e_write_scene(const float* __restrict__ pin, const float* __restrict__ vin,
                                float4* __restrict__ pos, float4* __restrict__ vel,
                                const uint32_t* __restrict__ orig, float4* __restrict__ bpos, uint32_t base,
                                uint32_t n, uint32_t nf) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t s = base + i;
  const uint32_t o = orig[s] - base;
  if (pin) {
    float4 p = pos[s];
    p.x = pin[3 * o];
    p.y = pin[3 * o + 1];
    p.z = pin[3 * o + 2];
    pos[s] = p;
    if (o >= nf) bpos[base + o] = make_float4(p.x, p.y, p.z, 0.0f);
  }
  if (vin) vel[s] = make_float4(vin[3 * o], vin[3 * o + 1], vin[3 * o + 2], 0.0f);
}

// Boundary segment re-upload of one scene (crates/vxl-phys-gpu/src/pipeline/coupling.rs:
// 20-50): boundary particle k of the scene sits in slot slot_of[base + nf + k].
__global__ void k_e_upload_boundary(const float* __restrict__ pin, const float* __restrict__ vin,
                                    float4* __restrict__ pos, float4* __restrict__ vel,
                                    const uint32_t* __restrict__ slot_of, float4* __restrict__ bpos,
                                    uint32_t* __restrict__ bbox_acc, uint32_t base, uint32_t nf, uint32_t nb) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = q < nb;
  float x = 0, y = 0, z = 0;
  if (valid) {
    const uint32_t g = base + nf + q;
    const uint32_t s = slot_of[g];
    x = pin[3 * q];
    y = pin[3 * q + 1];
    z = pin[3 * q + 2];
    float4 p = pos[s];
    p.x = x;
    p.y = y;
    p.z = z;
    pos[s] = p;
    vel[s] = make_float4(vin[3 * q], vin[3 * q + 1], vin[3 * q + 2], 0.0f);
    bpos[g] = make_float4(x, y, z, 0.0f);
  }
  block_bbox_accumulate(bbox_acc, x, y, z, valid);
}

// AABB of one scene's fluid (pos.w > 0) or boundary (pos.w < 0) slots into acc.
__global__ void k_e_bbox(const float4* __restrict__ pos, uint32_t base, uint32_t n, int want_fluid,
                         uint32_t* __restrict__ acc) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  float4 p = make_float4(0, 0, 0, 0);
  bool valid = false;
  if (i < n) {
    p = pos[base + i];
    valid = want_fluid ? (p.w > 0.0f) : (p.w < 0.0f);
  }
  block_bbox_accumulate(acc, p.x, p.y, p.z, valid);
}

// Move whole scenes to new bases (the served form's repack): slot ranges are copied into
// the second buffer set, reference indices shifted by the move. from_base/to_base/count
// per moved scene; one block row per scene (blockIdx.y).

// set_boundary_particles on the device (crates/vxl-phys-fluid/src/fluid_step.rs:13-53): for
// boundary particle k of a scene (reference order), with body-frame lattice point L and
// its body's pose, world position p = body.pos + rotate(q, L) (Quat::rotate_vec3:
// t = 2 (q.xyz x L); L + q.xyz x t + w t) and velocity v = linvel + angvel x (p - body.pos),
// in f32 in the reference's operation order. Written at the particle's current slot and in
// reference order (bpos); the boundary AABB is re-accumulated. The class/mass word is kept.
__device__ __forceinline__ void cross3(float ax, float ay, float az, float bx, float by, float bz, float& cx,
                                       float& cy, float& cz) {
  cx = ay * bz - az * by;
  cy = az * bx - ax * bz;
  cz = ax * by - ay * bx;
}

template <class Pose>
__global__ void k_e_body_rebuild(const float4* __restrict__ blocal, const Pose* __restrict__ poses,
                                 float4* __restrict__ pos, float4* __restrict__ vel,
                                 const uint32_t* __restrict__ slot_of, float4* __restrict__ bpos,
                                 uint32_t* __restrict__ bbox_acc, uint32_t base, uint32_t nf, uint32_t nb) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = q < nb;
  float x = 0, y = 0, z = 0;
  if (valid) {
    const uint32_t g = base + nf + q;
    const float4 L = blocal[g];
    const Pose P = poses[__float_as_uint(L.w)];
    float tx, ty, tz;
    cross3(P.qx, P.qy, P.qz, L.x, L.y, L.z, tx, ty, tz);
    tx = tx * 2.0f;
    ty = ty * 2.0f;
    tz = tz * 2.0f;
    float ux, uy, uz;
    cross3(P.qx, P.qy, P.qz, tx, ty, tz, ux, uy, uz);
    const float rx = (L.x + ux) + tx * P.qw;
    const float ry = (L.y + uy) + ty * P.qw;
    const float rz = (L.z + uz) + tz * P.qw;
    x = P.px + rx;
    y = P.py + ry;
    z = P.pz + rz;
    float ax, ay, az;
    cross3(P.wx, P.wy, P.wz, x - P.px, y - P.py, z - P.pz, ax, ay, az);
    const uint32_t s = slot_of[g];
    float4 p = pos[s];
    p.x = x;
    p.y = y;
    p.z = z;
    pos[s] = p;
    vel[s] = make_float4(P.vx + ax, P.vy + ay, P.vz + az, 0.0f);
    bpos[g] = make_float4(x, y, z, 0.0f);
  }
  block_bbox_accumulate(bbox_acc, x, y, z, valid);
}

__global__ void k_e_move(const float4* __restrict__ pos_in, const float4* __restrict__ vel_in,
                         const uint32_t* __restrict__ orig_in, const float4* __restrict__ bpos_in,
                         float4* __restrict__ pos_out, float4* __restrict__ vel_out, uint32_t* __restrict__ orig_out,
                         float4* __restrict__ bpos_out, const uint4* __restrict__ moves) {
  const uint4 m = moves[blockIdx.y];  // from, to, count, -
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m.z; i += gridDim.x * blockDim.x) {
    pos_out[m.y + i] = pos_in[m.x + i];
    vel_out[m.y + i] = vel_in[m.x + i];
    orig_out[m.y + i] = orig_in[m.x + i] - m.x + m.y;
    bpos_out[m.y + i] = bpos_in[m.x + i];
  }
}

__global__ void k_e_slot_of(const uint32_t* __restrict__ orig, uint32_t* __restrict__ slot_of, uint32_t n) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) slot_of[orig[s]] = s;
}

// ---------------------------------------------------------------- substep kernels

// Grid boxes and cell offsets (one block, any scene count): each scene's grid for this
// substep (crates/vxl-phys-fluid/src/grid.rs:37-44 -> crates/vxl-phys-core/src/grid.rs:34-50)
// from its AABB accumulators, which are then reset for the force pass's epilogue; then an
// exclusive scan of the scenes' cell counts;
// flags the substep when the total exceeds the cell capacity (every later kernel then
// returns without touching memory).
__global__ void k_e_celloff(SceneDev* __restrict__ sc, uint32_t nscenes, EngineCtl* ctl, uint32_t cell_cap) {
  __shared__ uint32_t sh[1024];
  __shared__ unsigned long long carry;
  __shared__ uint32_t doubled;
  if (threadIdx.x == 0) {
    carry = 0;
    doubled = 0;
  }
  if (threadIdx.x < kWorkSlots) ctl->work[threadIdx.x] = 0;  // persistent-pass counters of this substep
  if (threadIdx.x == 0) ctl->epoch = ctl->epoch + 1u;
  __syncthreads();
  for (uint32_t b0 = 0; b0 < nscenes; b0 += 1024) {
    const uint32_t q = b0 + threadIdx.x;
    uint32_t v = 0;
    if (q < nscenes) {
      // this substep's grid from the AABB accumulators (the reference's rule on all of the
      // scene's particles, crates/vxl-phys-core/src/grid.rs:34-50); reset the fluid one
      SceneDev& s = sc[q];
      float lo[3], hi[3];
      for (int a = 0; a < 3; ++a) {
        lo[a] = fminf(o2f(s.fbox[a]), o2f(s.bbox[a]));
        hi[a] = fmaxf(o2f(s.fbox[3 + a]), o2f(s.bbox[3 + a]));
      }
      GridBox g;
      if (!grid_box(lo[0], lo[1], lo[2], hi[0], hi[1], hi[2], s.k.h, s.k.max_bins, g))
        atomicOr(&ctl->err, kErrGridLoop);
      s.g = g;
      s.cells = g.total;
      for (int a = 0; a < 3; ++a) {
        s.fbox[a] = 0xffffffffu;
        s.fbox[3 + a] = 0u;
      }
      if (g.bin >= 2.0f * s.k.h) doubled = 1;
      v = g.total;
    }
    sh[threadIdx.x] = v;
    __syncthreads();
    for (uint32_t off = 1; off < 1024; off <<= 1) {
      const uint32_t add = threadIdx.x >= off ? sh[threadIdx.x - off] : 0u;
      __syncthreads();
      sh[threadIdx.x] += add;
      __syncthreads();
    }
    const unsigned long long ex = carry + (unsigned long long)(sh[threadIdx.x] - v);
    if (q < nscenes) sc[q].cell_off = ex > 0xffffffffull ? 0xffffffffu : (uint32_t)ex;
    __syncthreads();
    if (threadIdx.x == 1023) carry += sh[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    ctl->doubled = doubled;
    if (carry > (unsigned long long)cell_cap) {
      atomicOr(&ctl->err, kErrCellCap);
      ctl->cells = 0;
    } else {
      ctl->cells = (uint32_t)carry;
    }
  }
}

// Cell key + arrival rank per slot (tiles, one block per tile in turn). Lanes with equal
// keys share one atomic (warp-aggregated); the rank is only a placement ticket — canon
// makes the final order deterministic. Cells holding a fluid particle get wet[c] = epoch.
__global__ void k_e_keys(const float4* __restrict__ pos, const SceneDev* __restrict__ sc,
                         const TileDev* __restrict__ tiles, uint32_t ntiles, const EngineCtl* __restrict__ ctl,
                         uint32_t* __restrict__ counts, uint2* __restrict__ cellrank, uint32_t* __restrict__ halves,
                         uint32_t half_words, uint32_t* __restrict__ wet) {
  if (ctl->err & kErrCellCap) return;
  const uint32_t epoch = ctl->epoch;
  if (ctl->doubled)  // clear the half-cell masks that k_e_halfmask fills after the sort
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < half_words; w += gridDim.x * blockDim.x)
      halves[w] = 0u;
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const TileDev td = tiles[t];
    const GridBox g = sc[td.scene].g;
    const uint32_t off = sc[td.scene].cell_off;
    for (uint32_t b0 = 0; b0 < td.count; b0 += blockDim.x) {
      const uint32_t i = b0 + threadIdx.x;
      const bool valid = i < td.count;
      uint32_t c = 0xffffffffu;
      if (valid) {
        const float4 p = pos[td.first + i];
        c = off + cell_index(g, p.x, p.y, p.z);
        if (p.w > 0.0f) wet[c] = epoch;
      }
      const uint32_t active = __ballot_sync(0xffffffffu, valid);
      if (valid) {
        const uint32_t peers = __match_any_sync(active, c);
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(&counts[c], (uint32_t)__popc(peers));
        base = __shfl_sync(peers, base, leader);
        cellrank[td.first + i] = make_uint2(c, base + __popc(peers & ((1u << lane) - 1u)));
      }
    }
  }
}

// Phases 1-2 of the scan: per-tile sums of the counts (tiles of kScanTile cells,
// grid-stride), then, in whichever block finishes last (an atomic count of finished blocks;
// nothing waits), the exclusive scan of the tile sums in place and the total into
// start[cells].
__global__ void k_e_scan_partial(const uint32_t* __restrict__ counts, EngineCtl* ctl,
                                 uint32_t* __restrict__ partial, uint32_t* __restrict__ start) {
  if (ctl->err & kErrCellCap) return;
  const uint32_t total = ctl->cells;
  __shared__ uint32_t ws[kScanThreads / 32];
  for (uint32_t tile = blockIdx.x; (size_t)tile * kScanTile < total; tile += gridDim.x) {
    const uint32_t base = tile * kScanTile;
    uint32_t sum = 0;
    for (uint32_t i = base + threadIdx.x; i < min(base + kScanTile, total); i += kScanThreads) sum += counts[i];
    for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t t = 0;
      for (int w = 0; w < kScanThreads / 32; ++w) t += ws[w];
      partial[tile] = t;
    }
    __syncthreads();
  }
  __shared__ uint32_t last;
  if (threadIdx.x == 0) {
    __threadfence();  // this block's tile sums are visible before it counts itself done
    last = atomicAdd(&ctl->work[kWorkScan], 1u) == gridDim.x - 1 ? 1u : 0u;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  const uint32_t ntiles = (total + kScanTile - 1) / kScanTile;
  __shared__ uint32_t sh[kScanThreads];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t b0 = 0; b0 < ntiles; b0 += kScanThreads) {
    const uint32_t t = b0 + threadIdx.x;
    const uint32_t v = t < ntiles ? __ldcg(partial + t) : 0u;  // written by other blocks: skip L1
    sh[threadIdx.x] = v;
    __syncthreads();
    for (uint32_t off = 1; off < kScanThreads; off <<= 1) {
      const uint32_t add = threadIdx.x >= off ? sh[threadIdx.x - off] : 0u;
      __syncthreads();
      sh[threadIdx.x] += add;
      __syncthreads();
    }
    if (t < ntiles) partial[t] = carry + sh[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == kScanThreads - 1) carry += sh[kScanThreads - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) start[total] = carry;
}
// Phase 3: per-tile exclusive scan + tile offset -> start; zero counts for the next substep.
__global__ void k_e_scan_final(uint32_t* __restrict__ counts, const EngineCtl* __restrict__ ctl,
                               const uint32_t* __restrict__ partial, uint32_t* __restrict__ start) {
  if (ctl->err & kErrCellCap) return;
  const uint32_t total = ctl->cells;
  constexpr int kPer = kScanTile / kScanThreads;
  __shared__ uint32_t ws[kScanThreads / 32];
  for (uint32_t tile = blockIdx.x; (size_t)tile * kScanTile < total; tile += gridDim.x) {
    const uint32_t i0 = tile * kScanTile + threadIdx.x * kPer;
    uint32_t v[kPer], local = 0;
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
      v[q] = (i0 + q) < total ? counts[i0 + q] : 0u;
      local += v[q];
    }
    uint32_t incl = local;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, off);
      if (lane >= off) incl += y;
    }
    if (lane == 31) ws[wid] = incl;
    __syncthreads();
    uint32_t woff = 0;
    for (int w = 0; w < wid; ++w) woff += ws[w];
    uint32_t run = partial[tile] + woff + incl - local;
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
      if ((i0 + q) < total) {
        start[i0 + q] = run;
        counts[i0 + q] = 0u;
      }
      run += v[q];
    }
    __syncthreads();
  }
}

// Place each slot's (reference index, old slot) at start[cell] + rank (tiles).
__global__ void k_e_place(const uint2* __restrict__ cellrank, const uint32_t* __restrict__ start,
                          const uint32_t* __restrict__ orig, const TileDev* __restrict__ tiles, uint32_t ntiles,
                          const EngineCtl* __restrict__ ctl, uint2* __restrict__ items) {
  if (ctl->err & kErrCellCap) return;
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const TileDev td = tiles[t];
    for (uint32_t i = threadIdx.x; i < td.count; i += blockDim.x) {
      const uint32_t s = td.first + i;
      const uint2 cr = cellrank[s];
      items[start[cr.x] + cr.y] = make_uint2(orig[s], s);
    }
  }
}

// Per cell: order the placed entries by reference index (grid.rs:56-62) and gather
// position/velocity into the sorted buffer. A warp scans 32 consecutive cells at a time
// and handles each non-empty one cooperatively; rank = entries with a smaller index.
__device__ __forceinline__ void canon_cell(uint32_t b, uint32_t n, int lane, uint32_t* skeys, EngineCtl* ctl,
                                           const uint2* __restrict__ items, const float4* __restrict__ pos_in,
                                           const float4* __restrict__ vel_in, float4* __restrict__ pos_out,
                                           float4* __restrict__ vel_out, uint32_t* __restrict__ orig,
                                           uint32_t* __restrict__ slot_of) {
  if (n <= 32) {
    uint2 it = make_uint2(0xffffffffu, 0u);
    if ((uint32_t)lane < n) it = items[b + lane];
    uint32_t rank = 0;
    for (uint32_t j = 0; j < n; ++j) {
      const uint32_t kj = __shfl_sync(0xffffffffu, it.x, j);
      rank += (kj < it.x) ? 1u : 0u;
    }
    if ((uint32_t)lane < n) {
      const uint32_t dst = b + rank;
      pos_out[dst] = pos_in[it.y];
      vel_out[dst] = vel_in[it.y];
      orig[dst] = it.x;
      slot_of[it.x] = dst;
    }
  } else if (n <= (uint32_t)kCanonSmem / 2) {
    // keys and source slots both staged, so the cell's entries are read from memory once
    uint32_t* sslot = skeys + kCanonSmem / 2;
    for (uint32_t e = lane; e < n; e += 32) {
      const uint2 it = items[b + e];
      skeys[e] = it.x;
      sslot[e] = it.y;
    }
    __syncwarp();
    for (uint32_t e = lane; e < n; e += 32) {
      const uint32_t key = skeys[e], src = sslot[e];
      uint32_t rank = 0;
      for (uint32_t j = 0; j < n; ++j) rank += (skeys[j] < key) ? 1u : 0u;
      const uint32_t dst = b + rank;
      pos_out[dst] = pos_in[src];
      vel_out[dst] = vel_in[src];
      orig[dst] = key;
      slot_of[key] = dst;
    }
    __syncwarp();
  } else if (n <= (uint32_t)kCanonSmem) {
    for (uint32_t e = lane; e < n; e += 32) skeys[e] = items[b + e].x;
    __syncwarp();
    for (uint32_t e = lane; e < n; e += 32) {
      const uint2 it = items[b + e];
      uint32_t rank = 0;
      for (uint32_t j = 0; j < n; ++j) rank += (skeys[j] < it.x) ? 1u : 0u;
      const uint32_t dst = b + rank;
      pos_out[dst] = pos_in[it.y];
      vel_out[dst] = vel_in[it.y];
      orig[dst] = it.x;
      slot_of[it.x] = dst;
    }
    __syncwarp();
  } else {
    if (lane == 0) atomicOr(&ctl->err, kErrCanonLarge);
    for (uint32_t e = lane; e < n; e += 32) {
      const uint2 it = items[b + e];
      uint32_t rank = 0;
      for (uint32_t j = 0; j < n; ++j) rank += (items[b + j].x < it.x) ? 1u : 0u;
      const uint32_t dst = b + rank;
      pos_out[dst] = pos_in[it.y];
      vel_out[dst] = vel_in[it.y];
      orig[dst] = it.x;
      slot_of[it.x] = dst;
    }
  }
}

__global__ void k_e_canon(const uint2* __restrict__ items, const uint32_t* __restrict__ start, EngineCtl* ctl,
                          const float4* __restrict__ pos_in, const float4* __restrict__ vel_in,
                          float4* __restrict__ pos_out, float4* __restrict__ vel_out, uint32_t* __restrict__ orig,
                          uint32_t* __restrict__ slot_of) {
  __shared__ uint32_t skeys[8][kCanonSmem];
  if (ctl->err & kErrCellCap) return;
  const uint32_t total = ctl->cells;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32u; base < total; base += warps * 32u) {
    const uint32_t c = base + lane;
    uint32_t b = 0, n = 0;
    if (c < total) {
      b = start[c];
      n = start[c + 1] - b;
    }
    // Window path: the entries of these 32 cells are contiguous; when they are few and every
    // cell is small, rank and gather them 32 at a time across cell boundaries, with the
    // keys and a per-entry (cell start, cell size) table in shared memory.
    const uint32_t wb = __shfl_sync(0xffffffffu, b, 0);
    uint32_t we = c < total ? b + n : 0u;
    uint32_t maxn = n;
    for (int off = 16; off > 0; off >>= 1) {
      we = max(we, __shfl_xor_sync(0xffffffffu, we, off));
      maxn = max(maxn, __shfl_xor_sync(0xffffffffu, maxn, off));
    }
    if (maxn <= 32 && we - wb <= (uint32_t)kCanonWindow) {
      uint32_t* wkeys = skeys[wib];
      uint32_t* wseg = skeys[wib] + kCanonWindow;
      const uint32_t rel = b - wb;
      for (uint32_t q = 0; q < n; ++q) wseg[rel + q] = (rel << 6) | n;  // n <= 32 < 64
      const uint32_t T = we - wb;
      for (uint32_t e = lane; e < T; e += 32) wkeys[e] = items[wb + e].x;
      __syncwarp();
      for (uint32_t e = lane; e < T; e += 32) {
        const uint2 it = items[wb + e];
        const uint32_t seg = wseg[e];
        const uint32_t s0 = seg >> 6, sn = seg & 63u;
        uint32_t rank = 0;
        for (uint32_t j = 0; j < sn; ++j) rank += (wkeys[s0 + j] < it.x) ? 1u : 0u;
        const uint32_t dst = wb + s0 + rank;
        pos_out[dst] = pos_in[it.y];
        vel_out[dst] = vel_in[it.y];
        orig[dst] = it.x;
        slot_of[it.x] = dst;
      }
      __syncwarp();
      continue;
    }
    uint32_t mask = __ballot_sync(0xffffffffu, n > 0);
    while (mask) {
      const int l = __ffs(mask) - 1;
      mask &= mask - 1;
      const uint32_t cb = __shfl_sync(0xffffffffu, b, l);
      const uint32_t cn = __shfl_sync(0xffffffffu, n, l);
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
// far above the f32 rounding of cell faces and bin assignment. `start` is the scene's
// slice of the global cell table. With kSkipSelf, slot `self` is left out of the walk (it
// can only lie in the centre cell, so only that cell's loop tests for it). kCompact walks
// the same cells in the same order from a 27-bit mask built up front: fewer live registers
// (measured: the force pass's fallback walk and the boundary gather run 9-10% faster with
// it), but slower as the density pass's main loop (0.64 vs 0.47 ms on the 1M scene).
template <bool kSkipSelf = false, bool kCompact = false, class F>
__device__ __forceinline__ void walk27(const GridBox& g, const uint32_t* __restrict__ start, float px, float py,
                                       float pz, uint32_t cx, uint32_t cy, uint32_t cz, float h, F&& f,
                                       uint32_t self = ~0u) {
  const float lx = g.minx + (float)cx * g.bin, ly = g.miny + (float)cy * g.bin, lz = g.minz + (float)cz * g.bin;
  const float gxl = fmaxf(px - lx, 0.0f), gxr = fmaxf(lx + g.bin - px, 0.0f);
  const float gyl = fmaxf(py - ly, 0.0f), gyr = fmaxf(ly + g.bin - py, 0.0f);
  const float gzl = fmaxf(pz - lz, 0.0f), gzr = fmaxf(lz + g.bin - pz, 0.0f);
  const float reach = h + g.bin * (1.0f / 1024.0f);
  const float reach2 = reach * reach;
  if constexpr (kCompact) {
    uint32_t vm = 0;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz) {
      const bool zok = dz < 0 ? cz > 0 : (dz > 0 ? cz + 1 < g.nz : true);
      const float gz = dz < 0 ? gzl : (dz > 0 ? gzr : 0.0f);
      const float dz2 = gz * gz;
#pragma unroll
      for (int dy = -1; dy <= 1; ++dy) {
        const bool yok = dy < 0 ? cy > 0 : (dy > 0 ? cy + 1 < g.ny : true);
        const float gy = dy < 0 ? gyl : (dy > 0 ? gyr : 0.0f);
        const float dyz2 = dz2 + gy * gy;
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
          const bool xok = dx < 0 ? cx > 0 : (dx > 0 ? cx + 1 < g.nx : true);
          const float gx = dx < 0 ? gxl : (dx > 0 ? gxr : 0.0f);
          if (zok && yok && xok && !(dyz2 + gx * gx > reach2)) vm |= 1u << ((dz + 1) * 9 + (dy + 1) * 3 + (dx + 1));
        }
      }
    }
    const int nz = (int)g.nz, nyz = (int)(g.ny * g.nz);
    const int centre = (int)(((cx * g.ny) + cy) * g.nz + cz);
    while (vm) {
      const int d = __ffs(vm) - 1;
      vm &= vm - 1u;
      const int dzp = d / 9, rem = d - 9 * dzp, dyp = rem / 3, dxp = rem - 3 * dyp;
      const uint32_t idx = (uint32_t)(centre + (dxp - 1) * nyz + (dyp - 1) * nz + (dzp - 1));
      const uint32_t j1 = start[idx + 1];
      if (kSkipSelf && d == 13) {
        for (uint32_t j = start[idx]; j < j1; ++j)
          if (j != self) f(j);
      } else {
        for (uint32_t j = start[idx]; j < j1; ++j) f(j);
      }
    }
  } else {
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
          if (kSkipSelf && dz == 0 && dy == 0 && dx == 0) {
            for (uint32_t j = start[idx]; j < j1; ++j)
              if (j != self) f(j);
          } else {
            for (uint32_t j = start[idx]; j < j1; ++j) f(j);
          }
        }
      }
    }
  }
}

// Compact neighbour-list entries. Every neighbour of a particle in cell (cx, cy, cz) lies in
// one of the three x-planes x = cx - 1, cx, cx + 1 of its 27 cells, and inside plane x its
// slot is at least the first slot of cell (x, max(cy - 1, 0), max(cz - 1, 0)) — cell indices
// grow with x, y, z and the table is sorted by cell — and below the next plane's first
// slot. A list entry is (plane << 14) | (slot - plane's first slot), 16 bits; a neighbour
// 16,384 or more slots past its plane's first slot cannot be encoded, and its list is then
// marked unusable (bit 31 of the count) so that the consumers walk the cells again.
constexpr uint32_t kListBad = 0x80000000u;
constexpr uint32_t kListOffBits = 14;
constexpr uint32_t kListOffMask = (1u << kListOffBits) - 1u;

struct ListPlanes {
  uint32_t b0, b1, b2;  // first slot of plane cx - 1 (= b1 at the grid's edge), cx, cx + 1 (~0u if none)
};

__device__ __forceinline__ ListPlanes list_planes(const GridBox& g, const uint32_t* __restrict__ cst, uint32_t cx,
                                                  uint32_t cy, uint32_t cz) {
  const uint32_t ylo = cy > 0 ? cy - 1 : 0, zlo = cz > 0 ? cz - 1 : 0;
  const uint32_t yz = ylo * g.nz + zlo, nyz = g.ny * g.nz;
  ListPlanes lp;
  lp.b1 = cst[cx * nyz + yz];
  lp.b0 = cx > 0 ? cst[(cx - 1) * nyz + yz] : lp.b1;
  lp.b2 = cx + 1 < g.nx ? cst[(cx + 1) * nyz + yz] : 0xffffffffu;
  return lp;
}

// Entry of neighbour slot j, or 0xffffffff if it cannot be encoded.
__device__ __forceinline__ uint32_t list_encode(const ListPlanes& lp, uint32_t j) {
  const uint32_t pl = (j >= lp.b1 ? 1u : 0u) + (j >= lp.b2 ? 1u : 0u);
  const uint32_t off = j - (pl == 0u ? lp.b0 : (pl == 1u ? lp.b1 : lp.b2));
  return off > kListOffMask ? 0xffffffffu : (pl << kListOffBits) | off;
}

__device__ __forceinline__ uint32_t list_decode(const ListPlanes& lp, uint32_t e) {
  const uint32_t pl = e >> kListOffBits;
  return (pl == 0u ? lp.b0 : (pl == 1u ? lp.b1 : lp.b2)) + (e & kListOffMask);
}

// Half-cell masks of the sorted slots, for the density walk: for each aligned block of 32
// slots, halves[4 * (s >> 5) + a] has bit (s & 31) set iff slot s lies at or above the
// midplane of its own cell along axis a (x, y, z). One thread per slot over tiles;
// lanes that share a block and axis combine their bits before one atomicOr.
__global__ void k_e_halfmask(const float4* __restrict__ pos, const SceneDev* __restrict__ sc,
                             const TileDev* __restrict__ tiles, uint32_t ntiles, const EngineCtl* __restrict__ ctl,
                             uint32_t* __restrict__ halves) {
  if ((ctl->err & kErrCellCap) || !ctl->doubled) return;
  const int lane = threadIdx.x & 31;
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const TileDev td = tiles[t];
    const GridBox g = sc[td.scene].g;
    if (g.bin < 2.0f * sc[td.scene].k.h) continue;  // the density pass walks this scene unmasked
    const float hb = g.bin * 0.5f;
    for (uint32_t b0 = 0; b0 < td.count; b0 += blockDim.x) {
      const uint32_t i = b0 + threadIdx.x;
      const bool valid = i < td.count;
      uint32_t blk = 0xffffffffu, bit = 0, hx = 0, hy = 0, hz = 0;
      if (valid) {
        const uint32_t s = td.first + i;
        const float4 p = pos[s];
        uint32_t cx, cy, cz;
        bin_of(g, p.x, p.y, p.z, cx, cy, cz);
        hx = p.x >= g.minx + (float)cx * g.bin + hb;
        hy = p.y >= g.miny + (float)cy * g.bin + hb;
        hz = p.z >= g.minz + (float)cz * g.bin + hb;
        blk = s >> 5;
        bit = 1u << (s & 31);
      }
      const uint32_t active = __ballot_sync(0xffffffffu, valid);
      if (valid) {
        const uint32_t peers = __match_any_sync(active, blk);
        const uint32_t mx = __reduce_or_sync(peers, hx ? bit : 0u);
        const uint32_t my = __reduce_or_sync(peers, hy ? bit : 0u);
        const uint32_t mz = __reduce_or_sync(peers, hz ? bit : 0u);
        if (lane == __ffs(peers) - 1) {
          if (mx) atomicOr(&halves[4 * blk], mx);
          if (my) atomicOr(&halves[4 * blk + 1], my);
          if (mz) atomicOr(&halves[4 * blk + 2], mz);
        }
      }
    }
  }
}

// Thread order of the half-culled density walk: within each cell, the slots in the lower x
// half first, then those in the upper half (each group in slot order), from the half-cell
// masks. At 2h bins a particle's reachable halves follow from the halves it lies in, so a
// warp whose lanes share their x half skips the x-side cells its lanes cannot reach together
// (every lane in the lower half leaves the +x cells out) instead of idling through them.
// order[p] is the slot the density pass processes at position p; it permutes each cell's own
// slots, so every slot is processed once and each result is unchanged. One warp per cell.
__global__ void k_e_xorder(const uint32_t* __restrict__ start, const EngineCtl* __restrict__ ctl,
                           const uint32_t* __restrict__ halves, uint32_t* __restrict__ order) {
  if ((ctl->err & kErrCellCap) || !ctl->doubled) return;
  const uint32_t total = ctl->cells;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < total; c += nw) {
    const uint32_t b = start[c], n = start[c + 1] - b;
    uint32_t nlow = 0;
    for (uint32_t k0 = 0; k0 < n; k0 += 32) {
      const uint32_t sl = b + k0 + lane;
      const bool valid = k0 + lane < n;
      const bool up = valid && ((halves[4 * (sl >> 5)] >> (sl & 31)) & 1u);
      nlow += __popc(__ballot_sync(0xffffffffu, valid && !up));
    }
    uint32_t lo = 0, hi = 0;
    for (uint32_t k0 = 0; k0 < n; k0 += 32) {
      const uint32_t sl = b + k0 + lane;
      const bool valid = k0 + lane < n;
      const bool up = valid && ((halves[4 * (sl >> 5)] >> (sl & 31)) & 1u);
      const uint32_t ml = __ballot_sync(0xffffffffu, valid && !up);
      const uint32_t mh = __ballot_sync(0xffffffffu, up);
      if (valid) order[b + (up ? nlow + hi + __popc(mh & lt) : lo + __popc(ml & lt))] = sl;
      lo += __popc(ml);
      hi += __popc(mh);
    }
  }
}

// Per axis, which halves of the three cells (d = -1, 0, +1) along it a particle at p can
// reach: bit 2 (d + 1) for the lower half, bit 2 (d + 1) + 1 for the upper half. A half is
// dropped only when the gap from p to its nominal interval exceeds `reach` (h plus a
// margin far above the rounding of cell faces and midplanes). `last`: p's cell is the last
// on this axis, whose upper half also holds the particles clamped into it from beyond the
// grid (an axis at the 16,384-cell cap), p possibly among them: that half has no upper face.
// (No particle lies below the grid's lower corner, the scene AABB's minimum.)
__device__ __forceinline__ uint32_t half_reach_bits(float p, float l, float B, float reach, bool last) {
  const float hb = B * 0.5f;
  const float gm_lo = fmaxf(p - (l - hb), 0.0f);
  const float gm_hi = fmaxf(p - l, 0.0f);
  const float g0_lo = fmaxf(fmaxf(l - p, p - (l + hb)), 0.0f);
  const float g0_hi = fmaxf(fmaxf((l + hb) - p, last ? 0.0f : p - (l + B)), 0.0f);
  const float gp_lo = fmaxf((l + B) - p, 0.0f);
  const float gp_hi = fmaxf((l + B + hb) - p, 0.0f);
  return (gm_lo <= reach ? 1u : 0u) | (gm_hi <= reach ? 2u : 0u) | (g0_lo <= reach ? 4u : 0u) |
         (g0_hi <= reach ? 8u : 0u) | (gp_lo <= reach ? 16u : 0u) | (gp_hi <= reach ? 32u : 0u);
}

// Slot mask of the particles in a block whose half along one axis is reachable.
__device__ __forceinline__ uint32_t half_select(uint32_t two_bits, uint32_t upper) {
  return two_bits == 3u ? 0xffffffffu : (two_bits == 2u ? upper : ~upper);
}

// walk27 with half-cell culling: the same cells in the same order, and inside each cell
// the same slots in ascending order, except slots lying in a half-cell (along any axis)
// farther than h from p — they cannot be accepted, so the accepted set and its order are
// unchanged. Used when the grid's bins are at least 2h (the reference's cell budget
// doubled them), where a particle reaches only about a quarter of the 27 cells' slots.
template <class F>
__device__ __forceinline__ void walk27_half(const GridBox& g, const uint32_t* __restrict__ start,
                                            const uint32_t* __restrict__ halves, float px, float py, float pz,
                                            uint32_t cx, uint32_t cy, uint32_t cz, float h, F&& f) {
  const float B = g.bin;
  const float lx = g.minx + (float)cx * B, ly = g.miny + (float)cy * B, lz = g.minz + (float)cz * B;
  const float gxl = fmaxf(px - lx, 0.0f), gxr = fmaxf(lx + B - px, 0.0f);
  const float gyl = fmaxf(py - ly, 0.0f), gyr = fmaxf(ly + B - py, 0.0f);
  const float gzl = fmaxf(pz - lz, 0.0f), gzr = fmaxf(lz + B - pz, 0.0f);
  const float reach = h + B * (1.0f / 1024.0f);
  const float reach2 = reach * reach;
  const uint32_t bxs = half_reach_bits(px, lx, B, reach, cx + 1 == g.nx);
  const uint32_t bys = half_reach_bits(py, ly, B, reach, cy + 1 == g.ny);
  const uint32_t bzs = half_reach_bits(pz, lz, B, reach, cz + 1 == g.nz);
  for (int dz = -1; dz <= 1; ++dz) {
    const int z = (int)cz + dz;
    if (z < 0 || z >= (int)g.nz) continue;
    const float gz = dz < 0 ? gzl : (dz > 0 ? gzr : 0.0f);
    const float dz2 = gz * gz;
    const uint32_t zsel = (bzs >> (2 * (dz + 1))) & 3u;
    for (int dy = -1; dy <= 1; ++dy) {
      const int y = (int)cy + dy;
      if (y < 0 || y >= (int)g.ny) continue;
      const float gy = dy < 0 ? gyl : (dy > 0 ? gyr : 0.0f);
      const float dyz2 = dz2 + gy * gy;
      const uint32_t ysel = (bys >> (2 * (dy + 1))) & 3u;
      for (int dx = -1; dx <= 1; ++dx) {
        const int x = (int)cx + dx;
        if (x < 0 || x >= (int)g.nx) continue;
        const float gx = dx < 0 ? gxl : (dx > 0 ? gxr : 0.0f);
        if (dyz2 + gx * gx > reach2) continue;
        const uint32_t xsel = (bxs >> (2 * (dx + 1))) & 3u;
        if (!xsel || !ysel || !zsel) continue;
        const uint32_t idx = ((uint32_t)x * g.ny + (uint32_t)y) * g.nz + (uint32_t)z;
        const uint32_t j0 = start[idx], j1 = start[idx + 1];
        for (uint32_t base = j0 & ~31u; base < j1; base += 32) {
          const uint4 hm = *reinterpret_cast<const uint4*>(halves + 4 * (base >> 5));
          uint32_t m = half_select(xsel, hm.x) & half_select(ysel, hm.y) & half_select(zsel, hm.z);
          if (j0 > base) m &= ~0u << (j0 - base);
          if (j1 < base + 32) m &= (1u << (j1 - base)) - 1u;
          while (m) {
            const uint32_t j = base + (uint32_t)(__ffs(m) - 1);
            m &= m - 1u;
            f(j);
          }
        }
      }
    }
  }
}

// walk27 / walk27_half with a hook per cell and the slot `skip` left out: f(j) for every
// candidate in the same order; before a cell's candidates, fc(plane, end) with the cell's
// x-plane (dx + 1) and its end slot.
template <class FC, class F>
__device__ __forceinline__ void walk27_c(const GridBox& g, const uint32_t* __restrict__ start, float px, float py,
                                         float pz, uint32_t cx, uint32_t cy, uint32_t cz, float h, uint32_t skip,
                                         FC&& fc, F&& f) {
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
        fc((uint32_t)(dx + 1), j1);
        for (uint32_t j = start[idx]; j < j1; ++j)
          if (j != skip) f(j);
      }
    }
  }
}

template <class FC, class F>
__device__ __forceinline__ void walk27_half_c(const GridBox& g, const uint32_t* __restrict__ start,
                                              const uint32_t* __restrict__ halves, float px, float py, float pz,
                                              uint32_t cx, uint32_t cy, uint32_t cz, float h, uint32_t skip,
                                              FC&& fc, F&& f) {
  const float B = g.bin;
  const float lx = g.minx + (float)cx * B, ly = g.miny + (float)cy * B, lz = g.minz + (float)cz * B;
  const float gxl = fmaxf(px - lx, 0.0f), gxr = fmaxf(lx + B - px, 0.0f);
  const float gyl = fmaxf(py - ly, 0.0f), gyr = fmaxf(ly + B - py, 0.0f);
  const float gzl = fmaxf(pz - lz, 0.0f), gzr = fmaxf(lz + B - pz, 0.0f);
  const float reach = h + B * (1.0f / 1024.0f);
  const float reach2 = reach * reach;
  const uint32_t bxs = half_reach_bits(px, lx, B, reach, cx + 1 == g.nx);
  const uint32_t bys = half_reach_bits(py, ly, B, reach, cy + 1 == g.ny);
  const uint32_t bzs = half_reach_bits(pz, lz, B, reach, cz + 1 == g.nz);
  for (int dz = -1; dz <= 1; ++dz) {
    const int z = (int)cz + dz;
    if (z < 0 || z >= (int)g.nz) continue;
    const float gz = dz < 0 ? gzl : (dz > 0 ? gzr : 0.0f);
    const float dz2 = gz * gz;
    const uint32_t zsel = (bzs >> (2 * (dz + 1))) & 3u;
    for (int dy = -1; dy <= 1; ++dy) {
      const int y = (int)cy + dy;
      if (y < 0 || y >= (int)g.ny) continue;
      const float gy = dy < 0 ? gyl : (dy > 0 ? gyr : 0.0f);
      const float dyz2 = dz2 + gy * gy;
      const uint32_t ysel = (bys >> (2 * (dy + 1))) & 3u;
      for (int dx = -1; dx <= 1; ++dx) {
        const int x = (int)cx + dx;
        if (x < 0 || x >= (int)g.nx) continue;
        const float gx = dx < 0 ? gxl : (dx > 0 ? gxr : 0.0f);
        if (dyz2 + gx * gx > reach2) continue;
        const uint32_t xsel = (bxs >> (2 * (dx + 1))) & 3u;
        if (!xsel || !ysel || !zsel) continue;
        const uint32_t idx = ((uint32_t)x * g.ny + (uint32_t)y) * g.nz + (uint32_t)z;
        const uint32_t j0 = start[idx], j1 = start[idx + 1];
        fc((uint32_t)(dx + 1), j1);
        // windows of 32 slots from the cell's own first slot, the half masks read across two
        // aligned words: lanes of one octant in different cells of similar contents then
        // take the same number of trips through each window
        for (uint32_t base = j0; base < j1; base += 32) {
          const uint32_t sh = base & 31u;
          const uint4 lo = *reinterpret_cast<const uint4*>(halves + 4 * (base >> 5));
          const uint4 hi = *reinterpret_cast<const uint4*>(halves + 4 * (base >> 5) + 4);
          const uint32_t ux = __funnelshift_r(lo.x, hi.x, sh), uy = __funnelshift_r(lo.y, hi.y, sh),
                         uz = __funnelshift_r(lo.z, hi.z, sh);
          uint32_t m = half_select(xsel, ux) & half_select(ysel, uy) & half_select(zsel, uz);
          if (j1 < base + 32) m &= (1u << (j1 - base)) - 1u;
          if (skip - base < 32u) m &= ~(1u << (skip - base));  // once per window, not per candidate
          while (m) {
            f(base + (uint32_t)(__ffs(m) - 1));
            m &= m - 1u;
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------- grouped density walk
//
// Particles of one cell reach the same neighbour cells; when the cell budget has doubled
// the bins to 2h or more, particles of one octant of a cell (the same half along x, y and
// z) also reach the same half-cells. The grouped density pass lets eight lanes of a warp
// share one stream of candidates: k_e_groups orders each chunk of a tile (up to
// kGroupChunk slots) by octant (a stable counting sort, so the slots of an octant stay
// ascending) into order[], then cuts the runs of equal (cell, octant) into segments of at
// most kSegLanes positions, appended to segs[] as (first position in order[], count |
// scene << 4); ctl->work[kWorkSegs] counts them. The order of segments in segs[] is
// immaterial: each particle's sums are formed by one lane alone.
//
// The per-particle walk runs in order[] too: a warp whose lanes share one octant walks one
// culled cell set. Octants follow one another in Gray-code order (0 1 3 2 6 7 5 4), so a
// warp that straddles two octants walks the union of two sets that differ along one axis
// only (12 cells instead of 8; up to 27 for octants apart in all three). A chunk holds 8
// octant runs, 7 boundaries over kGroupChunk / 32 warps; chunks of 512 slots (tiles of 512)
// let fewer warps straddle, but cost the grouping pass about as much as they save.

constexpr uint32_t kSegLanes = 8;   // lanes (particles) per segment; four segments per warp
constexpr uint32_t kSegQueue = 64;  // candidate ring per segment (pending never exceeds 7 + 32)
#ifndef VXL_GROUP_CHUNK
#define VXL_GROUP_CHUNK 256
#endif
constexpr uint32_t kGroupChunk = VXL_GROUP_CHUNK;  // slots per chunk = threads per block
static_assert(kGroupChunk % 128 == 0 && kGroupChunk <= 1024, "chunk: 128..1024 slots, whole warps");

__device__ __forceinline__ uint32_t octant_rank(uint32_t oct) { return oct ^ (oct >> 1) ^ (oct >> 2); }

__global__ void __launch_bounds__(kGroupChunk) k_e_groups(const float4* __restrict__ pos, const SceneDev* __restrict__ sc,
                                                          const TileDev* __restrict__ tiles, uint32_t ntiles, EngineCtl* ctl,
                                                          uint32_t* __restrict__ order, uint2* __restrict__ segs,
                                                          uint32_t* __restrict__ halves) {
  if (ctl->err & kErrCellCap) return;
  constexpr uint32_t kW = kGroupChunk / 32;  // warps
  constexpr uint32_t kV = 8 * kW / 32;       // (rank, warp) counts per lane of the scan
  __shared__ uint32_t s_cnt[8 * kW];         // [octant rank][warp]: slots per octant in each warp
  __shared__ uint32_t s_cell[kGroupChunk], s_oct[kGroupChunk];
  __shared__ uint32_t s_last[kW], s_nseg[kW], s_segbase;
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  // the block's chunks one after another, each one's positions loaded while the previous
  // one is sorted
  uint32_t t = blockIdx.x, c1 = 0;
  TileDev tn = t < ntiles ? tiles[t] : TileDev{};
  float4 pn = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (t < ntiles && threadIdx.x < tn.count) pn = pos[tn.first + threadIdx.x];
  while (t < ntiles) {  // uniform over the block
    const TileDev td = tn;
    const uint32_t c0 = c1;
    const float4 p = pn;
    c1 += kGroupChunk;
    if (c1 >= tn.count) {
      t += gridDim.x;
      c1 = 0;
      if (t < ntiles) tn = tiles[t];
    }
    if (t < ntiles && c1 + threadIdx.x < tn.count) pn = pos[tn.first + c1 + threadIdx.x];
    const GridBox g = sc[td.scene].g;
    const bool half = g.bin >= 2.0f * sc[td.scene].k.h;
    const float hb = g.bin * 0.5f;
    {
      const uint32_t n = min(kGroupChunk, td.count - c0);
      const uint32_t i = threadIdx.x;
      const bool valid = i < n;
      uint32_t cell = 0, oct = 0;
      if (valid) {
        uint32_t cx, cy, cz;
        bin_of(g, p.x, p.y, p.z, cx, cy, cz);
        cell = (cx * g.ny + cy) * g.nz + cz;
        if (half)
          oct = (p.x >= g.minx + (float)cx * g.bin + hb ? 1u : 0u) | (p.y >= g.miny + (float)cy * g.bin + hb ? 2u : 0u) |
                (p.z >= g.minz + (float)cz * g.bin + hb ? 4u : 0u);
      }
      // the half-cell masks of the density walk (what k_e_halfmask writes for the scenes
      // with provider walls): bit (s & 31) of halves[4 (s >> 5) + a] for the upper half
      if (half) {
        const uint32_t active = __ballot_sync(0xffffffffu, valid);
        if (valid) {
          const uint32_t s = td.first + c0 + i;
          const uint32_t blk = s >> 5, bit = 1u << (s & 31);
          const uint32_t peers = __match_any_sync(active, blk);
          const uint32_t mx = __reduce_or_sync(peers, (oct & 1u) ? bit : 0u);
          const uint32_t my = __reduce_or_sync(peers, (oct & 2u) ? bit : 0u);
          const uint32_t mz = __reduce_or_sync(peers, (oct & 4u) ? bit : 0u);
          if (lane == __ffs(peers) - 1) {
            if (mx) atomicOr(&halves[4 * blk], mx);
            if (my) atomicOr(&halves[4 * blk + 1], my);
            if (mz) atomicOr(&halves[4 * blk + 2], mz);
          }
        }
      }
      const uint32_t key = octant_rank(oct);
      uint32_t rank = 0;
#pragma unroll
      for (uint32_t o = 0; o < 8; ++o) {
        const uint32_t b = __ballot_sync(0xffffffffu, valid && key == o);
        if (lane == 0) s_cnt[o * kW + w] = __popc(b);
        if (valid && key == o) rank = __popc(b & lt);
      }
      __syncthreads();
      if (w == 0) {  // exclusive scan of the 8 * kW counts in (rank, warp) order
        uint32_t v[kV], tot = 0;
#pragma unroll
        for (uint32_t k = 0; k < kV; ++k) {
          v[k] = s_cnt[lane * kV + k];
          tot += v[k];
        }
        uint32_t incl = tot;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
          const uint32_t u = __shfl_up_sync(0xffffffffu, incl, off);
          if ((int)lane >= off) incl += u;
        }
        uint32_t ex = incl - tot;
#pragma unroll
        for (uint32_t k = 0; k < kV; ++k) {
          s_cnt[lane * kV + k] = ex;
          ex += v[k];
        }
      }
      __syncthreads();
      if (valid) {
        const uint32_t q = s_cnt[key * kW + w] + rank;
        order[td.first + c0 + q] = td.first + c0 + i;
        s_cell[q] = cell;
        s_oct[q] = oct;
      }
      __syncthreads();
      // runs of equal (cell, octant) in the new order, cut into segments of kSegLanes
      const bool head = valid && (i == 0 || s_cell[i] != s_cell[i - 1] || s_oct[i] != s_oct[i - 1]);
      const uint32_t hbal = __ballot_sync(0xffffffffu, head);
      if (lane == 0) s_last[w] = hbal ? w * 32 + 31 - __clz(hbal) : 0xffffffffu;
      __syncthreads();
      uint32_t run0 = 0;
      const uint32_t le = hbal & (0xffffffffu >> (31 - lane));
      if (le) {
        run0 = w * 32 + 31 - __clz(le);
      } else {
        for (int k = (int)w - 1; k >= 0; --k)
          if (s_last[k] != 0xffffffffu) {
            run0 = s_last[k];
            break;
          }
      }
      const bool shead = valid && ((i - run0) % kSegLanes == 0u);
      uint32_t cnt = 0;
      if (shead) {
        cnt = 1;
        while (cnt < kSegLanes && i + cnt < n && s_cell[i + cnt] == s_cell[i] && s_oct[i + cnt] == s_oct[i]) ++cnt;
      }
      const uint32_t sb = __ballot_sync(0xffffffffu, shead);
      if (lane == 0) s_nseg[w] = __popc(sb);
      __syncthreads();
      if (threadIdx.x == 0) {
        uint32_t tot = 0;
        for (uint32_t k = 0; k < kW; ++k) {
          const uint32_t v = s_nseg[k];
          s_nseg[k] = tot;
          tot += v;
        }
        s_segbase = atomicAdd(&ctl->work[kWorkSegs], tot);
      }
      __syncthreads();
      if (shead) segs[s_segbase + s_nseg[w] + __popc(sb & lt)] = make_uint2(td.first + c0 + i, cnt | (td.scene << 4));
      __syncthreads();
    }
  }
}

// Density (poly6 with self term) + Tait EOS over the segments of k_e_groups: the same
// sums as k_e_density (crates/vxl-phys-fluid/src/fluid_density.rs:17-70) for scenes
// without provider walls. Lanes 8k..8k+7 of a warp hold the particles of one segment,
// which share their cell. The segment's cells are the union of its lanes' culled 27-cell
// sets (and, at 2h bins, of their reachable half-cells) — for each lane a superset of its
// own walk that adds only particles farther than h — taken in the reference's (dz, dy, dx)
// order and, inside a cell, in ascending slot order (crates/vxl-phys-fluid/src/grid.rs:
// 115-155). The segment's eight lanes append the candidate slots to a ring in shared
// memory (each lane four bits of a 32-slot window), load eight of them at a time into a
// staging row, and every lane then tests its own particle against the row in order, so
// each lane accepts exactly its walk's neighbours in its walk's order: the sums, the EOS
// and the recorded neighbour list are those of k_e_density, bit for bit. Segments of one
// warp advance in lock step, eight candidates per round.
template <int kWarps>
__global__ void __launch_bounds__(kWarps * 32, VXL_DENSITY_SEG_THREADS_PER_SM / (kWarps * 32)) k_e_density_seg(
    const float4* __restrict__ pos, const uint32_t* __restrict__ start, const SceneDev* __restrict__ sc,
    const EngineCtl* __restrict__ ctl, const uint32_t* __restrict__ halves, const uint32_t* __restrict__ order,
    const uint2* __restrict__ segs, float2* __restrict__ rc, float* __restrict__ press_out, uint16_t* __restrict__ nbr,
    uint32_t* __restrict__ nbr_n, uint32_t cap, uint32_t stride, const uint32_t* __restrict__ wet) {
  if (ctl->err & kErrCellCap) return;
  __shared__ uint32_t s_queue[kWarps][4][kSegQueue];
  __shared__ float4 s_pos[kWarps][4 * (kSegLanes + 1)];  // rows padded by one: segments hit different banks
  __shared__ uint32_t s_j[kWarps][4 * (kSegLanes + 1)];
  const uint32_t nseg = ctl->work[kWorkSegs];
  const uint32_t epoch = ctl->epoch;
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t seg = lane >> 3, sl = lane & 7u;
  uint32_t* queue = s_queue[w][seg];
  float4* stp = &s_pos[w][seg * (kSegLanes + 1)];
  uint32_t* stj = &s_j[w][seg * (kSegLanes + 1)];
  const uint32_t nwarps = gridDim.x * kWarps;
  for (uint32_t g0 = (blockIdx.x * kWarps + w) * 4; g0 < nseg; g0 += nwarps * 4) {
    const uint32_t sid = g0 + seg;
    const uint2 rec = sid < nseg ? segs[sid] : make_uint2(0u, 0u);
    const uint32_t nseg_lanes = rec.y & 15u;
    const bool act = sl < nseg_lanes;
    const SceneDev& S = sc[rec.y >> 4];
    const GridBox g = S.g;
    const float h = S.k.h, h2 = S.k.h2, k6 = S.k.k6;
    const bool half = halves != nullptr && g.bin >= 2.0f * h;
    uint32_t s = 0;
    float4 pi = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    uint32_t cx = 0, cy = 0, cz = 0;
    if (act) {
      s = order[rec.x + sl];
      pi = pos[s];
      bin_of(g, pi.x, pi.y, pi.z, cx, cy, cz);
    }
    const bool fluid_i = pi.w > 0.0f;
    // this lane's cells: in the grid and not farther than h (conservatively, as walk27),
    // and at 2h bins with some reachable half along every axis (as walk27_half)
    uint32_t cm = 0, bxs = 0, bys = 0, bzs = 0;
    if (act) {
      const float lx = g.minx + (float)cx * g.bin, ly = g.miny + (float)cy * g.bin, lz = g.minz + (float)cz * g.bin;
      const float gxl = fmaxf(pi.x - lx, 0.0f), gxr = fmaxf(lx + g.bin - pi.x, 0.0f);
      const float gyl = fmaxf(pi.y - ly, 0.0f), gyr = fmaxf(ly + g.bin - pi.y, 0.0f);
      const float gzl = fmaxf(pi.z - lz, 0.0f), gzr = fmaxf(lz + g.bin - pi.z, 0.0f);
      const float reach = h + g.bin * (1.0f / 1024.0f);
      const float reach2 = reach * reach;
      if (half) {
        bxs = half_reach_bits(pi.x, lx, g.bin, reach, cx + 1 == g.nx);
        bys = half_reach_bits(pi.y, ly, g.bin, reach, cy + 1 == g.ny);
        bzs = half_reach_bits(pi.z, lz, g.bin, reach, cz + 1 == g.nz);
      } else {
        bxs = bys = bzs = 63u;
      }
#pragma unroll
      for (int dz = -1; dz <= 1; ++dz) {
        const bool zok = (dz < 0 ? cz > 0 : (dz > 0 ? cz + 1 < g.nz : true)) && ((bzs >> (2 * (dz + 1))) & 3u);
        const float gz = dz < 0 ? gzl : (dz > 0 ? gzr : 0.0f);
        const float dz2 = gz * gz;
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy) {
          const bool yok = (dy < 0 ? cy > 0 : (dy > 0 ? cy + 1 < g.ny : true)) && ((bys >> (2 * (dy + 1))) & 3u);
          const float gy = dy < 0 ? gyl : (dy > 0 ? gyr : 0.0f);
          const float dyz2 = dz2 + gy * gy;
#pragma unroll
          for (int dx = -1; dx <= 1; ++dx) {
            const bool xok = (dx < 0 ? cx > 0 : (dx > 0 ? cx + 1 < g.nx : true)) && ((bxs >> (2 * (dx + 1))) & 3u);
            const float gx = dx < 0 ? gxl : (dx > 0 ? gxr : 0.0f);
            if (zok && yok && xok && !(dyz2 + gx * gx > reach2)) cm |= 1u << ((dz + 1) * 9 + (dy + 1) * 3 + (dx + 1));
          }
        }
      }
    }
    // A segment of boundary particles only sums fluid neighbours: with no fluid in its
    // cell's 27 cells (none marked wet this substep) it has nothing to walk. The segment's
    // lanes share the cell, so they test the 27 cells together.
    const uint32_t seg_mask = 0xffu << (8 * seg);
    const bool seg_fluid = (__ballot_sync(0xffffffffu, act && fluid_i) & seg_mask) != 0u;
    const uint32_t lead = seg * 8;
    const uint32_t ccx = __shfl_sync(0xffffffffu, cx, lead), ccy = __shfl_sync(0xffffffffu, cy, lead),
                   ccz = __shfl_sync(0xffffffffu, cz, lead);
    bool wet_seen = seg_fluid;
    if (!seg_fluid && nseg_lanes) {
      const uint32_t* wc = wet + S.cell_off;
      for (uint32_t d = sl; d < 27u; d += 8u) {
        const int dz = (int)(d / 9) - 1, dy = (int)((d / 3) % 3) - 1, dx = (int)(d % 3) - 1;
        const int x = (int)ccx + dx, y = (int)ccy + dy, z = (int)ccz + dz;
        if (x >= 0 && x < (int)g.nx && y >= 0 && y < (int)g.ny && z >= 0 && z < (int)g.nz &&
            wc[((uint32_t)x * g.ny + (uint32_t)y) * g.nz + (uint32_t)z] == epoch)
          wet_seen = true;
      }
    }
    const bool seg_wet = (__ballot_sync(0xffffffffu, wet_seen) & seg_mask) != 0u;
    if (!seg_wet) cm = 0;
#pragma unroll
    for (uint32_t o = 1; o < 8; o <<= 1) {
      cm |= __shfl_xor_sync(0xffffffffu, cm, o);
      bxs |= __shfl_xor_sync(0xffffffffu, bxs, o);
      bys |= __shfl_xor_sync(0xffffffffu, bys, o);
      bzs |= __shfl_xor_sync(0xffffffffu, bzs, o);
    }
    const uint32_t nz = g.nz, nyz = g.ny * g.nz;
    const uint32_t centre = (ccx * g.ny + ccy) * g.nz + ccz;
    const uint32_t* cst = start + S.cell_off;
    float sum = fluid_i ? S.k.w0 : 0.0f;
    float sum_b = 0.0f;
    uint32_t cnt = 0, bad = 0;
    uint16_t* wp = nbr + s;  // next list entry: nbr[cnt * stride + s]
    const ListPlanes lp = list_planes(g, cst, ccx, ccy, ccz);
    // segment walk state (equal on the segment's lanes)
    uint32_t ucm = cm, blk = 0, jb = 0, je = 0, xs = 3, ys = 3, zs = 3, qh = 0, qt = 0;
    for (;;) {
      while (qt - qh < kSegLanes) {
        if (blk >= je) {
          if (!ucm) break;
          const uint32_t d = __ffs(ucm) - 1;
          ucm &= ucm - 1u;
          const uint32_t dzp = d / 9, dyp = (d / 3) % 3, dxp = d % 3;
          const uint32_t idx = centre + dxp * nyz + dyp * nz + dzp - (nyz + nz + 1u);
          jb = cst[idx];
          je = cst[idx + 1];
          blk = half ? (jb & ~31u) : jb;
          xs = (bxs >> (2 * dxp)) & 3u;
          ys = (bys >> (2 * dyp)) & 3u;
          zs = (bzs >> (2 * dzp)) & 3u;
          continue;
        }
        uint32_t m;
        if (half) {
          const uint4 hm = *reinterpret_cast<const uint4*>(halves + 4 * (blk >> 5));
          m = half_select(xs, hm.x) & half_select(ys, hm.y) & half_select(zs, hm.z);
          if (jb > blk) m &= ~0u << (jb - blk);
          if (je < blk + 32u) m &= (1u << (je - blk)) - 1u;
        } else {
          const uint32_t left = je - blk;
          m = left >= 32u ? ~0u : (1u << left) - 1u;
        }
        const uint32_t nib = (m >> (4 * sl)) & 15u;
        uint32_t at = qt + __popc(m & ((1u << (4 * sl)) - 1u));
        const uint32_t j4 = blk + 4 * sl;
        if (nib & 1u) queue[(at++) & (kSegQueue - 1)] = j4;
        if (nib & 2u) queue[(at++) & (kSegQueue - 1)] = j4 + 1;
        if (nib & 4u) queue[(at++) & (kSegQueue - 1)] = j4 + 2;
        if (nib & 8u) queue[at & (kSegQueue - 1)] = j4 + 3;
        qt += __popc(m);
        blk += 32u;
      }
      const uint32_t nc = min(qt - qh, kSegLanes);
      if (!__any_sync(0xffffffffu, nc != 0u)) break;
      __syncwarp();
      if (sl < nc) {
        const uint32_t j = queue[(qh + sl) & (kSegQueue - 1)];
        stj[sl] = j;
        stp[sl] = pos[j];
      }
      __syncwarp();
#pragma unroll
      for (uint32_t c = 0; c < kSegLanes; ++c) {
        if (c < nc) {
          const uint32_t j = stj[c];
          const float4 pj = stp[c];
          if (act && j != s) {
            const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            const float r2 = dx * dx + dy * dy + dz * dz;
            if (r2 <= h2) {
              const float tt = h2 - r2;
              const float wv = k6 * tt * tt * tt;
              bool keep = true;
              if (fluid_i) {
                if (pj.w > 0.0f) sum += wv;
                else sum_b += (-pj.w) * wv;
              } else if (pj.w > 0.0f) {
                sum += pj.w * wv;
              } else {
                keep = false;
              }
              if (keep) {
                if (cnt < cap) {
                  const uint32_t e = list_encode(lp, j);
                  bad |= e >> 31;
                  __stcs(wp, (unsigned short)e);  // streaming store: the list is read once, by the force pass
                  wp += stride;
                }
                ++cnt;
              }
            }
          }
        }
      }
      qh += nc;
      __syncwarp();
    }
    if (act) {
      nbr_n[s] = cnt | (bad ? kListBad : 0u);
      const float rho = fluid_i ? (S.k.mass * sum + sum_b) : ((-pi.w) * S.k.w0 + sum);
      const float p = tait(S.k, rho);
      rc[s] = make_float2(rho, p / (rho * rho));
      if (press_out) press_out[s] = p;
    }
  }
}

// ---------------------------------------------------------------- provider walls
// ProviderColliders::bounds prefilter of the fluid passes: skip the provider when p lies
// outside its bounds expanded by m (fluid_density.rs:90-101, fluid_boundary.rs:60-71).
__device__ __forceinline__ bool provider_outside(const ProviderDev& pr, float x, float y, float z, float m) {
  return pr.has_bounds && (x < pr.bminx - m || x > pr.bmaxx + m || y < pr.bminy - m || y > pr.bmaxy + m ||
                           z < pr.bminz - m || z > pr.bmaxz + m);
}

// contacts_point(p, probe) of one provider, calling emit(point xyz, outward normal xyz) for
// each contact in the provider's order. FACES: every face with (p[axis] - plane) * sign <=
// 2 probe, at p with that coordinate set to the plane (crates/vxl-phys-fluid/src/tests.rs:
// 81-110). CONVEX: the decisive plane (largest n.p - d) when -(n.p - d) >= -probe, at
// p - n (n.p - d) (crates/vxl-phys-terrain/src/plane_set.rs:60-76, 166-181).
// TABLE: the particle's planes of the table side in use, in their table order.
template <class F>
__device__ __forceinline__ void provider_contacts(const ProviderDev& pr, const WallPlaneDev* __restrict__ pl,
                                                  const ContactTableDev& ct, uint32_t gref, float px, float py,
                                                  float pz, float probe, F&& emit) {
  if (pr.kind == kProviderTable) {
    const uint32_t e = ct.ent ? ct.ent[gref] : 0u;
    if (!e) return;
    for (uint32_t k = ct.start[e - 1], k1 = ct.start[e]; k < k1; ++k) {
      const float4 a = ct.planes[2 * k], n = ct.planes[2 * k + 1];
      emit(a.x, a.y, a.z, n.x, n.y, n.z);
    }
    return;
  }
  if (pr.kind == kProviderFaces) {
    for (uint32_t k = pr.first; k < pr.first + pr.count; ++k) {
      const WallPlaneDev f = pl[k];
      const float comp = f.axis == 0u ? px : (f.axis == 1u ? py : pz);
      const float sdf = (comp - f.d) * f.sign;
      if (sdf > 2.0f * probe) continue;
      float cx = px, cy = py, cz = pz, nx = 0.0f, ny = 0.0f, nz = 0.0f;
      if (f.axis == 0u) {
        cx = f.d;
        nx = f.sign;
      } else if (f.axis == 1u) {
        cy = f.d;
        ny = f.sign;
      } else {
        cz = f.d;
        nz = f.sign;
      }
      emit(cx, cy, cz, nx, ny, nz);
    }
    return;
  }
  if (pr.count == 0u) return;
  float best = -INFINITY;
  uint32_t kb = pr.first;
  for (uint32_t k = pr.first; k < pr.first + pr.count; ++k) {
    const WallPlaneDev q = pl[k];
    const float sd = (q.nx * px + q.ny * py + q.nz * pz) - q.d;
    if (sd > best) {
      best = sd;
      kb = k;
    }
  }
  if (-best < -probe) return;
  const WallPlaneDev q = pl[kb];
  const float t = (q.nx * px + q.ny * py + q.nz * pz) - q.d;
  emit(px - q.nx * t, py - q.ny * t, pz - q.nz * t, q.nx, q.ny, q.nz);
}

// Density (poly6 with self term) + Tait EOS, persistent over tiles, one thread per slot.
// Fluid: rho = mass * (w0 + sum_fluid W) + sum_boundary pmass_j W
// (crates/vxl-phys-fluid/src/fluid_density.rs:24-51); boundary: rho = pmass_i w0 +
// sum_fluid pmass_j W (fluid_density.rs:59-69). Writes (rho, p / rho^2) for the force
// pass (the reference recomputes press/(rho*rho) per pair: same value). Also records, in
// walk order, the slots of the neighbours that contributed (all for fluid, fluid ones for
// boundary particles): nbr[k * stride + s], k < cap, with the full count in nbr_n[s]
// (a count above cap sends the consumers back to walking the cells).
// kWalls: scenes with provider walls add, for a fluid particle, after each neighbour's term
// its mirror ghosts in the particle's provider planes (0 < sdf < h, at most 8; ghost
// g = pj - 2 ((pj - point).n) n with pj = pi - d, W(|pi - g|) if within h), in the
// reference's order (wall_planes_in and the ghost loop, fluid_density.rs:25-47, 76-118).
template <int kBlock, bool kWalls = false>
__global__ void __launch_bounds__(kBlock, VXL_DENSITY_THREADS_PER_SM / kBlock) k_e_density(
    const float4* __restrict__ pos, const uint32_t* __restrict__ start, const SceneDev* __restrict__ sc,
    const TileDev* __restrict__ tiles, uint32_t ntiles, EngineCtl* ctl, const uint32_t* __restrict__ halves,
    float2* __restrict__ rc, float* __restrict__ press_out, uint16_t* __restrict__ nbr,
    uint32_t* __restrict__ nbr_n, uint32_t cap, uint32_t stride, const uint32_t* __restrict__ wet,
    const uint32_t* __restrict__ xorder, const ProviderDev* __restrict__ prov = nullptr,
    const WallPlaneDev* __restrict__ wplanes = nullptr, const uint32_t* __restrict__ orig = nullptr,
    ContactTableDev ctm = ContactTableDev{nullptr, nullptr, nullptr}) {
  if (ctl->err & kErrCellCap) return;
  for (uint32_t t = first_tile(&ctl->work[kWorkDensity], ntiles); t < ntiles; t = following_tile(&ctl->work[kWorkDensity], ntiles)) {
    const TileDev td = tiles[t];
    const SceneDev& S = sc[td.scene];
    const GridBox g = S.g;
    const SphConst& k = S.k;
    const uint32_t* cst = start + S.cell_off;
    const float h = k.h, h2 = k.h2, k6 = k.k6, w0 = k.w0, mass = k.mass;
    const bool half_walk = halves != nullptr && g.bin >= 2.0f * h;  // uniform over the tile
    const uint32_t epoch = ctl->epoch;
    for (uint32_t i = threadIdx.x; i < td.count; i += kBlock) {
      const uint32_t s = half_walk ? xorder[td.first + i] : td.first + i;
      const float4 pi = pos[s];
      const bool fluid_i = pi.w > 0.0f;
      uint32_t cx, cy, cz;
      bin_of(g, pi.x, pi.y, pi.z, cx, cy, cz);
      float sum = fluid_i ? w0 : 0.0f;
      float sum_b = 0.0f;
      uint32_t cnt = 0, bad = 0;
      uint16_t* wp = nbr + s;  // next list entry: nbr[cnt * stride + s]
      const ListPlanes lp = list_planes(g, cst, cx, cy, cz);
      float wpt[kWalls ? 3 * kMaxWallPlanes : 1], wn[kWalls ? 3 * kMaxWallPlanes : 1];
      uint32_t np = 0;
      if (kWalls && fluid_i) {
        for (uint32_t q = S.prov_first; q < S.prov_first + S.prov_count; ++q) {
          const ProviderDev pr = prov[q];
          if (provider_outside(pr, pi.x, pi.y, pi.z, h)) continue;
          provider_contacts(pr, wplanes, ctm, orig ? orig[s] : 0u, pi.x, pi.y, pi.z, h,
                            [&](float cx_, float cy_, float cz_, float nx_, float ny_, float nz_) {
                              const float sdf = (pi.x - cx_) * nx_ + (pi.y - cy_) * ny_ + (pi.z - cz_) * nz_;
                              if (sdf > 0.0f && sdf < h && np < kMaxWallPlanes) {
                                wpt[3 * np] = cx_;
                                wpt[3 * np + 1] = cy_;
                                wpt[3 * np + 2] = cz_;
                                wn[3 * np] = nx_;
                                wn[3 * np + 1] = ny_;
                                wn[3 * np + 2] = nz_;
                                ++np;
                              }
                            });
        }
      }
      auto visit = [&](uint32_t j) {  // j != s (the callers skip it)
        const float4 pj = pos[j];
        const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
        const float r2 = dx * dx + dy * dy + dz * dz;
        if (r2 <= h2) {
          const float tt = h2 - r2;
          const float w = k6 * tt * tt * tt;
          bool rec = true;
          if (fluid_i) {
            if (pj.w > 0.0f) sum += w;
            else sum_b += (-pj.w) * w;
            if (kWalls) {
              for (uint32_t q = 0; q < np; ++q) {
                const float qx = pi.x - dx, qy = pi.y - dy, qz = pi.z - dz;  // pj = pi - d
                const float dn = (qx - wpt[3 * q]) * wn[3 * q] + (qy - wpt[3 * q + 1]) * wn[3 * q + 1] +
                                 (qz - wpt[3 * q + 2]) * wn[3 * q + 2];
                const float t2 = 2.0f * dn;
                const float ex = pi.x - (qx - wn[3 * q] * t2), ey = pi.y - (qy - wn[3 * q + 1] * t2),
                            ez = pi.z - (qz - wn[3 * q + 2] * t2);
                const float rg2 = ex * ex + ey * ey + ez * ez;
                if (rg2 <= h2) {
                  const float tg = h2 - rg2;
                  sum += k6 * tg * tg * tg;
                }
              }
            }
          } else if (pj.w > 0.0f) {
            sum += pj.w * w;
          } else {
            rec = false;
          }
          if (rec) {
            if (cnt < cap) {
              const uint32_t e = list_encode(lp, j);
              bad |= e >> 31;
              __stcs(wp, (unsigned short)e);  // streaming store: the list is read once, by the force pass
              wp += stride;
            }
            ++cnt;
          }
        }
      };
      // A boundary particle sums fluid neighbours only: with no fluid particle in its 27
      // cells (none marked wet this substep) its walk would accept nothing.
      bool dry = false;
      if (!fluid_i) {
        const uint32_t* wc = wet + S.cell_off;
        dry = true;
        for (int dz = -1; dz <= 1; ++dz) {
          const int z = (int)cz + dz;
          if (z < 0 || z >= (int)g.nz) continue;
          for (int dy = -1; dy <= 1; ++dy) {
            const int y = (int)cy + dy;
            if (y < 0 || y >= (int)g.ny) continue;
            for (int dx = -1; dx <= 1; ++dx) {
              const int x = (int)cx + dx;
              if (x < 0 || x >= (int)g.nx) continue;
              if (wc[((uint32_t)x * g.ny + (uint32_t)y) * g.nz + (uint32_t)z] == epoch) dry = false;
            }
          }
        }
      }
      // Without provider walls: the same test and sums as `visit`, with the list entry
      // formed from the walked cell's plane offset (kadd, set by cellhook before each cell).
      uint32_t kadd = 0;
      auto visit1 = [&](uint32_t j) {  // j != s (the walks skip it)
        const float4 pj = pos[j];
        const float ddx = pi.x - pj.x, ddy = pi.y - pj.y, ddz = pi.z - pj.z;
        const float r2 = ddx * ddx + ddy * ddy + ddz * ddz;
        if (r2 <= h2) {
          const float tt = h2 - r2;
          const float w = k6 * tt * tt * tt;
          // the neighbour's class selected, not branched on (the same sums: an unselected
          // term is not added)
          const bool fj = pj.w > 0.0f;
          const float tf = fluid_i ? w : pj.w * w;
          const float tb = (-pj.w) * w;
          sum = fj ? sum + tf : sum;
          sum_b = (fluid_i && !fj) ? sum_b + tb : sum_b;
          if (fj || fluid_i) {
            if (cnt < cap) {
              __stcs(wp, (unsigned short)(j + kadd));  // streaming store: read once, by the force pass
              wp += stride;
            }
            ++cnt;
          }
        }
      };
      // list entries of the cell about to be walked: (plane << 14) + slot - plane's first slot,
      // the plane's first slot being that of cell (cx + pl - 1, max(cy - 1, 0), max(cz - 1, 0));
      // a cell reaching 2^14 slots past it marks the list unusable (consumers walk again)
      auto cellhook = [&](uint32_t pl, uint32_t jend) {
        const uint32_t pb = cst[(cx + pl - 1u) * (g.ny * g.nz) + (cy > 0 ? cy - 1 : 0) * g.nz + (cz > 0 ? cz - 1 : 0)];
        kadd = (pl << kListOffBits) - pb;
        bad |= (jend > pb && jend - 1u - pb > kListOffMask) ? 1u : 0u;
      };
      if (dry) {
      } else if (half_walk) {
        if constexpr (kWalls) {
          walk27_half(g, cst, halves, pi.x, pi.y, pi.z, cx, cy, cz, h, [&](uint32_t j) {
            if (j != s) visit(j);
          });
        } else {
          walk27_half_c(g, cst, halves, pi.x, pi.y, pi.z, cx, cy, cz, h, s, cellhook, visit1);
        }
      } else {
        if constexpr (kWalls) {
          walk27<true>(g, cst, pi.x, pi.y, pi.z, cx, cy, cz, h, visit, s);
        } else {
          walk27_c(g, cst, pi.x, pi.y, pi.z, cx, cy, cz, h, s, cellhook, visit1);
        }
      }
      nbr_n[s] = cnt | (bad ? kListBad : 0u);
      const float rho = fluid_i ? (mass * sum + sum_b) : ((-pi.w) * w0 + sum);
      const float p = tait(k, rho);
      rc[s] = make_float2(rho, p / (rho * rho));
      if (press_out) press_out[s] = p;
    }
  }
}

// Force (gravity + spiky pressure + Monaghan viscosity + XSPH, fluid_force.rs:165-214)
// fused with integration (semi-implicit Euler + CFL clamp, fluid_step.rs:112-123) for
// fluid slots; boundary slots are copied unchanged (kinematic within the tick).
// Neighbours come from the density pass's list (same walk order, so the same sums); a
// particle whose list overflowed walks the 27 cells again. Reads the sorted buffer and
// writes the integrated state to (pos_out, vel_out) in the same slot order; accumulates
// each tile's fluid AABB into its scene's accumulator for the next grid box.
template <int kBlock>
__global__ void __launch_bounds__(kBlock, VXL_FORCE_THREADS_PER_SM / kBlock) k_e_force(
    const float4* __restrict__ pos, const float4* __restrict__ vel, const float2* __restrict__ rc,
    const uint32_t* __restrict__ start, const uint16_t* __restrict__ nbr, const uint32_t* __restrict__ nbr_n,
    uint32_t cap, uint32_t stride, SceneDev* __restrict__ sc, const TileDev* __restrict__ tiles, uint32_t ntiles,
    EngineCtl* ctl, float4* __restrict__ pos_out, float4* __restrict__ vel_out, float4* __restrict__ acc_out,
    float4* __restrict__ xsph_out) {
  if (ctl->err & kErrCellCap) return;
  for (uint32_t t = first_tile(&ctl->work[kWorkForce], ntiles); t < ntiles; t = following_tile(&ctl->work[kWorkForce], ntiles)) {
    const TileDev td = tiles[t];
    SceneDev& S = sc[td.scene];
    const SphConst& k = S.k;
    const float dt = S.dt, vmax = S.vmax, vmax2 = S.vmax2;
    for (uint32_t b0 = 0; b0 < td.count; b0 += kBlock) {
      const uint32_t i = b0 + threadIdx.x;
      const bool valid = i < td.count;
      float nx = 0, ny = 0, nz = 0;
      bool fluid_i = false;
      if (valid) {
        const uint32_t s = td.first + i;
        const float4 pi = pos[s];
        const float4 vi = vel[s];
        fluid_i = pi.w > 0.0f;
        if (!fluid_i) {
          pos_out[s] = pi;
          vel_out[s] = vi;
        } else {
          const float2 rci = rc[s];
          const float rho_i = rci.x, ci2 = rci.y;
          const float h = k.h, h2 = k.h2, ks = k.ks, k6 = k.k6, alpha_c = k.alpha_c, h001 = k.h001;
          float ax = k.gx, ay = k.gy, az = k.gz;
          float xx = 0.0f, xy = 0.0f, xz = 0.0f;
          auto pair = [&](uint32_t j, const float4& pj, float dx, float dy, float dz, float r2) {
            const float2 rcj = rc[j];
            const float4 vj = vel[j];
            const float rho_j = rcj.x, cj2 = rcj.y;
            const float mj = fabsf(pj.w);
            const float r = sqrtf(r2);
            const float tt = h - r;
            const float coef = mj * (ks * tt * tt) * (ci2 + cj2);
            const float denom = fmaxf(r, 1e-9f);
            const float q = coef / denom;
            ax = ax + dx * q;
            ay = ay + dy * q;
            az = az + dz * q;
            const float vx = vi.x - vj.x, vy = vi.y - vj.y, vz = vi.z - vj.z;
            const float vdn = -(vx * dx + vy * dy + vz * dz);
            {
              // artificial viscosity only when approaching (vdn > 0): computed for every pair and
              // selected, so the warp does not diverge around it (the sums are the same)
              const float mu = vdn * h / (r2 + h001);
              const float c = mj * (alpha_c * mu / (0.5f * (rho_i + rho_j))) * (ks * tt * tt);
              const float q2 = c / denom;
              const bool take = vdn > 0.0f;
              ax = take ? ax + dx * q2 : ax;
              ay = take ? ay + dy * q2 : ay;
              az = take ? az + dz * q2 : az;
            }
            const float t2 = h2 - r2;
            const float w = k6 * t2 * t2 * t2;
            const float f = mj * 2.0f / (rho_i + rho_j) * w;
            xx = xx + (vj.x - vi.x) * f;
            xy = xy + (vj.y - vi.y) * f;
            xz = xz + (vj.z - vi.z) * f;
          };
          const uint32_t cnt = nbr_n[s];
          const GridBox g = S.g;
          uint32_t cx, cy, cz;
          bin_of(g, pi.x, pi.y, pi.z, cx, cy, cz);
          if (cnt <= cap) {
            // the next list entry is loaded one neighbour ahead, so each iteration waits on
            // one dependent gather (pos/vel/rc of j) instead of two (measured: 6-8% faster),
            // and the one kListPrefetch ahead is fetched into L2 (the list is not L2-resident)
            const ListPlanes lp = list_planes(g, start + S.cell_off, cx, cy, cz);
            const uint16_t* np = nbr + s;
            uint32_t en = cnt ? *np : 0u;
            for (uint32_t q = 0; q < cnt; ++q) {
              const uint32_t j = list_decode(lp, en);
              np += stride;
              if (q + kListPrefetch < cnt)  // the entry kListPrefetch ahead into L2
                asm volatile("prefetch.global.L2 [%0];" ::"l"(np + (size_t)(kListPrefetch - 1) * stride));
              if (q + 1 < cnt) en = *np;
              const float4 pj = pos[j];
              const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
              pair(j, pj, dx, dy, dz, dx * dx + dy * dy + dz * dz);
            }
          } else {
            walk27<false, true>(g, start + S.cell_off, pi.x, pi.y, pi.z, cx, cy, cz, h, [&](uint32_t j) {
              if (j == s) return;
              const float4 pj = pos[j];
              const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
              const float r2 = dx * dx + dy * dy + dz * dz;
              if (r2 <= h2) pair(j, pj, dx, dy, dz, r2);
            });
          }
          if (acc_out) {
            acc_out[s] = make_float4(ax, ay, az, 0.0f);
            xsph_out[s] = make_float4(xx, xy, xz, 0.0f);
          }
          const float eps = k.eps;
          float ux = vi.x + ax * dt + xx * eps;
          float uy = vi.y + ay * dt + xy * eps;
          float uz = vi.z + az * dt + xz * eps;
          const float s2 = ux * ux + uy * uy + uz * uz;
          if (s2 > vmax2) {
            const float scl = vmax / sqrtf(s2);
            ux = ux * scl;
            uy = uy * scl;
            uz = uz * scl;
          }
          nx = pi.x + ux * dt;
          ny = pi.y + uy * dt;
          nz = pi.z + uz * dt;
          pos_out[s] = make_float4(nx, ny, nz, pi.w);
          vel_out[s] = make_float4(ux, uy, uz, 0.0f);
        }
      }
      // scenes with provider walls take their fluid AABB after the projection pass
      if (S.prov_count == 0u) block_bbox_accumulate(S.fbox, nx, ny, nz, valid && fluid_i);
    }
  }
}

// ---------------------------------------------------------------- provider walls after integration
// boundary_pass (crates/vxl-phys-fluid/src/fluid_boundary.rs:45-101) on the integrated state of
// the scenes with providers, one thread per fluid slot: for each contact of each provider at the
// integrated position pi (probe = skin = 0.15 h) with penetration pen = -(pi - point).n > 0, the
// particle moves by n min(pen + skin, h) and loses its inward normal velocity; the normal sum of a
// pushed particle is kept for the separation, by reference index (pflag, pnsum; w = scene).
// The scene's fluid AABB for the next grid is accumulated here, from the projected positions.
__global__ void k_e_wall_project(float4* __restrict__ pos, float4* __restrict__ vel, SceneDev* __restrict__ sc,
                                 const TileDev* __restrict__ tiles, uint32_t ntiles, const EngineCtl* __restrict__ ctl,
                                 const ProviderDev* __restrict__ prov, const WallPlaneDev* __restrict__ wplanes,
                                 const uint32_t* __restrict__ orig, uint32_t* __restrict__ pflag,
                                 float4* __restrict__ pnsum, ContactTableDev ctp) {
  if (ctl->err & kErrCellCap) return;
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const TileDev td = tiles[t];
    SceneDev& S = sc[td.scene];
    if (S.prov_count == 0u) continue;  // uniform over the block
    const float h = S.k.h, skin = 0.15f * h;  // fluid_access.rs:47
    for (uint32_t b0 = 0; b0 < td.count; b0 += blockDim.x) {
      const uint32_t i = b0 + threadIdx.x;
      const bool valid = i < td.count;
      float x = 0.0f, y = 0.0f, z = 0.0f;
      bool fluid = false;
      if (valid) {
        const uint32_t sl = td.first + i;
        const float4 p = pos[sl];
        fluid = p.w > 0.0f;
        x = p.x;
        y = p.y;
        z = p.z;
        if (fluid) {
          const float4 v = vel[sl];
          float vx = v.x, vy = v.y, vz = v.z, nsx = 0.0f, nsy = 0.0f, nsz = 0.0f;
          bool hit = false;
          for (uint32_t q = S.prov_first; q < S.prov_first + S.prov_count; ++q) {
            const ProviderDev pr = prov[q];
            if (provider_outside(pr, p.x, p.y, p.z, h)) continue;
            provider_contacts(pr, wplanes, ctp, orig[sl], p.x, p.y, p.z, skin,
                              [&](float cx, float cy, float cz, float nx, float ny, float nz) {
                                const float sdf = (p.x - cx) * nx + (p.y - cy) * ny + (p.z - cz) * nz;
                                const float pen = -sdf;
                                if (pen <= 0.0f) return;
                                const float m = fminf(pen + skin, h);
                                x = x + nx * m;
                                y = y + ny * m;
                                z = z + nz * m;
                                nsx = nsx + nx;
                                nsy = nsy + ny;
                                nsz = nsz + nz;
                                hit = true;
                                const float vn = vx * nx + vy * ny + vz * nz;
                                if (vn < 0.0f) {
                                  vx = vx - nx * vn;
                                  vy = vy - ny * vn;
                                  vz = vz - nz * vn;
                                }
                              });
          }
          pos[sl] = make_float4(x, y, z, p.w);
          vel[sl] = make_float4(vx, vy, vz, v.w);
          const uint32_t o = orig[sl];
          pflag[o] = hit ? 1u : 0u;
          if (hit) pnsum[o] = make_float4(nsx, nsy, nsz, __uint_as_float(td.scene));
        }
      }
      block_bbox_accumulate(S.fbox, x, y, z, valid && fluid);
    }
  }
}

// The pushed particles in ascending reference index (plist), in two passes over chunks of
// kPushedChunk indices: per-chunk counts, then each chunk's entries at its offset. The last
// chunk stores the total in ctl->work[kWorkPushed].
__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t* sh) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  uint32_t tot = 0;
  for (int w = 0; w < nw; ++w) tot += sh[w];
  return tot;
}

__global__ void k_e_pushed_count(const uint32_t* __restrict__ pflag, uint32_t n, const EngineCtl* __restrict__ ctl,
                                 uint32_t* __restrict__ blk) {
  if (ctl->err & kErrCellCap) return;
  __shared__ uint32_t sh[32];
  const uint32_t base = blockIdx.x * kPushedChunk;
  uint32_t c = 0;
  for (uint32_t k = threadIdx.x; k < kPushedChunk; k += blockDim.x) {
    const uint32_t o = base + k;
    if (o < n && pflag[o]) ++c;
  }
  c = block_sum(c, sh);
  if (threadIdx.x == 0) blk[blockIdx.x] = c;
}

__global__ void k_e_pushed_emit(const uint32_t* __restrict__ pflag, uint32_t n, const uint32_t* __restrict__ blk,
                                EngineCtl* __restrict__ ctl, uint32_t* __restrict__ plist) {
  if (ctl->err & kErrCellCap) return;
  __shared__ uint32_t sh[32], wtot[32];
  uint32_t part = 0;
  for (uint32_t k = threadIdx.x; k < blockIdx.x; k += blockDim.x) part += blk[k];
  uint32_t off = block_sum(part, sh);
  const uint32_t base = blockIdx.x * kPushedChunk;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  for (uint32_t r0 = 0; r0 < kPushedChunk; r0 += blockDim.x) {
    const uint32_t o = base + r0 + threadIdx.x;
    const bool f = o < n && pflag[o] != 0u;
    const uint32_t bal = __ballot_sync(0xffffffffu, f);
    __syncthreads();
    if (lane == 0) wtot[wid] = __popc(bal);
    __syncthreads();
    uint32_t before = 0, total = 0;
    for (int w = 0; w < nw; ++w) {
      if (w < wid) before += wtot[w];
      total += wtot[w];
    }
    if (f) plist[off + before + __popc(bal & ((1u << lane) - 1u))] = o;
    off += total;
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) ctl->work[kWorkPushed] = off;
}

// First position in the ascending list a[0, n) whose value is >= key.
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t* __restrict__ a, uint32_t n, uint32_t key) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// separate_coincident (fluid_boundary.rs:103-128) moves a pushed particle only if some
// earlier pushed particle of its scene lies closer than r_min = 0.2 h. If no pair is that
// close at the projected positions, nothing moves (by induction over the sequential loop):
// this pass, one thread per pushed particle, decides whether the sequential pass must run.
// A scene's reference indices are [base, base + count), so its pushed particles are one run
// of the ascending list, found by binary search.
__global__ void k_e_separate_check(const float4* __restrict__ pos, const SceneDev* __restrict__ sc,
                                   const uint32_t* __restrict__ plist, const float4* __restrict__ pnsum,
                                   const uint32_t* __restrict__ slot_of, EngineCtl* __restrict__ ctl) {
  if (ctl->err & kErrCellCap) return;
  const uint32_t P = ctl->work[kWorkPushed];
  for (uint32_t a = blockIdx.x * blockDim.x + threadIdx.x; a < P; a += gridDim.x * blockDim.x) {
    const uint32_t oa = plist[a];
    const float4 na = pnsum[oa];
    const float nl = sqrtf(na.x * na.x + na.y * na.y + na.z * na.z);
    if (nl <= 1e-9f) continue;  // never moves
    const uint32_t q = __float_as_uint(na.w);
    const float r_min = 0.2f * sc[q].k.h;
    const float rm2 = r_min * r_min;
    if (*(volatile const uint32_t*)&ctl->work[kWorkTrigger]) return;
    const float4 pa = pos[slot_of[oa]];
    for (uint32_t b = lower_bound_u32(plist, a, sc[q].base); b < a; ++b) {
      const float4 pb = pos[slot_of[plist[b]]];
      const float dx = pa.x - pb.x, dy = pa.y - pb.y, dz = pa.z - pb.z;
      if (dx * dx + dy * dy + dz * dz < rm2) {
        atomicOr(&ctl->work[kWorkTrigger], 1u);
        break;
      }
    }
  }
}

// The sequential separation itself, one block, only when the check found a close pair: for
// each pushed particle a in order (normal sum n_a, |n_a| > 1e-9), for each earlier pushed b of
// its scene in order, with the current (already separated) positions: if |pa - pb|^2 < r_min^2,
// pa += n_a / |n_a| (r_min - |pa - pb|). The block tests a window of b in parallel against the
// current pa and applies the first hit, then resumes after it. If anything moved, the AABB
// accumulators of the scenes with providers are reset for k_e_wall_rebox.
__global__ void __launch_bounds__(1024) k_e_separate(float4* __restrict__ pos, SceneDev* __restrict__ sc,
                                                     uint32_t nscenes, const uint32_t* __restrict__ plist,
                                                     const float4* __restrict__ pnsum,
                                                     const uint32_t* __restrict__ slot_of, EngineCtl* __restrict__ ctl) {
  if ((ctl->err & kErrCellCap) || !ctl->work[kWorkTrigger]) return;
  const uint32_t P = ctl->work[kWorkPushed];
  __shared__ float4 pa_s;
  __shared__ uint32_t first;
  bool moved = false;  // thread 0
  for (uint32_t a = 0; a < P; ++a) {
    const uint32_t oa = plist[a];
    const float4 na = pnsum[oa];
    const float nl = sqrtf(na.x * na.x + na.y * na.y + na.z * na.z);
    if (nl <= 1e-9f) continue;  // uniform over the block
    const uint32_t q = __float_as_uint(na.w);
    const float r_min = 0.2f * sc[q].k.h;
    const float rm2 = r_min * r_min;
    const float inv = 1.0f / nl;
    const float dirx = na.x * inv, diry = na.y * inv, dirz = na.z * inv;
    const uint32_t sa = slot_of[oa];
    if (threadIdx.x == 0) pa_s = pos[sa];
    __syncthreads();
    uint32_t b0 = lower_bound_u32(plist, a, sc[q].base);  // the scene's first pushed particle
    while (b0 < a) {
      if (threadIdx.x == 0) first = 0xffffffffu;
      __syncthreads();
      const float4 cur = pa_s;
      const uint32_t b = b0 + threadIdx.x;
      if (b < a) {
        const float4 pb = pos[slot_of[plist[b]]];
        const float dx = cur.x - pb.x, dy = cur.y - pb.y, dz = cur.z - pb.z;
        if (dx * dx + dy * dy + dz * dz < rm2) atomicMin(&first, b);
      }
      __syncthreads();
      const uint32_t f = first;
      if (f == 0xffffffffu) {
        b0 += blockDim.x;
      } else {
        if (threadIdx.x == 0) {
          const float4 pb = pos[slot_of[plist[f]]];
          const float dx = cur.x - pb.x, dy = cur.y - pb.y, dz = cur.z - pb.z;
          const float r = sqrtf(dx * dx + dy * dy + dz * dz);
          const float m = r_min - r;
          pa_s = make_float4(cur.x + dirx * m, cur.y + diry * m, cur.z + dirz * m, cur.w);
          moved = true;
        }
        b0 = f + 1;
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) pos[sa] = pa_s;
    __syncthreads();
  }
  if (threadIdx.x == 0 && moved) {
    ctl->work[kWorkMoved] = 1u;
    for (uint32_t q = 0; q < nscenes; ++q)
      if (sc[q].prov_count) {
        for (int c = 0; c < 3; ++c) {
          sc[q].fbox[c] = 0xffffffffu;
          sc[q].fbox[3 + c] = 0u;
        }
      }
  }
}

// After a separation that moved particles: the fluid AABB of the scenes with providers again,
// from the final positions.
__global__ void k_e_wall_rebox(const float4* __restrict__ pos, SceneDev* __restrict__ sc,
                               const TileDev* __restrict__ tiles, uint32_t ntiles, const EngineCtl* __restrict__ ctl) {
  if ((ctl->err & kErrCellCap) || !ctl->work[kWorkMoved]) return;
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const TileDev td = tiles[t];
    SceneDev& S = sc[td.scene];
    if (S.prov_count == 0u) continue;
    for (uint32_t b0 = 0; b0 < td.count; b0 += blockDim.x) {
      const uint32_t i = b0 + threadIdx.x;
      const bool valid = i < td.count;
      float4 p = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      if (valid) p = pos[td.first + i];
      block_bbox_accumulate(S.fbox, p.x, p.y, p.z, valid && p.w > 0.0f);
    }
  }
}

// Pair term of the boundary reaction for fluid i on boundary j, from i's side of the
// reference loop (crates/vxl-phys-fluid/src/fluid_force.rs:182-207): returns
// q = m_i (coef + cv) / denom, with d = p_i - p_j; the caller applies bforce -= d * q.
__device__ __forceinline__ float bforce_pair(const SphConst& k, float r2, float dx, float dy, float dz,
                                             float rho_i, float ci2, float mi, float4 vi, float rho_j, float cj2,
                                             float mj, float4 vj) {
  const float r = sqrtf(r2);
  const float t = k.h - r;
  const float coef = mj * (k.ks * t * t) * (ci2 + cj2);
  const float denom = fmaxf(r, 1e-9f);
  float cv = 0.0f;
  const float vx = vi.x - vj.x, vy = vi.y - vj.y, vz = vi.z - vj.z;
  const float vdn = -(vx * dx + vy * dy + vz * dz);
  if (vdn > 0.0f) {
    const float mu = vdn * k.h / (r2 + k.h001);
    cv = mj * (k.alpha_c * mu / (0.5f * (rho_i + rho_j))) * (k.ks * t * t);
  }
  return mi * (coef + cv) / denom;
}

// Reaction on each boundary particle j: the reference accumulates bforce[j] -= F_ij over
// fluid i in ascending reference index (the outer loop of force_pass_serial). Here the
// boundary particle takes its fluid neighbours (recorded by the density pass, or found by
// walking the 27 cells when that list overflowed), orders them by reference index and sums
// in that order, so the result is the same sum. Runs over boundary tiles in reference
// order (every lane a boundary particle; slot_of finds its sorted slot); output by global
// reference index.
__global__ void __launch_bounds__(128) k_e_bforce(
    const float4* __restrict__ pos, const float4* __restrict__ vel, const float2* __restrict__ rc,
    const uint32_t* __restrict__ start, const uint32_t* __restrict__ orig, const uint16_t* __restrict__ nbr,
    const uint32_t* __restrict__ nbr_n, uint32_t cap, uint32_t stride, const SceneDev* __restrict__ sc,
    const uint32_t* __restrict__ slot_of, const TileDev* __restrict__ btiles, uint32_t ntiles, EngineCtl* ctl,
    float4* __restrict__ bforce) {
  if (ctl->err & kErrCellCap) return;
  for (uint32_t t = first_tile(&ctl->work[kWorkBforce], ntiles); t < ntiles; t = following_tile(&ctl->work[kWorkBforce], ntiles)) {
    const TileDev td = btiles[t];
    const SceneDev& S = sc[td.scene];
    const SphConst& k = S.k;
    const GridBox g = S.g;
    const uint32_t* cst = start + S.cell_off;
    const float h2 = k.h2;
    for (uint32_t i = threadIdx.x; i < td.count; i += blockDim.x) {
      const uint32_t o = td.first + i;  // global reference index of a boundary particle
      const uint32_t s = slot_of[o];
      const float4 pj = pos[s];
      const float4 vj = vel[s];
      const float2 rcj = rc[s];
      const float mj = -pj.w;
      uint32_t cx, cy, cz;
      bin_of(g, pj.x, pj.y, pj.z, cx, cy, cz);
      // insertion-sort buffer: only entries [0, n) are ever read (not zero-filled: that
      // cost 64 local stores per particle)
      uint32_t key[kBGatherCap];
      uint32_t slot[kBGatherCap];
      int n = 0;
      bool overflow = false;
      auto insert = [&](uint32_t ii) {
        if (n < kBGatherCap) {
          const uint32_t o = orig[ii];
          int q = n++;
          for (; q > 0; --q) {
            const uint32_t kq = key[q - 1];
            if (kq <= o) break;
            key[q] = kq;
            slot[q] = slot[q - 1];
          }
          key[q] = o;
          slot[q] = ii;
        } else {
          overflow = true;
        }
      };
      const uint32_t cnt = nbr_n[s];
      if (cnt <= cap) {
        const ListPlanes lp = list_planes(g, cst, cx, cy, cz);
        for (uint32_t q = 0; q < cnt; ++q) insert(list_decode(lp, nbr[(size_t)q * stride + s]));
      } else {
        walk27<false, true>(g, cst, pj.x, pj.y, pj.z, cx, cy, cz, k.h, [&](uint32_t ii) {
          const float4 p = pos[ii];
          if (!(p.w > 0.0f)) return;
          const float dx = p.x - pj.x, dy = p.y - pj.y, dz = p.z - pj.z;
          if (!(dx * dx + dy * dy + dz * dz <= h2)) return;
          insert(ii);
        });
      }
      float bx = 0.0f, by = 0.0f, bz = 0.0f;
      auto apply = [&](uint32_t ii) {
        const float4 p = pos[ii];
        const float dx = p.x - pj.x, dy = p.y - pj.y, dz = p.z - pj.z;
        const float r2 = dx * dx + dy * dy + dz * dz;
        const float2 rci = rc[ii];
        const float q = bforce_pair(k, r2, dx, dy, dz, rci.x, rci.y, p.w, vel[ii], rcj.x, rcj.y, mj, vj);
        bx = bx - dx * q;
        by = by - dy * q;
        bz = bz - dz * q;
      };
      if (!overflow) {
        for (int q = 0; q < n; ++q) apply(slot[q]);
      } else {
        // Slow path: fluid neighbours in ascending reference index by repeated minimum
        // search (O(neighbours x candidates)); counted in ctl->slow_gathers.
        atomicAdd(&ctl->slow_gathers, 1u);
        uint32_t last = 0;
        bool first = true;
        for (;;) {
          uint32_t best = 0xffffffffu, best_slot = 0;
          walk27<false, true>(g, cst, pj.x, pj.y, pj.z, cx, cy, cz, k.h, [&](uint32_t ii) {
            const float4 p = pos[ii];
            if (!(p.w > 0.0f)) return;
            const uint32_t o = orig[ii];
            if (!first && o <= last) return;
            if (o >= best) return;
            const float dx = p.x - pj.x, dy = p.y - pj.y, dz = p.z - pj.z;
            if (!(dx * dx + dy * dy + dz * dz <= h2)) return;
            best = o;
            best_slot = ii;
          });
          if (best == 0xffffffffu) break;
          apply(best_slot);
          last = best;
          first = false;
        }
      }
      bforce[o] = make_float4(bx, by, bz, 0.0f);
    }
  }
}

// Per-span force and torque about the body origin (fluid_boundary.rs:10-28), added to
// the tick accumulator. A span of at most kReactExactSpan particles is summed in index order
// (the reference's sum, bit for bit) by one warp: the lanes load 32 consecutive particles
// and form each one's force and torque terms, then lane a (a < 6) adds component a of the
// 32 terms to its running sum in index order — six independent sequential sums, with the
// loads of a batch in flight together instead of one at a time. Larger spans (tank walls)
// take one block each (k_react_long), the same sums in the same order with the next
// batch's loads overlapping them. Span ranges are global reference indices.

// Torque origin of a span: its coupled rigid body's position, or the origin it was given.
__device__ __forceinline__ void span_origin(const SpanDev& sp, const RigidBodyDev* __restrict__ rb, float& ox,
                                            float& oy, float& oz) {
  if (sp.rigid != ~0u && rb) {
    ox = rb[sp.rigid].px;
    oy = rb[sp.rigid].py;
    oz = rb[sp.rigid].pz;
  } else {
    ox = sp.ox;
    oy = sp.oy;
    oz = sp.oz;
  }
}

// A span above kReactExactSpan, one block per span: the block stages the force and torque
// terms of kReactBatch consecutive particles in shared memory while thread a (a < 6) adds
// component a of the previous batch to its running sum in index order, so the loads of
// the next batch are in flight during the sequential sums.
__global__ void __launch_bounds__(kReactThreads) k_react_long(const float4* __restrict__ bforce,
                                                              const float4* __restrict__ bpos,
                                                              const SpanDev* __restrict__ spans,
                                                              const LongSpan* __restrict__ longs,
                                                              const RigidBodyDev* __restrict__ rb,
                                                              const EngineCtl* __restrict__ ctl,
                                                              float* __restrict__ breact) {
  if (ctl->err & kErrCellCap) return;
  __shared__ float terms[2][6][kReactBatch];
  const LongSpan ch = longs[blockIdx.x];
  SpanDev sp = spans[ch.span];
  span_origin(sp, rb, sp.ox, sp.oy, sp.oz);
  auto stage = [&](uint32_t b0, uint32_t buf) {
    for (uint32_t t = threadIdx.x; t < kReactBatch; t += kReactThreads) {
      const uint32_t kk = b0 + t;
      if (kk < sp.end) {
        const float4 fk = bforce[kk];
        const float4 p = bpos[kk];
        const float rx = p.x - sp.ox, ry = p.y - sp.oy, rz = p.z - sp.oz;
        terms[buf][0][t] = fk.x;
        terms[buf][1][t] = fk.y;
        terms[buf][2][t] = fk.z;
        terms[buf][3][t] = ry * fk.z - rz * fk.y;
        terms[buf][4][t] = rz * fk.x - rx * fk.z;
        terms[buf][5][t] = rx * fk.y - ry * fk.x;
      }
    }
  };
  float f = 0.0f;  // thread a < 6: component a (force xyz, torque xyz)
  uint32_t buf = 0;
  stage(sp.start, 0);
  __syncthreads();
  for (uint32_t b0 = sp.start; b0 < sp.end; b0 += kReactBatch) {
    if (b0 + kReactBatch < sp.end) stage(b0 + kReactBatch, buf ^ 1u);
    if (threadIdx.x < 6) {
      const uint32_t nb = min(kReactBatch, sp.end - b0);
      const float* tt = terms[buf][threadIdx.x];
      uint32_t t = 0;
      for (; t + 16 <= nb; t += 16) {  // 16 terms loaded together, then added one by one
        float v[16];
#pragma unroll
        for (int i = 0; i < 16; i += 4) {
          const float4 q = *reinterpret_cast<const float4*>(tt + t + i);
          v[i] = q.x;
          v[i + 1] = q.y;
          v[i + 2] = q.z;
          v[i + 3] = q.w;
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) f = f + v[i];
      }
      for (; t < nb; ++t) f = f + tt[t];
    }
    __syncthreads();
    buf ^= 1u;
  }
  if (threadIdx.x < 6) breact[6 * ch.span + threadIdx.x] = breact[6 * ch.span + threadIdx.x] + f;
}

// Spans of at most kReactExactSpan particles, one warp each (the others: k_react_long).
__global__ void k_react_spans(const float4* __restrict__ bforce, const float4* __restrict__ bpos,
                              const SpanDev* __restrict__ spans, const RigidBodyDev* __restrict__ rb,
                              const EngineCtl* __restrict__ ctl, float* __restrict__ breact, uint32_t nspans) {
  if (ctl->err & kErrCellCap) return;
  __shared__ float terms[kReactSpanWarps][6][33];
  const uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t q = blockIdx.x * kReactSpanWarps + w;
  if (q >= nspans) return;  // uniform over the warp
  SpanDev sp = spans[q];
  span_origin(sp, rb, sp.ox, sp.oy, sp.oz);
  if (sp.end - sp.start > kReactExactSpan) return;  // uniform over the warp
  float f = 0.0f;  // lane a < 6: component a (force xyz, torque xyz)
  {
    for (uint32_t b0 = sp.start; b0 < sp.end; b0 += 32) {
      const uint32_t kk = b0 + lane;
      if (kk < sp.end) {
        const float4 fk = bforce[kk];
        const float4 p = bpos[kk];
        const float rx = p.x - sp.ox, ry = p.y - sp.oy, rz = p.z - sp.oz;
        terms[w][0][lane] = fk.x;
        terms[w][1][lane] = fk.y;
        terms[w][2][lane] = fk.z;
        terms[w][3][lane] = ry * fk.z - rz * fk.y;
        terms[w][4][lane] = rz * fk.x - rx * fk.z;
        terms[w][5][lane] = rx * fk.y - ry * fk.x;
      }
      __syncwarp();
      if (lane < 6) {
        const uint32_t nb = min(32u, sp.end - b0);
        if (nb == 32u) {  // the batch's terms loaded together, then added one by one
          float v[32];
#pragma unroll
          for (int i = 0; i < 32; ++i) v[i] = terms[w][lane][i];
#pragma unroll
          for (int i = 0; i < 32; ++i) f = f + v[i];
        } else {
          for (uint32_t t = 0; t < nb; ++t) f = f + terms[w][lane][t];
        }
      }
      __syncwarp();
    }
  }
  if (lane < 6) breact[6 * q + lane] = breact[6 * q + lane] + f;
}

// Rigid substeps of the coupling loop without contacts, one thread per body, f32 in the
// reference's order: per substep the gravity field adds g * (1 / inv_mass)
// (crates/vxl-phys-field/src/lib.rs:22-31) and the fluid reaction pass adds the tick-averaged
// reaction of the body's span (crates/vxl-phys/src/world_step.rs:235-255); then
// Integrator::integrate_velocities with gravity ZERO (v += (0 + F inv_m) dt; w += I_world^-1 tau
// dt with I_world^-1 = R diag(I^-1) R^T, crates/vxl-phys-core/src/body.rs:172-176; whole-vector
// speed clamps) and integrate_positions (x += v dt; q = normalize(q + dt/2 (0, w) q),
// crates/vxl-phys-core/src/math.rs:216-252), crates/vxl-phys-integrate/src/lib.rs:18-60.
// `with_reaction` is 0 before the first fluid tick of the loop (no reaction yet).
__device__ __forceinline__ void rigid_world_inv_inertia(const RigidBodyDev& b, float lx, float ly, float lz,
                                                        float& ox, float& oy, float& oz) {
  const float xx = b.qx * b.qx, yy = b.qy * b.qy, zz = b.qz * b.qz;
  const float xy = b.qx * b.qy, xz = b.qx * b.qz, yz = b.qy * b.qz;
  const float wx = b.qw * b.qx, wy = b.qw * b.qy, wz = b.qw * b.qz;
  const float m00 = 1.0f - 2.0f * (yy + zz), m01 = 2.0f * (xy - wz), m02 = 2.0f * (xz + wy);
  const float m10 = 2.0f * (xy + wz), m11 = 1.0f - 2.0f * (xx + zz), m12 = 2.0f * (yz - wx);
  const float m20 = 2.0f * (xz - wy), m21 = 2.0f * (yz + wx), m22 = 1.0f - 2.0f * (xx + yy);
  const float tx = m00 * lx + m10 * ly + m20 * lz;
  const float ty = m01 * lx + m11 * ly + m21 * lz;
  const float tz = m02 * lx + m12 * ly + m22 * lz;
  const float vx = tx * b.iix, vy = ty * b.iiy, vz = tz * b.iiz;
  ox = m00 * vx + m01 * vy + m02 * vz;
  oy = m10 * vx + m11 * vy + m12 * vz;
  oz = m20 * vx + m21 * vy + m22 * vz;
}

__global__ void k_rigid_step(RigidBodyDev* __restrict__ bodies, uint32_t n, const float* __restrict__ breact,
                             int with_reaction, float gx, float gy, float gz, float dt, uint32_t substeps,
                             float max_linear, float max_angular) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  RigidBodyDev b = bodies[i];
  if (!b.dynamic) return;
  float rf[6] = {0, 0, 0, 0, 0, 0};
  if (with_reaction && b.span != ~0u)
    for (int a = 0; a < 6; ++a) rf[a] = breact[6 * b.span + a];
  const float hd = 0.5f * dt;
  for (uint32_t k = 0; k < substeps; ++k) {
    const float mass = 1.0f / b.inv_mass;
    float fx = 0.0f + gx * mass, fy = 0.0f + gy * mass, fz = 0.0f + gz * mass;
    fx = fx + rf[0];
    fy = fy + rf[1];
    fz = fz + rf[2];
    const float tqx = 0.0f + rf[3], tqy = 0.0f + rf[4], tqz = 0.0f + rf[5];
    b.vx = b.vx + (0.0f + fx * b.inv_mass) * dt;
    b.vy = b.vy + (0.0f + fy * b.inv_mass) * dt;
    b.vz = b.vz + (0.0f + fz * b.inv_mass) * dt;
    float ax, ay, az;
    rigid_world_inv_inertia(b, tqx, tqy, tqz, ax, ay, az);
    b.wx = b.wx + ax * dt;
    b.wy = b.wy + ay * dt;
    b.wz = b.wz + az * dt;
    const float sp = sqrtf(b.vx * b.vx + b.vy * b.vy + b.vz * b.vz);
    if (sp > max_linear) {
      const float s = max_linear / sp;
      b.vx = b.vx * s;
      b.vy = b.vy * s;
      b.vz = b.vz * s;
    }
    const float ws = sqrtf(b.wx * b.wx + b.wy * b.wy + b.wz * b.wz);
    if (ws > max_angular) {
      const float s = max_angular / ws;
      b.wx = b.wx * s;
      b.wy = b.wy * s;
      b.wz = b.wz * s;
    }
    b.px = b.px + b.vx * dt;
    b.py = b.py + b.vy * dt;
    b.pz = b.pz + b.vz * dt;
    // dq = (w, 0) * q (Hamilton), then q + dq dt/2, normalized
    const float dqx = 0.0f * b.qx + b.wx * b.qw + b.wy * b.qz - b.wz * b.qy;
    const float dqy = 0.0f * b.qy - b.wx * b.qz + b.wy * b.qw + b.wz * b.qx;
    const float dqz = 0.0f * b.qz + b.wx * b.qy - b.wy * b.qx + b.wz * b.qw;
    const float dqw = 0.0f * b.qw - b.wx * b.qx - b.wy * b.qy - b.wz * b.qz;
    const float nx = b.qx + dqx * hd, ny = b.qy + dqy * hd, nz = b.qz + dqz * hd, nw = b.qw + dqw * hd;
    const float len2 = nx * nx + ny * ny + nz * nz + nw * nw;
    if (len2 > 1e-16f) {
      const float inv = 1.0f / sqrtf(len2);
      b.qx = nx * inv;
      b.qy = ny * inv;
      b.qz = nz * inv;
      b.qw = nw * inv;
    } else {
      b.qx = 0.0f;
      b.qy = 0.0f;
      b.qz = 0.0f;
      b.qw = 1.0f;
    }
  }
  bodies[i] = b;
}

// Tick average (fluid_step.rs:84-88): e *= 1 / substeps.
__global__ void k_scale(float* __restrict__ breact, uint32_t n, float inv) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) breact[i] = breact[i] * inv;
}

// ---------------------------------------------------------------- export kernels

// One scene's state in its reference order (scene-local index).
__global__ void k_e_read_scene(const float4* __restrict__ pos, const float4* __restrict__ vel,
                               const uint32_t* __restrict__ orig, float* __restrict__ pout, float* __restrict__ vout,
                               uint32_t base, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t s = base + i;
  const uint32_t o = orig[s] - base;
  if (pout) {
    const float4 p = pos[s];
    pout[3 * o] = p.x;
    pout[3 * o + 1] = p.y;
    pout[3 * o + 2] = p.z;
  }
  if (vout) {
    const float4 v = vel[s];
    vout[3 * o] = v.x;
    vout[3 * o + 1] = v.y;
    vout[3 * o + 2] = v.z;
  }
}

__global__ void k_e_read_fields(const float2* __restrict__ rc, const float* __restrict__ press,
                                const float4* __restrict__ acc, const float4* __restrict__ xsph,
                                const uint32_t* __restrict__ orig, float* __restrict__ dout, float* __restrict__ pout,
                                float* __restrict__ aout, float* __restrict__ xout, uint32_t base, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t s = base + i;
  const uint32_t o = orig[s] - base;
  if (dout) dout[o] = rc[s].x;
  if (pout) pout[o] = press[s];
  if (aout) {
    const float4 a = acc[s];
    aout[3 * o] = a.x;
    aout[3 * o + 1] = a.y;
    aout[3 * o + 2] = a.z;
  }
  if (xout) {
    const float4 x = xsph[s];
    xout[3 * o] = x.x;
    xout[3 * o + 1] = x.y;
    xout[3 * o + 2] = x.z;
  }
}

// Per-particle cell (scene-local cell index) of one scene, from its slice of the table.
__global__ void k_e_export_bins(const uint32_t* __restrict__ start, const uint32_t* __restrict__ orig,
                                const SceneDev* __restrict__ sc, uint32_t scene, uint32_t* __restrict__ bins) {
  const SceneDev& S = sc[scene];
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= S.cells) return;
  const uint32_t gc = S.cell_off + c;
  for (uint32_t q = start[gc]; q < start[gc + 1]; ++q) bins[orig[q] - S.base] = c;
}

// One scene's slice of the cell table, rebased to the scene's first slot.
// Contact table entries by global reference index: ent[ids[e]] = e + 1 (ent zeroed before).
__global__ void k_e_ctab_scatter(const uint32_t* __restrict__ ids, uint32_t n, uint32_t* __restrict__ ent) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) ent[ids[e]] = e + 1u;
}

// Neighbour-list export of one scene (last substep): the list count of each slot in the
// scene's reference order.
__global__ void k_e_export_nbr_counts(const uint32_t* __restrict__ nbr_n, const uint32_t* __restrict__ orig,
                                      uint32_t base, uint32_t n, uint32_t* __restrict__ out) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) out[orig[base + t] - base] = nbr_n[base + t] & ~kListBad;
}

// The entries of each slot's list, in its walk order, as scene-local reference indices,
// at offsets[reference index]: the recorded list, or for a list longer than the cap the
// same neighbours walked again from the sorted positions and cell table of that substep
// (the walk the force pass and the boundary gather fall back to).
__global__ void k_e_export_nbr_entries(const float4* __restrict__ pos, const uint32_t* __restrict__ start,
                                       const SceneDev* __restrict__ sc, uint32_t q, const uint32_t* __restrict__ orig,
                                       const uint16_t* __restrict__ nbr, const uint32_t* __restrict__ nbr_n,
                                       uint32_t cap, uint32_t stride, const unsigned long long* __restrict__ offsets,
                                       uint32_t* __restrict__ out) {
  const SceneDev& S = sc[q];
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= S.count) return;
  const uint32_t s = S.base + t;
  const uint32_t base = S.base;
  unsigned long long o = offsets[orig[s] - base];
  const uint32_t c = nbr_n[s];
  const GridBox g = S.g;
  const float4 pi = pos[s];
  uint32_t cx, cy, cz;
  bin_of(g, pi.x, pi.y, pi.z, cx, cy, cz);
  if (c <= cap) {
    const ListPlanes lp = list_planes(g, start + S.cell_off, cx, cy, cz);
    for (uint32_t k = 0; k < c; ++k) out[o + k] = orig[list_decode(lp, nbr[(size_t)k * stride + s])] - base;
    return;
  }
  const bool fluid_i = pi.w > 0.0f;
  const float h2 = S.k.h2;
  walk27<true>(g, start + S.cell_off, pi.x, pi.y, pi.z, cx, cy, cz, S.k.h, [&](uint32_t j) {
    const float4 pj = pos[j];
    const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
    const float r2 = dx * dx + dy * dy + dz * dz;
    if (r2 <= h2 && (fluid_i || pj.w > 0.0f)) out[o++] = orig[j] - base;
  }, s);
}

__global__ void k_e_export_items(const uint32_t* __restrict__ orig, uint32_t base, uint32_t n,
                                 uint32_t* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = orig[base + i] - base;
}

}  // namespace
}  // namespace vxl
