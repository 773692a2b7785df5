// Neighbour-table build that allocates nothing: vxl_sph_build_grid_static.
//
// Some callers cannot allocate device memory while they run: an engine that reserves
// one fixed arena for all GPU work at start-up and forbids further cudaMalloc, or a
// per-frame plugin that must not call cudaMalloc/cudaFree because both can synchronise
// the device and stall the host's frame loop. This entry point serves them. The caller
// passes device buffers for the input positions and the output table; the working
// memory the sort needs (cell counts, per-particle cell and rank, the unordered
// placement and the scan partials) lives in one file-scope __device__ array of fixed
// size, which every GPU that loads this library holds until the process exits.
//
// The table is the one the handle-based path builds at the start of each substep
// (crates/vxl-phys-fluid/src/grid.rs:29-76 with the grid rule of
// crates/vxl-phys-core/src/grid.rs:34-50): items[] = particle indices grouped by cell,
// ascending index inside a cell; start[c]..start[c+1] = the slots of cell c.
#include <cstring>
#include <mutex>
#include <string>

#include "sph_device.cuh"
#include "vxl_sph.h"
#include "vxl_sph_internal.h"

using namespace vxl;

namespace {

constexpr uint32_t kStaticMaxParticles = 1u << 19;  // 524,288
constexpr uint32_t kStaticMaxCells = 1u << 19;      // 524,288
constexpr int kTile = 2048;
constexpr int kTileThreads = 256;
constexpr uint32_t kMaxTiles = (kStaticMaxCells + kTile - 1) / kTile;  // 256
constexpr int kWideThreads = 512;                                          // block of ks_canon_wide
constexpr uint32_t kWideRank = 2048;  // cells up to this size are ranked in shared memory
constexpr uint32_t kWideSmemWords = (kStaticMaxParticles + 31) / 32 > kWideRank ? (kStaticMaxParticles + 31) / 32
                                                                               : kWideRank;  // 64 KB

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kCountsOff = 0;
constexpr size_t kRankOff = align256(kCountsOff + (size_t)(kStaticMaxCells + 1) * 4);
constexpr size_t kTmpOff = align256(kRankOff + (size_t)kStaticMaxParticles * 8);
constexpr size_t kPartialOff = align256(kTmpOff + (size_t)kStaticMaxParticles * 4);
constexpr size_t kBoxOff = align256(kPartialOff + (size_t)kMaxTiles * 4);
constexpr size_t kGridOff = align256(kBoxOff + 6 * 4);
constexpr size_t kScratchBytes = align256(kGridOff + sizeof(GridBox));

// The working memory (about 8.4 MB). Host code must not pass this name to a kernel: on
// the host it is only a stand-in; the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_grid_scratch[kScratchBytes];

std::mutex g_mu;
void* g_scratch_addr[128] = {};  // per device ordinal, resolved on the first call there

vxl_status fail(vxl_status s, const std::string& m) {
  vxl_set_last_error(m.c_str());  // read back through vxl_sph_last_error()
  return s;
}

__device__ __forceinline__ void box_reduce(uint32_t* acc, float x, float y, float z, bool valid) {
  uint32_t mn[3], mx[3];
  const float v[3] = {x, y, z};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const bool ok = valid && (v[a] == v[a]);
    mn[a] = ok ? f2o(v[a]) : 0xffffffffu;
    mx[a] = ok ? f2o(v[a]) : 0u;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      mn[a] = min(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], off));
      mx[a] = max(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], off));
    }
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (mn[a] != 0xffffffffu) atomicMin(&acc[a], mn[a]);
      if (mx[a] != 0u) atomicMax(&acc[3 + a], mx[a]);
    }
}

__global__ void ks_init(uint32_t* box) {
  if (threadIdx.x < 3) box[threadIdx.x] = 0xffffffffu;
  else if (threadIdx.x < 6) box[threadIdx.x] = 0u;
}

__global__ void ks_bbox(const float* __restrict__ xyz, uint32_t n, uint32_t* box) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool ok = i < n;
  box_reduce(box, ok ? xyz[3 * i] : 0.f, ok ? xyz[3 * i + 1] : 0.f, ok ? xyz[3 * i + 2] : 0.f, ok);
}

__global__ void ks_gridbox(const uint32_t* box, float h, uint32_t max_bins, GridBox* g) {
  if (threadIdx.x != 0) return;
  GridBox gb;
  grid_box(o2f(box[0]), o2f(box[1]), o2f(box[2]), o2f(box[3]), o2f(box[4]), o2f(box[5]), h, max_bins, gb);
  *g = gb;
}

__global__ void ks_keys(const float* __restrict__ xyz, uint32_t n, const GridBox* __restrict__ gp,
                        uint32_t* __restrict__ counts, uint2* __restrict__ cellrank) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < n;
  uint32_t c = 0xffffffffu;
  if (valid) c = cell_index(*gp, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
  const uint32_t active = __ballot_sync(0xffffffffu, valid);
  if (!valid) return;
  const uint32_t peers = __match_any_sync(active, c);
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(peers) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(&counts[c], (uint32_t)__popc(peers));
  base = __shfl_sync(peers, base, leader);
  cellrank[i] = make_uint2(c, base + __popc(peers & ((1u << lane) - 1u)));
}

__global__ void ks_scan_partial(const uint32_t* __restrict__ counts, const GridBox* __restrict__ gp,
                                uint32_t* __restrict__ partial) {
  const uint32_t total = gp->total, base = blockIdx.x * kTile;
  if (base >= total) return;
  uint32_t sum = 0;
  for (uint32_t i = base + threadIdx.x; i < min(base + kTile, total); i += kTileThreads) sum += counts[i];
  for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off);
  __shared__ uint32_t ws[kTileThreads / 32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < kTileThreads / 32; ++w) t += ws[w];
    partial[blockIdx.x] = t;
  }
}

__global__ void ks_scan_top(uint32_t* __restrict__ partial, const GridBox* __restrict__ gp,
                            uint32_t* __restrict__ start) {
  const uint32_t total = gp->total, ntiles = (total + kTile - 1) / kTile;
  __shared__ uint32_t sh[kMaxTiles];
  const uint32_t t = threadIdx.x;
  const uint32_t v = t < ntiles ? partial[t] : 0u;
  sh[t] = v;
  __syncthreads();
  for (uint32_t off = 1; off < kMaxTiles; off <<= 1) {
    const uint32_t add = t >= off ? sh[t - off] : 0u;
    __syncthreads();
    sh[t] += add;
    __syncthreads();
  }
  if (t < ntiles) partial[t] = sh[t] - v;
  if (t == kMaxTiles - 1) start[total] = sh[kMaxTiles - 1];
}

__global__ void ks_scan_final(const uint32_t* __restrict__ counts, const GridBox* __restrict__ gp,
                              const uint32_t* __restrict__ partial, uint32_t* __restrict__ start) {
  const uint32_t total = gp->total, base = blockIdx.x * kTile;
  if (base >= total) return;
  constexpr int kPer = kTile / kTileThreads;
  uint32_t v[kPer], local = 0;
  const uint32_t i0 = base + threadIdx.x * kPer;
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
  __shared__ uint32_t ws[kTileThreads / 32];
  if (lane == 31) ws[wid] = incl;
  __syncthreads();
  uint32_t woff = 0;
  for (int w = 0; w < wid; ++w) woff += ws[w];
  uint32_t run = partial[blockIdx.x] + woff + incl - local;
#pragma unroll
  for (int q = 0; q < kPer; ++q) {
    if ((i0 + q) < total) start[i0 + q] = run;
    run += v[q];
  }
}

__global__ void ks_place(const uint2* __restrict__ cellrank, const uint32_t* __restrict__ start, uint32_t n,
                         uint32_t* __restrict__ tmp) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint2 cr = cellrank[i];
  tmp[start[cr.x] + cr.y] = i;
}

// One warp per cell of at most 32 entries: the placed indices of the cell, in ascending
// order, into items (each lane ranks its entry against the others).
__global__ void ks_canon(const uint32_t* __restrict__ tmp, const uint32_t* __restrict__ start,
                         const GridBox* __restrict__ gp, uint32_t* __restrict__ items) {
  const uint32_t total = gp->total;
  const int lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < total; c += warps) {
    const uint32_t b = start[c], n = start[c + 1] - b;
    if (n > 32) continue;  // ks_canon_wide
    const uint32_t key = lane < (int)n ? tmp[b + lane] : 0xffffffffu;
    uint32_t rank = 0;
    for (uint32_t j = 0; j < n; ++j) rank += __shfl_sync(0xffffffffu, key, (int)j) < key ? 1u : 0u;
    if (lane < (int)n) items[b + rank] = key;
  }
}

// Cells of more than 32 entries, one block per cell in turn. Up to kWideRank entries:
// each thread ranks entries against the cell's keys in shared memory (m^2 / kWideThreads
// shared reads per thread). More: the cell's indices are distinct values below n, so
// they are set in a bitmap of n bits in shared memory and read back in ascending order
// (n / 32 words scanned once, whatever the cell's size).
__global__ void __launch_bounds__(kWideThreads) ks_canon_wide(const uint32_t* __restrict__ tmp,
                                                              const uint32_t* __restrict__ start,
                                                              const GridBox* __restrict__ gp, uint32_t n,
                                                              uint32_t* __restrict__ items) {
  extern __shared__ uint32_t sm[];  // kWideSmemWords
  __shared__ uint32_t s_warp[kWideThreads / 32];
  const uint32_t total = gp->total;
  const uint32_t t = threadIdx.x, lane = t & 31, wid = t >> 5;
  for (uint32_t c = blockIdx.x; c < total; c += gridDim.x) {
    const uint32_t b = start[c], m = start[c + 1] - b;
    if (m <= 32) continue;
    if (m <= kWideRank) {
      for (uint32_t e = t; e < m; e += kWideThreads) sm[e] = tmp[b + e];
      __syncthreads();
      for (uint32_t e = t; e < m; e += kWideThreads) {
        const uint32_t key = sm[e];
        uint32_t rank = 0;
        for (uint32_t j = 0; j < m; ++j) rank += sm[j] < key ? 1u : 0u;
        items[b + rank] = key;
      }
      __syncthreads();
      continue;
    }
    const uint32_t words = (n + 31) / 32;
    for (uint32_t w = t; w < words; w += kWideThreads) sm[w] = 0;
    __syncthreads();
    for (uint32_t e = t; e < m; e += kWideThreads) {
      const uint32_t v = tmp[b + e];
      atomicOr(&sm[v >> 5], 1u << (v & 31));
    }
    __syncthreads();
    // thread t owns words [w0, w1); exclusive scan of their set bits over the block
    const uint32_t per = (words + kWideThreads - 1) / kWideThreads;
    const uint32_t w0 = min(t * per, words), w1 = min(w0 + per, words);
    uint32_t cnt = 0;
    for (uint32_t w = w0; w < w1; ++w) cnt += __popc(sm[w]);
    uint32_t incl = cnt;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, off);
      if ((int)lane >= off) incl += y;
    }
    if (lane == 31) s_warp[wid] = incl;
    __syncthreads();
    uint32_t r = incl - cnt;
    for (uint32_t k = 0; k < wid; ++k) r += s_warp[k];
    for (uint32_t w = w0; w < w1; ++w) {
      uint32_t bits = sm[w];
      while (bits) {
        const uint32_t bit = (uint32_t)__ffs(bits) - 1u;
        bits &= bits - 1u;
        items[b + r++] = w * 32u + bit;
      }
    }
    __syncthreads();
  }
}

// Device address of the scratch array on the current device (resolved once per device).
vxl_status scratch_on(int dev, unsigned char** out) {
  if (dev < 0 || dev >= 128) return fail(VXL_INVALID_ARGUMENT, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_grid_scratch);
    if (e != cudaSuccess || !p)
      return fail(VXL_CUDA_ERROR, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    e = cudaFuncSetAttribute(ks_canon_wide, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(kWideSmemWords * sizeof(uint32_t)));
    if (e != cudaSuccess)
      return fail(VXL_CUDA_ERROR, std::string("cudaFuncSetAttribute(ks_canon_wide): ") + cudaGetErrorString(e));
    g_scratch_addr[dev] = p;
  }
  *out = (unsigned char*)g_scratch_addr[dev];
  return VXL_OK;
}

}  // namespace

extern "C" vxl_status vxl_sph_build_grid_static(const float* d_pos_xyz, uint32_t n, float h, uint32_t max_bins,
                                                uint32_t* d_items, uint32_t* d_start, uint64_t start_cap,
                                                vxl_sph_grid_info* info, void* cuda_stream) {
  if (!d_pos_xyz || !d_items || !d_start || !info) return fail(VXL_NULL_POINTER, "NULL argument");
  if (info->hdr.size != sizeof(vxl_sph_grid_info) || info->hdr.version != VXL_SPH_ABI_VERSION)
    return fail(VXL_SIZE_MISMATCH, "grid_info header");
  if (n == 0 || n > kStaticMaxParticles)
    return fail(VXL_INVALID_ARGUMENT, "n must be in [1, " + std::to_string(kStaticMaxParticles) + "]");
  const uint32_t budget = max_bins ? max_bins : kStaticMaxCells;
  if (budget > kStaticMaxCells)
    return fail(VXL_INVALID_ARGUMENT, "max_bins above the static limit of " + std::to_string(kStaticMaxCells));
  if (start_cap < (uint64_t)budget + 1)
    return fail(VXL_SIZE_MISMATCH, "start must hold max_bins + 1 entries");
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(VXL_CUDA_ERROR, "cudaGetDevice failed");
  unsigned char* base = nullptr;
  vxl_status st = scratch_on(dev, &base);
  if (st != VXL_OK) return st;
  cudaStream_t s = (cudaStream_t)cuda_stream;
  uint32_t* counts = (uint32_t*)(base + kCountsOff);
  uint2* cellrank = (uint2*)(base + kRankOff);
  uint32_t* tmp = (uint32_t*)(base + kTmpOff);
  uint32_t* partial = (uint32_t*)(base + kPartialOff);
  uint32_t* box = (uint32_t*)(base + kBoxOff);
  GridBox* g = (GridBox*)(base + kGridOff);
  const uint32_t nblk = (n + 255) / 256, tiles = (budget + kTile - 1) / kTile;
  // the array keeps the previous call's contents: zero the counts and reset the box
  cudaError_t e = cudaMemsetAsync(counts, 0, ((size_t)budget + 1) * 4, s);
  if (e != cudaSuccess) return fail(VXL_CUDA_ERROR, std::string("grid build: ") + cudaGetErrorString(e));
  ks_init<<<1, 32, 0, s>>>(box);
  ks_bbox<<<nblk, 256, 0, s>>>(d_pos_xyz, n, box);
  ks_gridbox<<<1, 32, 0, s>>>(box, h, budget, g);
  ks_keys<<<nblk, 256, 0, s>>>(d_pos_xyz, n, g, counts, cellrank);
  ks_scan_partial<<<tiles, kTileThreads, 0, s>>>(counts, g, partial);
  ks_scan_top<<<1, kMaxTiles, 0, s>>>(partial, g, d_start);
  ks_scan_final<<<tiles, kTileThreads, 0, s>>>(counts, g, partial, d_start);
  ks_place<<<nblk, 256, 0, s>>>(cellrank, d_start, n, tmp);
  ks_canon<<<148 * 4, 256, 0, s>>>(tmp, d_start, g, d_items);
  ks_canon_wide<<<148 * 2, kWideThreads, kWideSmemWords * sizeof(uint32_t), s>>>(tmp, d_start, g, n, d_items);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(VXL_CUDA_ERROR, std::string("grid build launch: ") + cudaGetErrorString(e));
  GridBox hg;
  e = cudaMemcpyAsync(&hg, g, sizeof(GridBox), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(VXL_CUDA_ERROR, std::string("grid build: ") + cudaGetErrorString(e));
  info->min[0] = hg.minx;
  info->min[1] = hg.miny;
  info->min[2] = hg.minz;
  info->inv = hg.inv;
  info->bin = hg.bin;
  info->dims[0] = hg.nx;
  info->dims[1] = hg.ny;
  info->dims[2] = hg.nz;
  info->total = hg.total;
  return VXL_OK;
}
