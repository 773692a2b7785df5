// C ABI of the plain (single-scene) WCSPH step: resident device state, the substep
// launch sequence, CUDA-graph replay of whole ticks, and the export paths.
//
// Reference seam: FluidStepper (crates/vxl-phys-core/src/interop.rs:293-316) as
// implemented by GpuFluidStepper (crates/vxl-phys-gpu/src/pipeline/stepper.rs:22-147).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "sph_kernels.cuh"
#include "vxl_sph.h"
#include "vxl_sph_internal.h"

using namespace vxl;

namespace {

thread_local std::string g_last_error;

vxl_status fail(vxl_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

#define CU(call)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return fail(VXL_CUDA_ERROR, std::string(#call) + ": " + cudaGetErrorString(e_));       \
  } while (0)

constexpr int kThreads = 256;

// VXL_SPH_DEBUG=1: report, on stderr, any CUDA runtime error left pending at the entry
// or exit of a public call (attributes a sticky error to the call that caused it).
bool debug_on() {
  static int on = -1;
  if (on < 0) {
    const char* e = std::getenv("VXL_SPH_DEBUG");
    on = (e && e[0] == '1') ? 1 : 0;
  }
  return on == 1;
}

struct ApiTrace {
  const char* fn;
  explicit ApiTrace(const char* f) : fn(f) {
    if (debug_on()) {
      cudaError_t e = cudaPeekAtLastError();
      if (e != cudaSuccess) std::fprintf(stderr, "[vxl_sph] pending at entry of %s: %s\n", fn, cudaGetErrorString(e));
    }
  }
  ~ApiTrace() {
    if (debug_on()) {
      cudaError_t e = cudaPeekAtLastError();
      if (e != cudaSuccess) std::fprintf(stderr, "[vxl_sph] pending at exit of %s: %s\n", fn, cudaGetErrorString(e));
    }
  }
};
#define API_TRACE() ApiTrace api_trace_(__func__)

inline uint32_t blocks_for(uint64_t n, int t = kThreads) { return (uint32_t)((n + t - 1) / t); }

}  // namespace

void vxl_set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }

struct vxl_sph_handle {
  int device = 0;
  cudaStream_t stream = nullptr;      // stream all work is enqueued on
  cudaStream_t own_stream = nullptr;  // the handle's own stream (destroyed with it)
  vxl_sph_params params{};
  SphConst k{};
  uint64_t nf = 0, nb = 0, nt = 0;
  uint32_t max_bins = 0;
  uint32_t substeps = 1;

  float4* pos[2] = {nullptr, nullptr};
  float4* vel[2] = {nullptr, nullptr};
  uint32_t* orig = nullptr;
  uint32_t* slot_of = nullptr;
  uint2* cellrank = nullptr;
  uint2* items = nullptr;
  uint32_t* counts = nullptr;
  uint32_t* start = nullptr;
  uint32_t* partial = nullptr;
  float2* rc = nullptr;
  float* press = nullptr;
  float4* acc = nullptr;
  float4* xsph = nullptr;
  float4* bforce = nullptr;
  float4* bpos = nullptr;
  uint32_t* nbr = nullptr;    // neighbour list, nbr[k * nt + s], k < nbr_cap
  uint32_t* nbr_n = nullptr;  // neighbour count per slot
  uint32_t nbr_cap = 64;
  Ctl* ctl = nullptr;
  float* stage = nullptr;  // 8 * nt floats: device staging for host uploads/exports
  SpanDev* spans_d = nullptr;
  SpanDev* spans_h = nullptr;  // pinned
  uint32_t spans_cap = 0;
  float* breact_d = nullptr;
  float* breact_h = nullptr;  // pinned
  SpanChunk* chunks_d = nullptr;
  SpanChunk* chunks_h = nullptr;  // pinned
  uint32_t* chunk_first_d = nullptr;
  uint32_t* chunk_first_h = nullptr;  // pinned
  float* react_partial = nullptr;
  uint32_t chunks_cap = 0;
  uint32_t nchunks = 0;
  uint32_t graph_nchunks = 0;
  Ctl* ctl_h = nullptr;       // pinned
  bool record = false;
  bool ran_substep = false;

  cudaGraphExec_t graph = nullptr;
  float graph_dt = 0.f;
  uint32_t graph_nspans = 0;
  bool graph_record = false;
  bool use_graph = true;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  uint64_t launches_last_tick = 0;
  uint64_t launches_counter = 0;
  uint64_t device_bytes = 0;
  uint32_t last_nspans = 0;

  // per-kernel device timers (vxl_sph_set_profile)
  bool prof = false;
  bool capturing = false;  // inside cudaStreamBeginCapture .. EndCapture
  bool graph_prof = false;
  bool prof_pending = false;
  std::vector<cudaEvent_t> prof_ev;
  std::vector<int> prof_kid;
  size_t prof_used = 0;
  double prof_ms[16] = {};
  uint64_t prof_n[16] = {};
};

namespace {

template <class T>
vxl_status dalloc(vxl_sph_handle* h, T** p, size_t count) {
  size_t bytes = count * sizeof(T);
  if (bytes == 0) bytes = sizeof(T);
  cudaError_t e = cudaMalloc((void**)p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    return fail(VXL_OUT_OF_MEMORY, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  h->device_bytes += bytes;
  return VXL_OK;
}

void free_all(vxl_sph_handle* h) {
  if (h->graph) cudaGraphExecDestroy(h->graph);
  void* ptrs[] = {h->pos[0], h->pos[1], h->vel[0], h->vel[1], h->orig, h->slot_of, h->cellrank, h->items,
                  h->counts, h->start, h->partial, h->rc, h->press, h->acc, h->xsph, h->bforce, h->bpos,
                  h->ctl, h->stage, h->spans_d, h->breact_d, h->nbr, h->nbr_n, h->chunks_d,
                  h->chunk_first_d, h->react_partial};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (h->spans_h) cudaFreeHost(h->spans_h);
  if (h->breact_h) cudaFreeHost(h->breact_h);
  if (h->chunks_h) cudaFreeHost(h->chunks_h);
  if (h->chunk_first_h) cudaFreeHost(h->chunk_first_h);
  if (h->ctl_h) cudaFreeHost(h->ctl_h);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  for (cudaEvent_t e : h->prof_ev) cudaEventDestroy(e);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
}

// Kernel names of the per-kernel timer table (index = id).
enum KernelId : int {
  KID_GRIDBOX, KID_KEYS, KID_SCAN_PARTIAL, KID_SCAN_TOP, KID_SCAN_FINAL, KID_PLACE, KID_CANON,
  KID_DENSITY, KID_FORCE, KID_BFORCE, KID_REACT_CHUNKS, KID_REACT_SPANS, KID_SCALE, KID_COUNT
};
const char* const kKernelNames[KID_COUNT] = {
  "k_gridbox", "k_keys", "k_scan_partial", "k_scan_top", "k_scan_final", "k_place", "k_canon",
  "k_density", "k_force", "k_bforce", "k_react_chunks", "k_react_spans", "k_scale"};

// Inside stream capture a plain cudaEventRecord only expresses a dependency; the
// External flag makes the graph record the event each time it runs.
void record_event(vxl_sph_handle* h, cudaEvent_t e) {
  if (h->capturing) cudaEventRecordWithFlags(e, h->stream, cudaEventRecordExternal);
  else cudaEventRecord(e, h->stream);
}

int prof_begin(vxl_sph_handle* h, int kid) {
  if (!h->prof) return -1;
  if (2 * h->prof_used + 2 > h->prof_ev.size()) {
    for (int q = 0; q < 64; ++q) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      h->prof_ev.push_back(e);
    }
    h->prof_kid.resize(h->prof_ev.size() / 2);
  }
  size_t i = h->prof_used++;
  h->prof_kid[i] = kid;
  record_event(h, h->prof_ev[2 * i]);
  return (int)i;
}

void prof_end(vxl_sph_handle* h, int i) {
  if (i >= 0) record_event(h, h->prof_ev[2 * i + 1]);
}

// Add the elapsed times of the last enqueued tick (waits for it).
void prof_collect(vxl_sph_handle* h) {
  if (!h->prof_pending) return;
  cudaStreamSynchronize(h->stream);
  for (size_t i = 0; i < h->prof_used; ++i) {
    float ms = 0.f;
    cudaError_t e = cudaEventElapsedTime(&ms, h->prof_ev[2 * i], h->prof_ev[2 * i + 1]);
    if (e == cudaSuccess) {
      h->prof_ms[h->prof_kid[i]] += ms;
      h->prof_n[h->prof_kid[i]] += 1;
    } else {
      if (debug_on()) std::fprintf(stderr, "[vxl_sph] cudaEventElapsedTime(%zu): %s\n", i, cudaGetErrorString(e));
      cudaGetLastError();  // the timer pair is dropped; do not leave the error pending
    }
  }
  h->prof_pending = false;
}

#define LAUNCH(kid, ...)                 \
  do {                                   \
    int pe_ = prof_begin(h, kid);        \
    __VA_ARGS__;                         \
    prof_end(h, pe_);                    \
    h->launches_counter += 1;            \
  } while (0)

bool check_header(const vxl_block_header& hd, uint32_t size) {
  return hd.size == size && hd.version == VXL_SPH_ABI_VERSION;
}

// crates/vxl-phys-fluid/src/fluid_access.rs:8-13: h, h2, k6, ks, w0, B in f32 with the
// reference's operation order (host code is built with -ffp-contract=off).
SphConst make_const(const vxl_sph_params& p, uint64_t nf, uint64_t nt, uint32_t max_bins) {
  SphConst k{};
  float h = std::fmax(p.smoothing_radius, 1e-5f);
  float h2 = h * h;
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

// Launch one substep (crates/vxl-phys-fluid/src/fluid_step.rs:91-127) on h->stream.
void enqueue_substep(vxl_sph_handle* h, float dt, uint32_t nspans) {
  cudaStream_t st = h->stream;
  const uint32_t nt = (uint32_t)h->nt;
  const uint32_t nblk = blocks_for(nt);
  const uint32_t tiles = (h->max_bins + kScanTile - 1) / kScanTile;
  StepConst sc;
  sc.dt = dt;
  sc.vmax = h->params.max_speed_frac * h->k.h / dt;
  sc.vmax2 = sc.vmax * sc.vmax;
  LAUNCH(KID_GRIDBOX, k_gridbox<<<1, 32, 0, st>>>(h->ctl, h->k.h, h->max_bins));
  LAUNCH(KID_KEYS, k_keys<<<nblk, kThreads, 0, st>>>(h->pos[0], h->ctl, h->counts, h->cellrank, nt));
  LAUNCH(KID_SCAN_PARTIAL, k_scan_partial<<<tiles, kScanThreads, 0, st>>>(h->counts, h->ctl, h->partial));
  LAUNCH(KID_SCAN_TOP, k_scan_top<<<1, 1024, 0, st>>>(h->partial, h->ctl, h->start));
  LAUNCH(KID_SCAN_FINAL, k_scan_final<<<tiles, kScanThreads, 0, st>>>(h->counts, h->ctl, h->partial, h->start));
  LAUNCH(KID_PLACE, k_place<<<nblk, kThreads, 0, st>>>(h->cellrank, h->start, h->orig, h->items, nt));
  LAUNCH(KID_CANON, k_canon<<<148 * 8, 256, 0, st>>>(h->items, h->start, h->ctl, h->pos[0], h->vel[0], h->pos[1],
                                                     h->vel[1], h->orig, h->slot_of));
  LAUNCH(KID_DENSITY, k_density<<<nblk, kThreads, 0, st>>>(h->pos[1], h->start, h->ctl, h->rc, h->press, h->nbr,
                                                           h->nbr_n, h->nbr_cap, h->k));
  LAUNCH(KID_FORCE, k_force<<<nblk, kThreads, 0, st>>>(h->pos[1], h->vel[1], h->rc, h->start, h->nbr, h->nbr_n,
                                                       h->nbr_cap, h->ctl, h->pos[0], h->vel[0],
                                                       h->record ? h->acc : nullptr, h->record ? h->xsph : nullptr,
                                                       h->k, sc));
  if (h->nb > 0 && (nspans > 0 || h->record)) {
    LAUNCH(KID_BFORCE, k_bforce<<<blocks_for(nt, 128), 128, 0, st>>>(h->pos[1], h->vel[1], h->rc, h->start, h->orig,
                                                                     h->nbr, h->nbr_n, h->nbr_cap, h->ctl,
                                                                     h->bforce, h->k));
  }
  if (nspans > 0 && h->nchunks > 0) {
    LAUNCH(KID_REACT_CHUNKS, k_react_chunks<<<h->nchunks, kReactThreads, 0, st>>>(
                                 h->bforce, h->bpos, h->spans_d, h->chunks_d, h->react_partial, (uint32_t)h->nf));
    LAUNCH(KID_REACT_SPANS, k_react_spans<<<blocks_for(nspans, 64), 64, 0, st>>>(h->react_partial, h->chunk_first_d,
                                                                                 h->breact_d, nspans));
  }
}

// Everything of one tick after the span table is in its pinned staging buffer.
void enqueue_tick(vxl_sph_handle* h, float dt_tick, uint32_t nspans) {
  cudaStream_t st = h->stream;
  uint32_t sub = h->substeps;
  float dt = dt_tick / (float)sub;  // fluid_step.rs:77
  if (nspans > 0) {
    cudaMemcpyAsync(h->spans_d, h->spans_h, nspans * sizeof(SpanDev), cudaMemcpyHostToDevice, st);
    if (h->nchunks > 0)
      cudaMemcpyAsync(h->chunks_d, h->chunks_h, h->nchunks * sizeof(SpanChunk), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(h->chunk_first_d, h->chunk_first_h, (nspans + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(h->breact_d, 0, nspans * 6 * sizeof(float), st);
  }
  for (uint32_t s = 0; s < sub; ++s) enqueue_substep(h, dt, nspans);
  if (nspans > 0) {
    if (sub > 1) {
      float inv = 1.0f / (float)sub;  // fluid_step.rs:85
      LAUNCH(KID_SCALE, k_scale<<<blocks_for(nspans * 6), kThreads, 0, st>>>(h->breact_d, nspans * 6, inv));
    }
    cudaMemcpyAsync(h->breact_h, h->breact_d, nspans * 6 * sizeof(float), cudaMemcpyDeviceToHost, st);
  }
  cudaMemcpyAsync(h->ctl_h, h->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st);
}

vxl_status stage_spans(vxl_sph_handle* h, const vxl_sph_span* spans, uint32_t nspans) {
  if (nspans == 0) return VXL_OK;
  if (!spans) return fail(VXL_NULL_POINTER, "spans is NULL with nspans > 0");
  std::vector<SpanDev> next(nspans);
  std::vector<SpanChunk> chunks;
  std::vector<uint32_t> first(nspans + 1, 0);
  for (uint32_t q = 0; q < nspans; ++q) {
    const vxl_sph_span& sp = spans[q];
    if (sp.start < h->nf || sp.end < sp.start || sp.end > h->nt)
      return fail(VXL_INVALID_ARGUMENT, "span " + std::to_string(q) + " is outside the boundary segment");
    next[q] = SpanDev{sp.body, sp.origin[0], sp.origin[1], sp.origin[2], sp.start, sp.end};
    first[q] = (uint32_t)chunks.size();
    for (uint32_t b = sp.start; b < sp.end; b += kReactChunk)
      chunks.push_back(SpanChunk{q, b, std::min(sp.end, b + kReactChunk), 0u});
  }
  first[nspans] = (uint32_t)chunks.size();
  uint32_t nch = (uint32_t)chunks.size();
  if (nspans > h->spans_cap || nch > h->chunks_cap) {
    CU(cudaStreamSynchronize(h->stream));
    if (h->graph) {
      cudaGraphExecDestroy(h->graph);
      h->graph = nullptr;
    }
    void* dptr[] = {h->spans_d, h->breact_d, h->chunks_d, h->chunk_first_d, h->react_partial};
    for (void* q : dptr)
      if (q) cudaFree(q);
    void* hptr[] = {h->spans_h, h->breact_h, h->chunks_h, h->chunk_first_h};
    for (void* q : hptr)
      if (q) cudaFreeHost(q);
    h->spans_d = nullptr; h->spans_h = nullptr; h->breact_d = nullptr; h->breact_h = nullptr;
    h->chunks_d = nullptr; h->chunks_h = nullptr; h->chunk_first_d = nullptr; h->chunk_first_h = nullptr;
    h->react_partial = nullptr;
    uint32_t cap = std::max<uint32_t>(nspans, 64);
    uint32_t ccap = std::max<uint32_t>(nch, cap + (uint32_t)(h->nb / kReactChunk) + 1);
    vxl_status st;
    if ((st = dalloc(h, &h->spans_d, cap)) != VXL_OK) return st;
    if ((st = dalloc(h, &h->breact_d, (size_t)cap * 6)) != VXL_OK) return st;
    if ((st = dalloc(h, &h->chunks_d, ccap)) != VXL_OK) return st;
    if ((st = dalloc(h, &h->chunk_first_d, (size_t)cap + 1)) != VXL_OK) return st;
    if ((st = dalloc(h, &h->react_partial, (size_t)ccap * 6)) != VXL_OK) return st;
    CU(cudaMallocHost((void**)&h->spans_h, cap * sizeof(SpanDev)));
    CU(cudaMallocHost((void**)&h->breact_h, cap * 6 * sizeof(float)));
    CU(cudaMallocHost((void**)&h->chunks_h, ccap * sizeof(SpanChunk)));
    CU(cudaMallocHost((void**)&h->chunk_first_h, (cap + 1) * sizeof(uint32_t)));
    std::memset(h->spans_h, 0xff, cap * sizeof(SpanDev));
    h->spans_cap = cap;
    h->chunks_cap = ccap;
  }
  // The tick graph copies the pinned tables when it runs; an earlier tick may still be
  // queued, so wait for it before changing them (steady state: unchanged, no wait).
  if (std::memcmp(next.data(), h->spans_h, nspans * sizeof(SpanDev)) != 0 || nch != h->nchunks) {
    CU(cudaStreamSynchronize(h->stream));
    std::memcpy(h->spans_h, next.data(), nspans * sizeof(SpanDev));
    if (nch) std::memcpy(h->chunks_h, chunks.data(), nch * sizeof(SpanChunk));
    std::memcpy(h->chunk_first_h, first.data(), (nspans + 1) * sizeof(uint32_t));
    h->nchunks = nch;
  }
  return VXL_OK;
}

vxl_status run_tick(vxl_sph_handle* h, float dt_tick, uint32_t nspans) {
  bool need_capture = !h->graph || h->graph_dt != dt_tick || h->graph_nspans != nspans ||
                      h->graph_record != h->record || h->graph_prof != h->prof || h->graph_nchunks != h->nchunks;
  prof_collect(h);
  h->launches_counter = 0;
  if (!h->use_graph) {
    h->prof_used = 0;
    enqueue_tick(h, dt_tick, nspans);
    h->prof_pending = h->prof;
    h->launches_last_tick = h->launches_counter;
    CU(cudaGetLastError());
    return VXL_OK;
  }
  if (need_capture) {
    if (h->graph) {
      cudaGraphExecDestroy(h->graph);
      h->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    h->prof_used = 0;
    CU(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    h->capturing = true;
    enqueue_tick(h, dt_tick, nspans);
    h->capturing = false;
    CU(cudaStreamEndCapture(h->stream, &g));
    cudaError_t e = cudaGraphInstantiate(&h->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(VXL_CUDA_ERROR, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    h->graph_dt = dt_tick;
    h->graph_nspans = nspans;
    h->graph_record = h->record;
    h->graph_prof = h->prof;
    h->graph_nchunks = h->nchunks;
    h->launches_last_tick = h->launches_counter;
  }
  CU(cudaGraphLaunch(h->graph, h->stream));
  h->prof_pending = h->prof;
  return VXL_OK;
}

vxl_status finish_sync(vxl_sph_handle* h, vxl_sph_reaction* out, uint32_t nspans) {
  CU(cudaStreamSynchronize(h->stream));
  prof_collect(h);
  if (h->ctl_h->err & kErrGridLoop) return fail(VXL_DEVICE_FAULT_FLAG, "grid box doubling loop did not settle");
  if (out && nspans > 0) {
    for (uint32_t q = 0; q < nspans; ++q) {
      out[q].body = h->spans_h[q].body;
      for (int a = 0; a < 3; ++a) {
        out[q].force[a] = h->breact_h[6 * q + a];
        out[q].torque[a] = h->breact_h[6 * q + 3 + a];
      }
    }
  }
  return VXL_OK;
}

vxl_status recompute_bboxes(vxl_sph_handle* h) {
  static const uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
  CU(cudaMemcpyAsync(h->ctl->fbox, init, sizeof(init), cudaMemcpyHostToDevice, h->stream));
  CU(cudaMemcpyAsync(h->ctl->bbox, init, sizeof(init), cudaMemcpyHostToDevice, h->stream));
  uint32_t nblk = blocks_for(h->nt);
  k_bbox<<<nblk, kThreads, 0, h->stream>>>(h->pos[0], (uint32_t)h->nt, 1, h->ctl->fbox);
  k_bbox<<<nblk, kThreads, 0, h->stream>>>(h->pos[0], (uint32_t)h->nt, 0, h->ctl->bbox);
  CU(cudaGetLastError());
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

}  // namespace

extern "C" {

uint32_t vxl_sph_abi_version(void) { return VXL_SPH_ABI_VERSION; }

const char* vxl_sph_last_error(void) { return g_last_error.c_str(); }

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
  API_TRACE();
  try {
    if (!desc || !out) return fail(VXL_NULL_POINTER, "desc or out is NULL");
    *out = nullptr;
    if (desc->hdr.version != VXL_SPH_ABI_VERSION || desc->params.hdr.version != VXL_SPH_ABI_VERSION)
      return fail(VXL_VERSION_MISMATCH, "ABI version mismatch");
    if (!check_header(desc->hdr, sizeof(vxl_sph_desc)) || !check_header(desc->params.hdr, sizeof(vxl_sph_params)))
      return fail(VXL_SIZE_MISMATCH, "struct size mismatch");
    uint64_t nf = desc->n_fluid, nb = desc->n_boundary, nt = nf + nb;
    if (nt > 0 && (!desc->pos_xyz || !desc->vel_xyz)) return fail(VXL_NULL_POINTER, "pos/vel is NULL");
    if (nb > 0 && !desc->pmass) return fail(VXL_NULL_POINTER, "pmass is NULL with boundary particles");
    if (nt >= (1ull << 31)) return fail(VXL_INVALID_ARGUMENT, "more than 2^31 particles");
    const vxl_sph_params& p = desc->params;
    uint32_t max_bins = p.max_bins ? p.max_bins : (1u << 21);
    if (max_bins > (1u << 21)) return fail(VXL_INVALID_ARGUMENT, "max_bins above 2^21");
    if (!(p.particle_mass > 0.0f) || !(p.rest_density > 0.0f) || !(p.gamma_tait > 0.0f))
      return fail(VXL_INVALID_ARGUMENT, "particle_mass, rest_density and gamma_tait must be positive");
    if (desc->pmass)
      for (uint64_t i = 0; i < nf; ++i)
        if (desc->pmass[i] != p.particle_mass)
          return fail(VXL_INVALID_ARGUMENT, "fluid pmass must equal params.particle_mass");
    for (uint64_t i = nf; i < nt; ++i)
      if (!(desc->pmass[i] > 0.0f)) return fail(VXL_INVALID_ARGUMENT, "boundary pmass must be positive");

    auto* h = new (std::nothrow) vxl_sph_handle();
    if (!h) return fail(VXL_OUT_OF_MEMORY, "host allocation failed");
    h->device = desc->device;
    DeviceGuard dg(h->device);
    cudaError_t e = cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking);
    h->stream = h->own_stream;
    if (e != cudaSuccess) {
      delete h;
      return fail(VXL_CUDA_ERROR, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    }
    h->params = p;
    h->nf = nf;
    h->nb = nb;
    h->nt = nt;
    h->max_bins = max_bins;
    h->substeps = p.substeps ? p.substeps : 1;
    h->k = make_const(p, nf, nt, max_bins);
    vxl_status s = VXL_OK;
    auto A = [&](vxl_status r) {
      if (s == VXL_OK) s = r;
    };
    uint64_t nta = nt ? nt : 1;
    A(dalloc(h, &h->pos[0], nta));
    A(dalloc(h, &h->pos[1], nta));
    A(dalloc(h, &h->vel[0], nta));
    A(dalloc(h, &h->vel[1], nta));
    A(dalloc(h, &h->orig, nta));
    A(dalloc(h, &h->slot_of, nta));
    A(dalloc(h, &h->cellrank, nta));
    A(dalloc(h, &h->items, nta));
    A(dalloc(h, &h->counts, (size_t)max_bins + 1));
    A(dalloc(h, &h->start, (size_t)max_bins + 1));
    A(dalloc(h, &h->partial, 1024));
    A(dalloc(h, &h->rc, nta));
    A(dalloc(h, &h->press, nta));
    A(dalloc(h, &h->acc, nta));
    A(dalloc(h, &h->xsph, nta));
    A(dalloc(h, &h->nbr, (size_t)h->nbr_cap * nta));
    A(dalloc(h, &h->nbr_n, nta));
    A(dalloc(h, &h->bforce, nb ? nb : 1));
    A(dalloc(h, &h->bpos, nb ? nb : 1));
    A(dalloc(h, &h->ctl, 1));
    A(dalloc(h, &h->stage, 8 * nta));
    if (s == VXL_OK) {
      if (cudaMallocHost((void**)&h->ctl_h, sizeof(Ctl)) != cudaSuccess) s = fail(VXL_OUT_OF_MEMORY, "pinned alloc");
      else std::memset(h->ctl_h, 0, sizeof(Ctl));
    }
    if (s == VXL_OK) {
      cudaEventCreate(&h->ev0);
      cudaEventCreate(&h->ev1);
      cudaMemsetAsync(h->counts, 0, ((size_t)max_bins + 1) * 4, h->stream);
      cudaMemsetAsync(h->start, 0, ((size_t)max_bins + 1) * 4, h->stream);
      cudaMemsetAsync(h->ctl, 0, sizeof(Ctl), h->stream);
      cudaMemsetAsync(h->acc, 0, nta * sizeof(float4), h->stream);
      cudaMemsetAsync(h->xsph, 0, nta * sizeof(float4), h->stream);
      cudaMemsetAsync(h->bforce, 0, (nb ? nb : 1) * sizeof(float4), h->stream);
      cudaMemsetAsync(h->rc, 0, nta * sizeof(float2), h->stream);
      cudaMemsetAsync(h->press, 0, nta * sizeof(float), h->stream);
      if (nt > 0) {
        cudaMemcpyAsync(h->stage, desc->pos_xyz, nt * 12, cudaMemcpyHostToDevice, h->stream);
        cudaMemcpyAsync(h->stage + 3 * nt, desc->vel_xyz, nt * 12, cudaMemcpyHostToDevice, h->stream);
        float* pm_d = nullptr;
        if (nb > 0) {
          cudaMalloc((void**)&pm_d, nt * 4);
          cudaMemcpyAsync(pm_d, desc->pmass, nt * 4, cudaMemcpyHostToDevice, h->stream);
        }
        k_init_state<<<blocks_for(nt), kThreads, 0, h->stream>>>(h->stage, h->stage + 3 * nt, pm_d, h->pos[0],
                                                                  h->vel[0], h->orig, h->slot_of, h->bpos, h->k);
        s = recompute_bboxes(h);
        cudaStreamSynchronize(h->stream);
        if (pm_d) cudaFree(pm_d);
      }
      cudaError_t e2 = cudaStreamSynchronize(h->stream);
      if (s == VXL_OK && e2 != cudaSuccess) s = fail(VXL_CUDA_ERROR, cudaGetErrorString(e2));
    }
    if (s != VXL_OK) {
      free_all(h);
      delete h;
      return s;
    }
    *out = h;
    return VXL_OK;
  } catch (...) {
    return fail(VXL_PANIC_CAUGHT, "exception in vxl_sph_create");
  }
}

vxl_status vxl_sph_destroy(vxl_sph_handle* h) {
  API_TRACE();
  if (!h) return fail(VXL_NULL_POINTER, "handle is NULL");
  DeviceGuard dg(h->device);
  cudaStreamSynchronize(h->stream);
  free_all(h);
  delete h;
  return VXL_OK;
}

vxl_status vxl_sph_upload_boundary(vxl_sph_handle* h, uint64_t n_fluid, const float* pos_xyz, const float* vel_xyz,
                                   uint64_t nb) {
  API_TRACE();
  if (!h) return fail(VXL_NULL_POINTER, "handle is NULL");
  if (n_fluid != h->nf || nb != h->nb)
    return fail(VXL_SIZE_MISMATCH, "boundary segment length differs from the scene (rebuild the scene)");
  if (nb == 0) return VXL_OK;
  if (!pos_xyz || !vel_xyz) return fail(VXL_NULL_POINTER, "pos/vel is NULL");
  DeviceGuard dg(h->device);
  static const uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
  CU(cudaMemcpyAsync(h->stage, pos_xyz, nb * 12, cudaMemcpyHostToDevice, h->stream));
  CU(cudaMemcpyAsync(h->stage + 3 * nb, vel_xyz, nb * 12, cudaMemcpyHostToDevice, h->stream));
  CU(cudaMemcpyAsync(h->ctl->bbox, init, sizeof(init), cudaMemcpyHostToDevice, h->stream));
  k_upload_boundary<<<blocks_for(nb), kThreads, 0, h->stream>>>(h->stage, h->stage + 3 * nb, h->pos[0], h->vel[0],
                                                                 h->slot_of, h->bpos, h->ctl->bbox, h->k);
  CU(cudaGetLastError());
  // the caller's arrays are borrowed for this call only: finish the copies before returning
  CU(cudaStreamSynchronize(h->stream));
  return VXL_OK;
}

vxl_status vxl_sph_step_tick_async(vxl_sph_handle* h, float dt_tick, const vxl_sph_span* spans, uint32_t nspans) {
  API_TRACE();
  try {
    if (!h) return fail(VXL_NULL_POINTER, "handle is NULL");
    if (!(dt_tick > 0.0f) || !std::isfinite(dt_tick)) return fail(VXL_INVALID_ARGUMENT, "dt_tick must be > 0");
    DeviceGuard dg(h->device);
    if (h->nf == 0) return VXL_OK;  // fluid_step.rs:93-95: boundary particles are not driven alone
    vxl_status s = stage_spans(h, spans, nspans);
    if (s != VXL_OK) return s;
    h->last_nspans = nspans;
    s = run_tick(h, dt_tick, nspans);
    h->ran_substep = true;
    return s;
  } catch (...) {
    return fail(VXL_PANIC_CAUGHT, "exception in vxl_sph_step_tick_async");
  }
}

vxl_status vxl_sph_sync(vxl_sph_handle* h, vxl_sph_reaction* out_reactions, uint32_t nspans) {
  API_TRACE();
  if (!h) return fail(VXL_NULL_POINTER, "handle is NULL");
  DeviceGuard dg(h->device);
  if (nspans > h->last_nspans) return fail(VXL_SIZE_MISMATCH, "more reactions requested than spans stepped");
  return finish_sync(h, out_reactions, nspans);
}

vxl_status vxl_sph_step_tick(vxl_sph_handle* h, float dt_tick, const vxl_sph_span* spans, uint32_t nspans,
                             vxl_sph_reaction* out_reactions) {
  API_TRACE();
  if (nspans > 0 && !out_reactions) return fail(VXL_NULL_POINTER, "out_reactions is NULL with nspans > 0");
  vxl_status s = vxl_sph_step_tick_async(h, dt_tick, spans, nspans);
  if (s != VXL_OK) return s;
  return vxl_sph_sync(h, out_reactions, nspans);
}

vxl_status vxl_sph_substep(vxl_sph_handle* h, float dt) {
  API_TRACE();
  if (!h) return fail(VXL_NULL_POINTER, "handle is NULL");
  if (!(dt > 0.0f)) return fail(VXL_INVALID_ARGUMENT, "dt must be > 0");
  DeviceGuard dg(h->device);
  if (h->nf == 0) return VXL_OK;
  prof_collect(h);
  h->prof_used = 0;
  enqueue_substep(h, dt, 0);
  h->prof_pending = h->prof;
  CU(cudaMemcpyAsync(h->ctl_h, h->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, h->stream));
  CU(cudaGetLastError());
  h->ran_substep = true;
  return finish_sync(h, nullptr, 0);
}

vxl_status vxl_sph_bounds(vxl_sph_handle* h, float lo[3], float hi[3]) {
  API_TRACE();
  if (!h || !lo || !hi) return fail(VXL_NULL_POINTER, "NULL argument");
  DeviceGuard dg(h->device);
  uint32_t box[6];
  CU(cudaMemcpyAsync(box, h->ctl->fbox, sizeof(box), cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  for (int a = 0; a < 3; ++a) {
    lo[a] = vxl_o2f_host(box[a]);
    hi[a] = vxl_o2f_host(box[3 + a]);
  }
  if (!(std::isfinite(lo[0]) && std::isfinite(hi[0]))) return fail(VXL_NOT_READY, "no fluid bounds");
  return VXL_OK;
}

vxl_status vxl_sph_read_state(vxl_sph_handle* h, float* pos_xyz, float* vel_xyz) {
  API_TRACE();
  if (!h) return fail(VXL_NULL_POINTER, "handle is NULL");
  DeviceGuard dg(h->device);
  if (h->nt == 0) return VXL_OK;
  float* dp = h->stage;
  float* dv = h->stage + 3 * h->nt;
  k_read_state<<<blocks_for(h->nt), kThreads, 0, h->stream>>>(h->pos[0], h->vel[0], h->orig, pos_xyz ? dp : nullptr,
                                                               vel_xyz ? dv : nullptr, (uint32_t)h->nt);
  if (pos_xyz) CU(cudaMemcpyAsync(pos_xyz, dp, h->nt * 12, cudaMemcpyDeviceToHost, h->stream));
  if (vel_xyz) CU(cudaMemcpyAsync(vel_xyz, dv, h->nt * 12, cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  return VXL_OK;
}

vxl_status vxl_sph_write_state(vxl_sph_handle* h, const float* pos_xyz, const float* vel_xyz) {
  API_TRACE();
  if (!h) return fail(VXL_NULL_POINTER, "handle is NULL");
  DeviceGuard dg(h->device);
  if (h->nt == 0) return VXL_OK;
  float* dp = h->stage;
  float* dv = h->stage + 3 * h->nt;
  if (pos_xyz) CU(cudaMemcpyAsync(dp, pos_xyz, h->nt * 12, cudaMemcpyHostToDevice, h->stream));
  if (vel_xyz) CU(cudaMemcpyAsync(dv, vel_xyz, h->nt * 12, cudaMemcpyHostToDevice, h->stream));
  k_write_state<<<blocks_for(h->nt), kThreads, 0, h->stream>>>(pos_xyz ? dp : nullptr, vel_xyz ? dv : nullptr,
                                                                h->pos[0], h->vel[0], h->orig, h->bpos, h->k);
  if (pos_xyz) {
    vxl_status s = recompute_bboxes(h);
    if (s != VXL_OK) return s;
  }
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(h->stream));  // the caller's arrays are borrowed for this call only
  return VXL_OK;
}

vxl_status vxl_sph_set_record(vxl_sph_handle* h, int on) {
  API_TRACE();
  if (!h) return fail(VXL_NULL_POINTER, "handle is NULL");
  h->record = on != 0;
  return VXL_OK;
}

vxl_status vxl_sph_read_fields(vxl_sph_handle* h, float* dens, float* press, float* acc_xyz, float* xsph_xyz,
                               float* bforce_xyz) {
  API_TRACE();
  if (!h) return fail(VXL_NULL_POINTER, "handle is NULL");
  DeviceGuard dg(h->device);
  uint64_t nt = h->nt;
  if (nt == 0) return VXL_OK;
  if ((acc_xyz || xsph_xyz) && !h->record) return fail(VXL_NOT_READY, "acc/xsph are recorded only with set_record(1)");
  float* d_d = h->stage;
  float* d_p = h->stage + nt;
  float* d_a = h->stage + 2 * nt;
  float* d_x = h->stage + 5 * nt;
  k_read_fields<<<blocks_for(nt), kThreads, 0, h->stream>>>(h->rc, h->press, h->acc, h->xsph, h->orig,
                                                             dens ? d_d : nullptr, press ? d_p : nullptr,
                                                             acc_xyz ? d_a : nullptr, xsph_xyz ? d_x : nullptr,
                                                             (uint32_t)nt);
  if (dens) CU(cudaMemcpyAsync(dens, d_d, nt * 4, cudaMemcpyDeviceToHost, h->stream));
  if (press) CU(cudaMemcpyAsync(press, d_p, nt * 4, cudaMemcpyDeviceToHost, h->stream));
  if (acc_xyz) CU(cudaMemcpyAsync(acc_xyz, d_a, nt * 12, cudaMemcpyDeviceToHost, h->stream));
  if (xsph_xyz) CU(cudaMemcpyAsync(xsph_xyz, d_x, nt * 12, cudaMemcpyDeviceToHost, h->stream));
  if (bforce_xyz && h->nb > 0) {
    std::vector<float> tmp(h->nb * 4);
    CU(cudaMemcpyAsync(tmp.data(), h->bforce, h->nb * 16, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    for (uint64_t q = 0; q < h->nb; ++q)
      for (int a = 0; a < 3; ++a) bforce_xyz[3 * q + a] = tmp[4 * q + a];
  }
  CU(cudaStreamSynchronize(h->stream));
  return VXL_OK;
}

vxl_status vxl_sph_export_grid(vxl_sph_handle* h, uint32_t* items, uint32_t* start, uint64_t start_cap,
                               uint32_t* bins, vxl_sph_grid_info* info) {
  API_TRACE();
  if (!h) return fail(VXL_NULL_POINTER, "handle is NULL");
  DeviceGuard dg(h->device);
  if (!h->ran_substep) return fail(VXL_NOT_READY, "no substep has run yet");
  Ctl c;
  CU(cudaMemcpyAsync(&c, h->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  uint64_t total = c.grid.total;
  if (info) {
    if (!check_header(info->hdr, sizeof(vxl_sph_grid_info))) return fail(VXL_SIZE_MISMATCH, "grid_info header");
    info->min[0] = c.grid.minx; info->min[1] = c.grid.miny; info->min[2] = c.grid.minz;
    info->inv = c.grid.inv;
    info->bin = c.grid.bin;
    info->dims[0] = c.grid.nx; info->dims[1] = c.grid.ny; info->dims[2] = c.grid.nz;
    info->total = total;
  }
  if (start) {
    if (start_cap < total + 1) return fail(VXL_SIZE_MISMATCH, "start buffer smaller than cells + 1");
    CU(cudaMemcpyAsync(start, h->start, (total + 1) * 4, cudaMemcpyDeviceToHost, h->stream));
  }
  if (items) CU(cudaMemcpyAsync(items, h->orig, h->nt * 4, cudaMemcpyDeviceToHost, h->stream));
  if (bins) {
    uint32_t* d_bins = (uint32_t*)h->stage;
    k_export_bins<<<blocks_for(total), kThreads, 0, h->stream>>>(h->start, h->orig, h->ctl, d_bins);
    CU(cudaMemcpyAsync(bins, d_bins, h->nt * 4, cudaMemcpyDeviceToHost, h->stream));
  }
  CU(cudaStreamSynchronize(h->stream));
  return VXL_OK;
}

vxl_status vxl_sph_set_stream(vxl_sph_handle* h, void* cuda_stream) {
  API_TRACE();
  if (!h) return fail(VXL_NULL_POINTER, "handle is NULL");
  DeviceGuard dg(h->device);
  prof_collect(h);
  CU(cudaStreamSynchronize(h->stream));
  h->stream = cuda_stream ? (cudaStream_t)cuda_stream : h->own_stream;
  return VXL_OK;
}

vxl_status vxl_sph_set_profile(vxl_sph_handle* h, int on) {
  API_TRACE();
  if (!h) return fail(VXL_NULL_POINTER, "handle is NULL");
  DeviceGuard dg(h->device);
  prof_collect(h);
  h->prof = on != 0;
  // events for every launch of a tick, created here (never during graph capture)
  size_t need = 2 * ((size_t)h->substeps * 12 + 8);
  while (h->prof && h->prof_ev.size() < need) {
    cudaEvent_t e;
    CU(cudaEventCreate(&e));
    h->prof_ev.push_back(e);
  }
  h->prof_kid.resize(h->prof_ev.size() / 2);
  for (int k = 0; k < KID_COUNT; ++k) {
    h->prof_ms[k] = 0.0;
    h->prof_n[k] = 0;
  }
  return VXL_OK;
}

vxl_status vxl_sph_profile_read(vxl_sph_handle* h, uint32_t k, const char** name, double* total_ms,
                                uint64_t* launches) {
  API_TRACE();
  if (!h) return fail(VXL_NULL_POINTER, "handle is NULL");
  if (k >= (uint32_t)KID_COUNT) return fail(VXL_INVALID_ARGUMENT, "kernel index past the table");
  DeviceGuard dg(h->device);
  prof_collect(h);
  if (name) *name = kKernelNames[k];
  if (total_ms) *total_ms = h->prof_ms[k];
  if (launches) *launches = h->prof_n[k];
  return VXL_OK;
}

vxl_status vxl_sph_get_stats(vxl_sph_handle* h, vxl_sph_stats* out) {
  API_TRACE();
  if (!h || !out) return fail(VXL_NULL_POINTER, "NULL argument");
  if (!check_header(out->hdr, sizeof(vxl_sph_stats))) return fail(VXL_SIZE_MISMATCH, "stats header");
  DeviceGuard dg(h->device);
  Ctl c;
  CU(cudaMemcpyAsync(&c, h->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  out->n_fluid = h->nf;
  out->n_boundary = h->nb;
  out->cells = c.grid.total;
  out->launches_last_tick = h->launches_last_tick;
  out->device_bytes = h->device_bytes;
  out->last_tick_ms = 0.0f;
  return VXL_OK;
}

}  // extern "C"
