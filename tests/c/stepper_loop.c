/* A C caller of the library, as a non-Python host (a Rust shim through FFI, a C++ engine)
 * drives it: the FluidStepper::step call pattern — upload the boundary segment, step one
 * tick with the spans, collect the reactions — for a number of ticks, then read the state.
 * Input file: u64 n_fluid, n_boundary, nspans, ticks; f32 dt_tick; vxl_sph_params;
 * f32 pos[3n], vel[3n], pmass[n]; vxl_sph_span[nspans]. Output file: f32 pos[3n], vel[3n],
 * vxl_sph_reaction[nspans] of the last tick. Used by tests/test_gpu_c_caller.py. */
#include <stdio.h>
#include <stdlib.h>

#include "vxl_sph.h"

static void* read_n(FILE* f, size_t n) {
  void* p = malloc(n ? n : 1);
  if (!p || (n && fread(p, 1, n, f) != n)) {
    fprintf(stderr, "input file too short\n");
    exit(2);
  }
  return p;
}

static int check(vxl_status s, const char* what) {
  if (s != VXL_OK) {
    fprintf(stderr, "%s failed (%d): %s\n", what, (int)s, vxl_sph_last_error());
    return 1;
  }
  return 0;
}

int main(int argc, char** argv) {
  if (argc != 3) {
    fprintf(stderr, "usage: %s input output\n", argv[0]);
    return 2;
  }
  FILE* in = fopen(argv[1], "rb");
  if (!in) return 2;
  uint64_t* hdr = (uint64_t*)read_n(in, 4 * sizeof(uint64_t));
  const uint64_t nf = hdr[0], nb = hdr[1], nspans = hdr[2], ticks = hdr[3], n = nf + nb;
  float* dt = (float*)read_n(in, sizeof(float));
  vxl_sph_params* prm = (vxl_sph_params*)read_n(in, sizeof(vxl_sph_params));
  float* pos = (float*)read_n(in, 3 * n * sizeof(float));
  float* vel = (float*)read_n(in, 3 * n * sizeof(float));
  float* pmass = (float*)read_n(in, n * sizeof(float));
  vxl_sph_span* spans = (vxl_sph_span*)read_n(in, nspans * sizeof(vxl_sph_span));
  fclose(in);

  vxl_sph_desc d;
  d.hdr.size = sizeof(vxl_sph_desc);
  d.hdr.version = VXL_SPH_ABI_VERSION;
  d.params = *prm;
  d.n_fluid = nf;
  d.n_boundary = nb;
  d.pos_xyz = pos;
  d.vel_xyz = vel;
  d.pmass = pmass;
  d.device = 0;
  vxl_sph_handle* h = NULL;
  if (check(vxl_sph_create(&d, &h), "vxl_sph_create")) return 3;
  vxl_sph_reaction* react = (vxl_sph_reaction*)malloc((nspans ? nspans : 1) * sizeof(vxl_sph_reaction));
  for (uint64_t t = 0; t < ticks; ++t) {
    if (check(vxl_sph_upload_boundary(h, nf, pos + 3 * nf, vel + 3 * nf, nb), "vxl_sph_upload_boundary")) return 3;
    if (check(vxl_sph_step_tick(h, *dt, spans, (uint32_t)nspans, react), "vxl_sph_step_tick")) return 3;
  }
  float* out_pos = (float*)malloc(3 * n * sizeof(float));
  float* out_vel = (float*)malloc(3 * n * sizeof(float));
  if (check(vxl_sph_read_state(h, out_pos, out_vel), "vxl_sph_read_state")) return 3;
  if (check(vxl_sph_destroy(h), "vxl_sph_destroy")) return 3;
  FILE* out = fopen(argv[2], "wb");
  if (!out) return 2;
  fwrite(out_pos, sizeof(float), 3 * n, out);
  fwrite(out_vel, sizeof(float), 3 * n, out);
  fwrite(react, sizeof(vxl_sph_reaction), nspans, out);
  fclose(out);
  return 0;
}
