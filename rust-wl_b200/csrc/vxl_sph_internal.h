// Host helpers shared by the library's translation units.
#pragma once

#include <cstdint>
#include <cstring>

// Rust `f32::powi` (LLVM ExpandPowI / compiler-rt __powisf2): square-and-multiply,
// multiplying the running result by the current square for each set exponent bit.
inline float vxl_powi(float a, int b) {
  bool recip = b < 0;
  float r = 1.0f;
  for (;;) {
    if (b & 1) r *= a;
    b /= 2;
    if (b == 0) break;
    a *= a;
  }
  return recip ? 1.0f / r : r;
}

// Inverse of the device's ordered-uint float code.
inline float vxl_o2f_host(uint32_t o) {
  uint32_t u = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

// The thread-local message returned by vxl_sph_last_error() (defined in sph_engine.cu).
void vxl_set_last_error(const char* msg);
const char* vxl_get_last_error();
