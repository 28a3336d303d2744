// ref_morton_shim.cpp - the reference's host-callable Morton code
// (morton.h:11-28) exported for golden vectors, compiled without fast-math
// into oracle/_ref/libref_morton.so.  TEST INFRASTRUCTURE ONLY.
#include <cstdint>

#include "morton.h"

extern "C" {

void ref_morton_codes(const float* xyz, int64_t n, float lo, float hi, uint64_t* out) {
    for (int64_t i = 0; i < n; ++i) out[i] = get_morton_code(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], lo, hi);
}

uint64_t ref_expand_bits(uint32_t v) { return expand_bits(v); }

}  // extern "C"
