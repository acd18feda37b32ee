// ORACLE -- test infrastructure only.
//
// The two pieces of the reference's matvec path that compile from their own
// source files with nothing but the C++ standard library, built from the
// reference tree itself (the headers are included by path at build time,
// see the `ref` target of oracle/Makefile; nothing is copied):
//   ribesl  -- Cody's modified Bessel function I_{n+alpha}(x), as vendored
//              by the reference (src/fmm/bessel_gamma.h:269); the reference
//              builds its scaled i_n from it (src/fmm/fmm_math_funcs.h:24-113)
//   interactions -- the stored 1512-entry interaction-list table
//              (src/fmm/interaction_list.h:93-1607)
// The rest of the path (fmm.h, fmm_globals.h, octree.h, node_patch.h) needs
// LTL, Boost and Charm++ headers that are not installed, so it is not built.
#include <bessel_gamma.h>
#include <interaction_list.h>

#include <cstdint>

extern "C" {

int ref_ribesl(double x, double alpha, int nb, int ize, double* b) { return ribesl(x, alpha, nb, ize, b); }

// 7 ints per entry: neighbour, direction, target child, source child, dx, dy,
// dz, in the table's order; returns the entry count
int ref_interaction_list(int32_t* out) {
  for (int k = 0; k < ILIST_SIZE; ++k) {
    const INTERACTION& e = interactions[k];
    const int32_t v[7] = {e.neighbour, (int32_t)e.dir, e.targ, e.src, e.dx, e.dy, e.dz};
    if (out)
      for (int c = 0; c < 7; ++c) out[7 * k + c] = v[c];
  }
  return ILIST_SIZE;
}
}
