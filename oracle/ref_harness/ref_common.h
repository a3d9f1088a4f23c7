/* Helpers shared by the reference-kernel harness translation units. */
#pragma once
#include "model/box.h"

static inline Box ref_make_box(const double* lo, const double* hi) {
  Box b;
  b._type = Box::BoxType::ORTHOGONAL;
  b._pbc_x = b._pbc_y = b._pbc_z = true;
  for (int d = 0; d < 3; ++d) {
    b._coord_min[d] = (rbmd::Real)lo[d];
    b._coord_max[d] = (rbmd::Real)hi[d];
    b._length[d] = (rbmd::Real)(hi[d] - lo[d]);
    b._length_inv[d] = (rbmd::Real)(1.0 / (hi[d] - lo[d]));
  }
  return b;
}

static inline int ref_sync() {
  const cudaError_t e = cudaDeviceSynchronize();
  return e == cudaSuccess ? 0 : (int)e;
}
