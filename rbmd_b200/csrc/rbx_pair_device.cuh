// rbx_pair_device.cuh -- device helpers shared by the pair-force and the
// adjoint kernels: warp sums and the exact FP64 RBL pair classification.
#pragma once
#include "rbx_common.cuh"
#include "rbx_kernels.h"

namespace rbx {

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

struct Classified {
  bool core_active;    // core list and lj126_rs window (r^2 > EPS)
  bool shell_window;   // shell list and rcs window (r_core^2 < r^2 < cut_off^2)
};

__device__ __forceinline__ Classified classify_exact(double d2, const PairParams& pp) {
  Classified c;
  const bool A = d2 < pp.core2_list;
  c.core_active = A && d2 > RBX_EPSILON;  // d2 < rs2 holds: core2_list < rs2
  c.shell_window = !A && d2 < pp.force2_list && d2 > pp.rs2;  // force2_list < rc2
  return c;
}

__device__ __forceinline__ double exact_d2(const PairParams& pp, const double* __restrict__ x,
                                           const double* __restrict__ y,
                                           const double* __restrict__ z, int i, int j) {
  return dist2_list(pp.box, __ldg(x + i), __ldg(y + i), __ldg(z + i), __ldg(x + j),
                    __ldg(y + j), __ldg(z + j));
}

}  // namespace rbx
