// rbx_capi_util.h -- argument checks and scratch allocation shared by the
// C-ABI translation units (internal).
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "rbx.h"
#include "rbx_common.cuh"

namespace rbx {
// Orthogonal box with positive, finite edges.
inline bool valid_box(const rbx_box* b) {
  if (!b) return false;
  for (int d = 0; d < 3; ++d)
    if (!(b->hi[d] - b->lo[d] > 0.0) || !isfinite(b->hi[d] - b->lo[d])) return false;
  return true;
}
// The library runs only on sm_100-class devices; there is no CPU path.
int require_device();
}  // namespace rbx

#define RBX_CHECK_BOX(b)                           \
  do {                                             \
    if (!rbx::valid_box(b)) {                      \
      rbx::set_error("invalid box (hi must exceed lo)"); \
      return RBX_ERR_INVALID;                      \
    }                                              \
  } while (0)

#define RBX_TRY(expr)       \
  do {                      \
    const int _rc = (expr); \
    if (_rc) return _rc;    \
  } while (0)

template <typename T>
inline int async_alloc(T** p, size_t count, cudaStream_t st) {
  if (count == 0) count = 1;
  if (cudaMallocAsync((void**)p, sizeof(T) * count, st) != cudaSuccess) {
    cudaGetLastError();
    rbx::set_error("cudaMallocAsync of %zu bytes failed", sizeof(T) * count);
    return RBX_ERR_NOMEM;
  }
  return RBX_OK;
}

