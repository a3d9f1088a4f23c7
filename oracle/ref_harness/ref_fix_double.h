/* Forced-include header for the FP64 build of the reference kernels.
 * RBMD's rbmd_define.h declares double7::operator[] returning float& bound to
 * a double member, so USE_DOUBLE=1 does not compile.  With the system headers
 * it pulls in already included, the header is read once with `float` spelled
 * `double`; in its USE_DOUBLE branch that touches only those two accessors. */
#pragma once
#include <cuda_runtime.h>
#include <cuda_runtime_api.h>
#include <cmath>
#include <cub/cub.cuh>
#include <thrust/copy.h>
#include <thrust/device_vector.h>
#include <thrust/gather.h>
#include <thrust/reduce.h>
#include <thrust/sort.h>
#define float double
#include "common/rbmd_define.h"
#undef float
/* The RBSOG kernels declare locals named like the math functions they call
 * (`rbmd::Real exp = EXP(mid);`), which only compiles while EXP is expf; with
 * the math macros naming the global functions explicitly it compiles as FP64. */
#undef EXP
#define EXP ::exp
#undef COS
#define COS ::cos
#undef SIN
#define SIN ::sin
#undef SQRT
#define SQRT ::sqrt
#undef POW
#define POW ::pow
#undef ERF
#define ERF ::erf
#undef ERFC
#define ERFC ::erfc
#undef LOG
#define LOG ::log
