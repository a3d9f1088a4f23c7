// rbx_common.cuh -- device helpers shared by the sm_100a kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "rbx.h"

#define RBX_PI 3.14159265358979323846
#define RBX_EPSILON 0.0001  // EPSILON under USE_DOUBLE, src/common/rbmd_define.h:46-50

namespace rbx {

// Orthogonal periodic box in the form the kernels want.
struct DBox {
  double lo[3];
  double len[3];
  double half[3];  // 0.5 * len, exactly as box._length[d] * 0.5
};

inline DBox make_dbox(const rbx_box& b) {
  DBox d;
  for (int i = 0; i < 3; ++i) {
    d.lo[i] = b.lo[i];
    d.len[i] = b.hi[i] - b.lo[i];
    d.half[i] = d.len[i] * 0.5;
  }
  return d;
}

// MinImageDistance, single shift (src/data_manager/include/model/box.h:51-73).
__device__ __forceinline__ double min_image1(double d, double len, double half) {
  if (fabs(d) > half) d -= (d > 0 ? len : -len);
  return d;
}

// Fixed-point coordinate of the mixed form: floor((v - lo) * 2^32 / L).
__device__ __forceinline__ unsigned to_fixed(double v, double lo, double scale) {
  return (unsigned)(unsigned long long)__double2ll_rd((v - lo) * scale);
}

// Warp maximum of a non-negative double, then one atomicMax on its bits.
// Every lane of the warp must call it.
__device__ __forceinline__ void warp_max_atomic(double d2, unsigned long long* out) {
  unsigned long long bits = (unsigned long long)__double_as_longlong(d2);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long t = __shfl_xor_sync(0xffffffffu, bits, o);
    bits = t > bits ? t : bits;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(out, bits);
}

// CaculateDistance (src/neighbor_list/src/op/full_neighbor_list_op.h:98-106):
// i minus j, min image, squares summed left to right with no fused
// multiply-add, so list membership rounds like the reference.
__device__ __forceinline__ double dist2_list(const DBox& b, double xi, double yi,
                                             double zi, double xj, double yj,
                                             double zj) {
  const double dx = min_image1(__dsub_rn(xi, xj), b.len[0], b.half[0]);
  const double dy = min_image1(__dsub_rn(yi, yj), b.len[1], b.half[1]);
  const double dz = min_image1(__dsub_rn(zi, zj), b.len[2], b.half[2]);
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// MixRblSampleKey (rbl_full_neighbor_list_op.hip.cu:6-11).
__host__ __device__ __forceinline__ unsigned long long rbl_mix(unsigned long long v) {
  v += 0x9e3779b97f4a7c15ULL;
  v = (v ^ (v >> 30)) * 0xbf58476d1ce4e5b9ULL;
  v = (v ^ (v >> 27)) * 0x94d049bb133111ebULL;
  return v ^ (v >> 31);
}

// Low word of the 64-bit value (hi, lo) shifted right by s (0 < s < 32).
__host__ __device__ __forceinline__ unsigned funnel_r(unsigned lo, unsigned hi, unsigned s) {
#ifdef __CUDA_ARCH__
  return __funnelshift_r(lo, hi, s);
#else
  return (unsigned)((((unsigned long long)hi << 32) | lo) >> s);
#endif
}

// Batch test mix(key) % freq == 0 for freq in {1, 2, 4} (mask = freq - 1).
// With w = v ^ (v >> 27) after the second round and u = w * C2, the test reads
// bits 0 and 1 of h = u ^ (u >> 31): h_0 = u_0 ^ u_31 and h_1 = u_1 ^ u_32.
// u mod 2^33 needs only the 32x32->64 product p of the low halves of w and C2
// and the parity of w_hi * C2_lo + w_lo * C2_hi, which is w_32 ^ w_0 because
// both halves of C2 are odd: u_32 = p_32 ^ w_32 ^ w_0.  The funnel shift of p
// by 31 lines p_31 and p_32 up with bits 0 and 1.
__host__ __device__ __forceinline__ bool rbl_selected_low2(unsigned long long key,
                                                           unsigned mask) {
  unsigned long long v = key + 0x9e3779b97f4a7c15ULL;
  v = (v ^ (v >> 30)) * 0xbf58476d1ce4e5b9ULL;
  const unsigned lo = (unsigned)v, hi = (unsigned)(v >> 32);
  const unsigned w_lo = lo ^ funnel_r(lo, hi, 27);  // low half of w
  const unsigned t = hi ^ (hi >> 27) ^ w_lo;        // bit 0: w_32 ^ w_0
  const unsigned long long p = (unsigned long long)w_lo * 0x133111ebu;
  const unsigned p_lo = (unsigned)p;
  const unsigned f = funnel_r(p_lo, (unsigned)(p >> 32), 31);  // bit 0: p_31, bit 1: p_32
  return ((p_lo ^ f ^ (t << 1)) & mask) == 0u;
}

// Per-atom halves of the RBL pair key: A_i = mix(gid_i), B_j = mix(gid_j + C).
__host__ __device__ __forceinline__ unsigned long long rbl_key_a(int gid) {
  return rbl_mix((unsigned long long)(long long)gid);
}
__host__ __device__ __forceinline__ unsigned long long rbl_key_b(int gid) {
  return rbl_mix((unsigned long long)(long long)gid + 0xd1b54a32d192ed03ULL);
}

// Divisibility test x % d == 0 for a runtime d >= 1 without a 64-bit divide
// (Granlund & Montgomery, "Division by invariant integers using
// multiplication", PLDI'94, sec. 9): d = d_odd * 2^k, x % d == 0 iff
// rotr(x * inv(d_odd), k) <= floor((2^64 - 1) / d).
struct DivTest {
  unsigned long long inv;    // multiplicative inverse of d_odd mod 2^64
  unsigned long long limit;  // floor((2^64-1)/d)
  int shift;                 // k
  int trivial;               // d <= 1
};

inline DivTest make_divtest(int d) {
  DivTest t;
  t.trivial = d <= 1;
  if (t.trivial) {
    t.inv = 1;
    t.limit = ~0ULL;
    t.shift = 0;
    return t;
  }
  unsigned long long dd = (unsigned long long)d;
  int k = 0;
  while ((dd & 1ULL) == 0) {
    dd >>= 1;
    ++k;
  }
  unsigned long long inv = dd;  // Newton iteration for the 2-adic inverse
  for (int i = 0; i < 6; ++i) inv *= 2ULL - dd * inv;
  t.inv = inv;
  t.shift = k;
  t.limit = ~0ULL / (unsigned long long)d;
  return t;
}

__host__ __device__ __forceinline__ bool divisible(unsigned long long x, const DivTest& t) {
  if (t.trivial) return true;
  unsigned long long y = x * t.inv;
  if (t.shift) y = (y >> t.shift) | (y << (64 - t.shift));
  return y <= t.limit;
}

// RblShellSampleSelected (rbl_full_neighbor_list_op.hip.cu:13-30) with the
// per-atom mixes precomputed: key = epoch ^ A_i ^ B_j, keep iff mix(key) % freq == 0.
__device__ __forceinline__ bool rbl_selected(unsigned long long epoch_xor_ai,
                                             unsigned long long bj,
                                             const DivTest& t) {
  if (t.trivial) return true;
  return divisible(rbl_mix(epoch_xor_ai ^ bj), t);
}

// Philox4x32-10 (Salmon et al., SC'11).
__host__ __device__ inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
    c[1] = (uint32_t)p1;
    c[3] = (uint32_t)p0;
    c[0] = n0;
    c[2] = n2;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// Block-wide deterministic sum of doubles (fixed tree).  All threads of the
// block must call it; returns the total on every thread.
template <int BLOCK>
__device__ __forceinline__ double block_sum_det(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double t = 0.0;
  if (w == 0) {
    t = (lane < BLOCK / 32) ? sh[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0) sh[0] = t;
  }
  __syncthreads();
  t = sh[0];
  __syncthreads();
  return t;
}

}  // namespace rbx

// Launch bookkeeping and error plumbing (rbx_capi.cu).
namespace rbx {
void set_error(const char* fmt, ...);
void count_launch(int n = 1);
int check_launch(const char* what);
int grid_for(long long work, int per_block, int max_blocks = 1 << 30);
int sm_count();
}  // namespace rbx
