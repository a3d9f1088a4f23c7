// rbx_rbe.cu -- Random Batch Ewald k-space kernels for sm_100a.
//
// Work per step is 2 * N * P (atom, k) phase evaluations: one pass builds the
// structure factors rho(k_p) = sum_j q_j exp(i k_p . r_j), one pass scatters
// F_i = q_i sum_p c_p (cos(k_p.r_i) Im rho_p - sin(k_p.r_i) Re rho_p) k_p
// (src/force/src/kspace_calculator_op/rocm/kspace_calculator_op.hip.cu:98-125,
// 238-289, 678-738).  Both passes are SFU/issue bound, not HBM bound: the
// 16-32 B/atom inputs stay in L2.
//
// Plain form: FP64 positions, FP64 sincos.
// Mixed form: 32-bit fixed-point fractional coordinates u = frac((x-lo)/L)*2^32
// so the phase m.u mod 2^32 is exact integer arithmetic; the angle goes to the
// SFU (__sincosf) in FP32; per-thread FP32 partial sums are folded with a
// TwoSum-compensated pair; the cross-block reduction, energy and virial are FP64.
#include <math.h>

#include "rbx_common.cuh"
#include "rbx_kernels.h"

namespace rbx {

// ---------------------------------------------------------------------------
// rho(k) partial sums: block (bx, by) covers atom chunk bx and k-group by.
// A thread owns KPT k-vectors {kg*32*KPT + lane + 32*t} (KPT a template
// parameter, default 4); warps of the block take disjoint atom sub-ranges; the
// block combines its warps in fixed order and writes one partial per k.  No
// atomics: the result is deterministic.
// ---------------------------------------------------------------------------
constexpr int RBE_BLOCK = 256;
constexpr int RBE_WARPS = RBE_BLOCK / 32;

__device__ __forceinline__ int table_pick(const double* cdf, int cnt, double total, uint64_t u53) {
  const double target = (double)u53 * (1.0 / 9007199254740992.0) * total;
  int lo = 0, hi = cnt - 1;  // first index with target < cdf[idx], else cnt - 1
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (target < cdf[mid])
      hi = mid;
    else
      lo = mid + 1;
  }
  const int idx = lo;
  if (idx == 0) return 0;
  return (idx & 1) ? (idx + 1) / 2 : -(idx / 2);
}

// One RBE k-sample s of MD step `step` (RBESampleMH's density, drawn exactly
// per axis): Philox4x32-10 of counter {s, attempt, step} under key (k0, k1),
// the three inverse-CDF picks, |m| = 0 redrawn (at most 64 attempts).  false
// when every attempt gave m = 0.
__device__ __forceinline__ bool rbe_draw(int s, const SampleArgs& sa, const double* w0,
                                         uint64_t step, int m[3]) {
  const double* w1 = w0 + sa.c0;
  const double* w2 = w1 + sa.c1;
  for (int a = 0; a < 64; ++a) {
    uint32_t c[4] = {(uint32_t)s, (uint32_t)(2 * a), (uint32_t)step, (uint32_t)(step >> 32)};
    philox4x32_10(c, sa.key0, sa.key1);
    uint32_t d[4] = {(uint32_t)s, (uint32_t)(2 * a + 1), (uint32_t)step, (uint32_t)(step >> 32)};
    philox4x32_10(d, sa.key0, sa.key1);
    m[0] = table_pick(w0, sa.c0, sa.t0, ((((uint64_t)c[0]) << 32) | c[1]) >> 11);
    m[1] = table_pick(w1, sa.c1, sa.t1, ((((uint64_t)c[2]) << 32) | c[3]) >> 11);
    m[2] = table_pick(w2, sa.c2, sa.t2, ((((uint64_t)d[0]) << 32) | d[1]) >> 11);
    if (m[0] != 0 || m[1] != 0 || m[2] != 0) return true;
  }
  return false;
}

// With sa.tables the k-vectors of the block's k-group are drawn here (one
// per thread, into shared memory) instead of read, from the cumulative tables
// staged in shared memory when they fit: block column 0 also writes them out
// (double and integer copies) and raises sa.status on a failed draw.
constexpr int SAMPLE_TAB_SMEM = 768;  // table entries staged in shared memory

template <int KPT>
__device__ __forceinline__ void rbe_group_samples(const SampleArgs& sa, int p, int kbase,
                                                  int (*s_m)[32 * KPT], bool col0) {
  __shared__ double s_cdf[SAMPLE_TAB_SMEM];
  const int ent = sa.c0 + sa.c1 + sa.c2;
  const bool staged = ent <= SAMPLE_TAB_SMEM;
  if (staged)
    for (int e = threadIdx.x; e < ent; e += blockDim.x) s_cdf[e] = sa.tables[e];
  __syncthreads();
  const double* w0 = staged ? s_cdf : sa.tables;
  const uint64_t step = sa.step_dev ? (uint64_t)(int64_t)*sa.step_dev : sa.step_arg;
  for (int slot = threadIdx.x; slot < 32 * KPT; slot += blockDim.x) {
    const int k = kbase + slot;
    int m[3] = {0, 0, 0};
    if (k < p) {
      const bool ok = rbe_draw(k, sa, w0, step, m);
      if (col0) {
        if (!ok) atomicOr(sa.status, 1);
        sa.mx[k] = m[0];
        sa.my[k] = m[1];
        sa.mz[k] = m[2];
        if (sa.mi) {
          sa.mi[3 * k] = m[0];
          sa.mi[3 * k + 1] = m[1];
          sa.mi[3 * k + 2] = m[2];
        }
      }
    }
    s_m[0][slot] = m[0];
    s_m[1][slot] = m[1];
    s_m[2][slot] = m[2];
  }
  __syncthreads();
}

template <int KPT>
__global__ void __launch_bounds__(RBE_BLOCK)
k_rbe_rho_partial_f64(int n, int p, int chunk, double kxs, double kys, double kzs,
                      const double* __restrict__ mx, const double* __restrict__ my,
                      const double* __restrict__ mz, const double* __restrict__ q,
                      const double* __restrict__ x, const double* __restrict__ y,
                      const double* __restrict__ z, double* __restrict__ part_re,
                      double* __restrict__ part_im, SampleArgs sa) {
  __shared__ double s_re[RBE_WARPS][(32 * KPT)];
  __shared__ double s_im[RBE_WARPS][(32 * KPT)];
  __shared__ int s_m[3][32 * KPT];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int kbase = blockIdx.y * (32 * KPT);
  if (sa.tables) rbe_group_samples<KPT>(sa, p, kbase, s_m, blockIdx.x == 0);
  double kx[KPT], ky[KPT], kz[KPT], sr[KPT], si[KPT];
#pragma unroll
  for (int t = 0; t < KPT; ++t) {
    const int k = kbase + lane + 32 * t;
    const bool ok = k < p;
    const double m0 = sa.tables ? (double)s_m[0][lane + 32 * t] : (ok ? mx[k] : 0.0);
    const double m1 = sa.tables ? (double)s_m[1][lane + 32 * t] : (ok ? my[k] : 0.0);
    const double m2 = sa.tables ? (double)s_m[2][lane + 32 * t] : (ok ? mz[k] : 0.0);
    // k = 2 pi m / L, evaluated as (2 pi * m) / L like the reference.
    kx[t] = ok ? (2 * RBX_PI * m0) / kxs : 0.0;
    ky[t] = ok ? (2 * RBX_PI * m1) / kys : 0.0;
    kz[t] = ok ? (2 * RBX_PI * m2) / kzs : 0.0;
    sr[t] = 0.0;
    si[t] = 0.0;
  }
  const int a0 = blockIdx.x * chunk;
  const int a1 = min(n, a0 + chunk);
  const int sub = (chunk + RBE_WARPS - 1) / RBE_WARPS;
  const int w0 = a0 + warp * sub, w1 = min(a1, w0 + sub);
  for (int j = w0; j < w1; ++j) {
    const double xj = __ldg(x + j), yj = __ldg(y + j), zj = __ldg(z + j), qj = __ldg(q + j);
#pragma unroll
    for (int t = 0; t < KPT; ++t) {
      const double dot = kx[t] * xj + ky[t] * yj + kz[t] * zj;
      double s, c;
      sincos(dot, &s, &c);
      sr[t] += qj * c;
      si[t] += qj * s;
    }
  }
#pragma unroll
  for (int t = 0; t < KPT; ++t) {
    s_re[warp][lane + 32 * t] = sr[t];
    s_im[warp][lane + 32 * t] = si[t];
  }
  __syncthreads();
  for (int s = threadIdx.x; s < (32 * KPT); s += RBE_BLOCK) {
    const int k = kbase + s;
    if (k >= p) continue;
    double r = 0.0, im = 0.0;
    for (int w = 0; w < RBE_WARPS; ++w) {
      r += s_re[w][s];
      im += s_im[w][s];
    }
    part_re[(size_t)k * gridDim.x + blockIdx.x] = r;
    part_im[(size_t)k * gridDim.x + blockIdx.x] = im;
  }
}

// TwoSum (Knuth): s + e == a + b exactly.
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
  s = a + b;
  const float bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

// Mixed form.  Atom record: {ux, uy, uz, float bits of q}.  Lanes own k-vectors
// (integer m), atoms stream through the warp as broadcast loads.  Every
// RBE_TILE atoms the plain FP32 tile sums are folded into a compensated
// (hi, lo) pair.
constexpr int RBE_TILE = 32;

struct RhoMixedArgs {
  int n, p, chunk;
  const int* mi;
  const uint4* atoms;
  double *part_re, *part_im;
  SampleArgs sa;
  int gx;  // atom chunks (the grid is gx x k-groups)
};

// Block (bx, by) of the replica's grid.
template <int KPT>
__device__ __forceinline__ void rho_mixed_body(const RhoMixedArgs& A, int bx, int by) {
  const int n = A.n, p = A.p, chunk = A.chunk, gx = A.gx;
  const int* __restrict__ mi = A.mi;
  const uint4* __restrict__ atoms = A.atoms;
  double* __restrict__ part_re = A.part_re;
  double* __restrict__ part_im = A.part_im;
  const SampleArgs& sa = A.sa;
  __shared__ double s_re[RBE_WARPS][(32 * KPT)];
  __shared__ double s_im[RBE_WARPS][(32 * KPT)];
  __shared__ int s_m[3][32 * KPT];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int kbase = by * (32 * KPT);
  if (sa.tables) rbe_group_samples<KPT>(sa, p, kbase, s_m, bx == 0);
  int m0[KPT], m1[KPT], m2[KPT];
  float hr[KPT], lr[KPT], hi[KPT], li[KPT];
#pragma unroll
  for (int t = 0; t < KPT; ++t) {
    const int k = kbase + lane + 32 * t;
    const bool ok = k < p;
    m0[t] = sa.tables ? s_m[0][lane + 32 * t] : (ok ? mi[3 * k] : 0);
    m1[t] = sa.tables ? s_m[1][lane + 32 * t] : (ok ? mi[3 * k + 1] : 0);
    m2[t] = sa.tables ? s_m[2][lane + 32 * t] : (ok ? mi[3 * k + 2] : 0);
    hr[t] = lr[t] = hi[t] = li[t] = 0.f;
  }
  const float ang = (float)(2.0 * RBX_PI / 4294967296.0);
  const int a0 = bx * chunk;
  const int a1 = min(n, a0 + chunk);
  const int sub = (chunk + RBE_WARPS - 1) / RBE_WARPS;
  const int w0 = a0 + warp * sub, w1 = min(a1, w0 + sub);
  for (int jt = w0; jt < w1; jt += RBE_TILE) {
    const int je = min(w1, jt + RBE_TILE);
    float tr[KPT], ti[KPT];
#pragma unroll
    for (int t = 0; t < KPT; ++t) tr[t] = ti[t] = 0.f;
    for (int j = jt; j < je; ++j) {
      const uint4 a = __ldg(atoms + j);
      const float qj = __uint_as_float(a.w);
#pragma unroll
      for (int t = 0; t < KPT; ++t) {
        const unsigned ph = (unsigned)m0[t] * a.x + (unsigned)m1[t] * a.y + (unsigned)m2[t] * a.z;
        float s, c;
        __sincosf((float)(int)ph * ang, &s, &c);
        tr[t] = fmaf(qj, c, tr[t]);
        ti[t] = fmaf(qj, s, ti[t]);
      }
    }
#pragma unroll
    for (int t = 0; t < KPT; ++t) {
      float s, e;
      two_sum(hr[t], tr[t], s, e);
      hr[t] = s;
      lr[t] += e;
      two_sum(hi[t], ti[t], s, e);
      hi[t] = s;
      li[t] += e;
    }
  }
#pragma unroll
  for (int t = 0; t < KPT; ++t) {
    s_re[warp][lane + 32 * t] = (double)hr[t] + (double)lr[t];
    s_im[warp][lane + 32 * t] = (double)hi[t] + (double)li[t];
  }
  __syncthreads();
  for (int s = threadIdx.x; s < (32 * KPT); s += RBE_BLOCK) {
    const int k = kbase + s;
    if (k >= p) continue;
    double r = 0.0, im = 0.0;
    for (int w = 0; w < RBE_WARPS; ++w) {
      r += s_re[w][s];
      im += s_im[w][s];
    }
    part_re[(size_t)k * gx + bx] = r;
    part_im[(size_t)k * gx + bx] = im;
  }
}

template <int KPT>
__global__ void __launch_bounds__(RBE_BLOCK) k_rbe_rho_partial_mixed(RhoMixedArgs a) {
  rho_mixed_body<KPT>(a, blockIdx.x, blockIdx.y);
}

template <int KPT>
__global__ void __launch_bounds__(RBE_BLOCK)
k_rbe_rho_partial_mixed_batch(const RhoMixedArgs* __restrict__ a, const int* __restrict__ start,
                              int nrep) {
  const int r = batch_replica(start, nrep, blockIdx.x);
  const int b = blockIdx.x - __ldg(start + r), gx = a[r].gx;
  rho_mixed_body<KPT>(a[r], b % gx, b / gx);
}

// ---------------------------------------------------------------------------
// Finalize (one block of 1024 threads): rho_p = sum over the k-major partials
// (one warp per k, fixed tree); optional energy/virial (ComputeRBEVirial0,
// kspace_calculator_op.hip.cu:573-674) summed over k in fixed order; force
// table tab[p] = {kx, ky, kz, coef*Re, coef*Im} with coef = -4 pi qqr2e S /
// (P V k^2); optional mean of a force-partial array (RBL mean removal).
// ---------------------------------------------------------------------------
constexpr int FIN_BLOCK = 256;
constexpr int FIN_WIDE = 1024;

__global__ void __launch_bounds__(FIN_WIDE)
k_rbe_finalize(int p, int nparts, const double* __restrict__ part_re,
               const double* __restrict__ part_im, const double* __restrict__ mx,
               const double* __restrict__ my, const double* __restrict__ mz, double Lx,
               double Ly, double Lz, double alpha, double S, double qqr2e, double qsq,
               double qsum, double* __restrict__ rho_re, double* __restrict__ rho_im,
               double* __restrict__ energy, double* __restrict__ virial,
               KTab* __restrict__ tab, int mean_parts, const double* __restrict__ fpart,
               double n_atoms, double* __restrict__ mean_out) {
  __shared__ double s_e[7][FIN_WIDE / 32];
  __shared__ double sh[FIN_WIDE / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double V = Lx * Ly * Lz;
  const double coef = (2 * RBX_PI * S) / (p * V);
  const double fcoef = -4 * RBX_PI * qqr2e * S / p;
  // per-warp running sums of the per-k energy/virial terms, k in increasing order
  double we[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int k = warp; k < p; k += FIN_WIDE / 32) {
    double r = 0.0, im = 0.0;
    const double* pr = part_re + (size_t)k * nparts;
    const double* pi = part_im + (size_t)k * nparts;
    for (int b = lane; b < nparts; b += 32) {
      r += pr[b];
      im += pi[b];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      r += __shfl_xor_sync(0xffffffffu, r, o);
      im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    if (lane == 0) {
      if (rho_re) {
        rho_re[k] = r;
        rho_im[k] = im;
      }
      const double kx = 2 * RBX_PI * mx[k] / Lx;
      const double ky = 2 * RBX_PI * my[k] / Ly;
      const double kz = 2 * RBX_PI * mz[k] / Lz;
      const double k2 = kx * kx + ky * ky + kz * kz;
      const double rho2 = r * r + im * im;
      const double base = coef * rho2 / k2;
      const double inner = (1.0 / (4 * alpha)) + (1.0 / k2);
      we[0] += base;
      we[1] += base * (1.0 - 2 * kx * kx * inner);
      we[2] += base * (1.0 - 2 * ky * ky * inner);
      we[3] += base * (1.0 - 2 * kz * kz * inner);
      we[4] += base * (-2 * kx * ky * inner);
      we[5] += base * (-2 * kx * kz * inner);
      we[6] += base * (-2 * ky * kz * inner);
      if (tab) {
        const double c = fcoef / (V * k2);
        KTab t;
        t.kx = kx;
        t.ky = ky;
        t.kz = kz;
        t.a = c * r;
        t.b = c * im;
        t.m[0] = (int)mx[k];
        t.m[1] = (int)my[k];
        t.m[2] = (int)mz[k];
        t.m[3] = 0;
        tab[k] = t;
      }
    }
  }
  if (energy) {
    if (lane == 0)
      for (int c = 0; c < 7; ++c) s_e[c][warp] = we[c];
    __syncthreads();
    if (threadIdx.x == 0) {
      double t[7] = {0, 0, 0, 0, 0, 0, 0};
      for (int w = 0; w < FIN_WIDE / 32; ++w)
        for (int c = 0; c < 7; ++c) t[c] += s_e[c][w];
      const double MY_PIS = 1.77245385090551602729, MY_PI2 = 1.57079632679489661923;
      const double etot = t[0] - (sqrt(alpha) * qsq / MY_PIS + MY_PI2 * qsum * qsum / (alpha * V));
      *energy = etot * qqr2e;
      for (int c = 0; c < 6; ++c) virial[c] = t[1 + c] * qqr2e;
    }
  }
  if (mean_out) {
    for (int d = 0; d < 3; ++d) {
      double s = 0.0;
      for (int b = threadIdx.x; b < mean_parts; b += FIN_WIDE) s += fpart[(size_t)b * 3 + d];
      s = block_sum_det<FIN_WIDE>(s, sh);
      if (threadIdx.x == 0) mean_out[d] = s / n_atoms;
    }
  }
}

// Parallel finalize: block k < p reduces the partials of k-vector k (fixed
// strided order, then a fixed tree) and writes rho(k), the force table entry
// and its seven energy/virial terms to kterm[k][0..6]; blocks p..p+2 reduce
// the per-block pair-force sums into the mean force.  The per-k terms are then
// added in increasing k by one warp in a fixed order: k_rbe_energy_sum, or,
// with es.ctr, the last block of this kernel to finish.
constexpr int FK_BLOCK = 128;

struct EnergySum {
  unsigned* ctr;  // block counter, zero before the launch; cleared again by the last block
  double alpha, V, qqr2e, qsq, qsum;
  double* energy;
  double* virial;
};

__device__ __forceinline__ void rbe_energy_sum_warp(int p, const double* __restrict__ kterm,
                                                    const EnergySum& es, bool coherent) {
  const int lane = threadIdx.x & 31;
  double t[7] = {0, 0, 0, 0, 0, 0, 0};
  // each lane adds its k in increasing order; the seven loads of a k are independent
  for (int k = lane; k < p; k += 32) {
    const double* r = kterm + (size_t)k * 8;
#pragma unroll
    for (int c = 0; c < 7; ++c) t[c] += coherent ? __ldcg(r + c) : r[c];
  }
#pragma unroll
  for (int c = 0; c < 7; ++c)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t[c] += __shfl_down_sync(0xffffffffu, t[c], o);
  if (lane == 0) {
    const double MY_PIS = 1.77245385090551602729, MY_PI2 = 1.57079632679489661923;
    const double etot =
        t[0] - (sqrt(es.alpha) * es.qsq / MY_PIS + MY_PI2 * es.qsum * es.qsum / (es.alpha * es.V));
    *es.energy = etot * es.qqr2e;
    for (int c = 0; c < 6; ++c) es.virial[c] = t[1 + c] * es.qqr2e;
  }
}

__device__ void rbe_finalize_one(int k, int p, int nparts, const double* __restrict__ part_re,
                                 const double* __restrict__ part_im, const double* __restrict__ mx,
                                 const double* __restrict__ my, const double* __restrict__ mz,
                                 double Lx, double Ly, double Lz, double alpha, double S,
                                 double qqr2e, double* __restrict__ rho_re,
                                 double* __restrict__ rho_im, KTab* __restrict__ tab,
                                 double* __restrict__ kterm, double* sh);

struct FinalizeArgs {
  int p, nparts;
  const double *part_re, *part_im, *mx, *my, *mz;
  double Lx, Ly, Lz, alpha, S, qqr2e;
  double *rho_re, *rho_im;
  KTab* tab;
  double* kterm;
  int mean_parts;
  const double* fpart;
  double n_atoms;
  double* mean_out;
  EnergySum es;
};

// Block blk of a grid of gx blocks.
__device__ __forceinline__ void finalize_k_body(const FinalizeArgs& A, int blk, int gx) {
  const int p = A.p, nparts = A.nparts, mean_parts = A.mean_parts;
  const double* __restrict__ part_re = A.part_re;
  const double* __restrict__ part_im = A.part_im;
  const double* __restrict__ fpart = A.fpart;
  double* __restrict__ kterm = A.kterm;
  double* __restrict__ mean_out = A.mean_out;
  const double n_atoms = A.n_atoms;
  const EnergySum& es = A.es;
  __shared__ double sh[FK_BLOCK / 32];
  __shared__ bool s_last;
  if (blk >= p) {  // mean of the pair-force block sums, one component per block
    const int d = blk - p;
    double s = 0.0;
    for (int b = threadIdx.x; b < mean_parts; b += FK_BLOCK) s += fpart[(size_t)b * 3 + d];
    s = block_sum_det<FK_BLOCK>(s, sh);
    if (threadIdx.x == 0) mean_out[d] = s / n_atoms;
  } else {
    rbe_finalize_one(blk, p, nparts, part_re, part_im, A.mx, A.my, A.mz, A.Lx, A.Ly, A.Lz,
                     A.alpha, A.S, A.qqr2e, A.rho_re, A.rho_im, A.tab, kterm, sh);
  }
  if (!es.ctr) return;
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(es.ctr, 1u) == (unsigned)gx - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (threadIdx.x < 32) rbe_energy_sum_warp(p, kterm, es, true);
  if (threadIdx.x == 0) *es.ctr = 0u;
}

__global__ void __launch_bounds__(FK_BLOCK) k_rbe_finalize_k(FinalizeArgs a) {
  finalize_k_body(a, blockIdx.x, gridDim.x);
}

__global__ void __launch_bounds__(FK_BLOCK)
k_rbe_finalize_k_batch(const FinalizeArgs* __restrict__ a, const int* __restrict__ start,
                       int nrep) {
  const int r = batch_replica(start, nrep, blockIdx.x);
  const int b0 = __ldg(start + r);
  finalize_k_body(a[r], blockIdx.x - b0, __ldg(start + r + 1) - b0);
}

// Block k's part of the finalize (all threads of the block call it).
__device__ void rbe_finalize_one(int k, int p, int nparts, const double* __restrict__ part_re,
                                 const double* __restrict__ part_im, const double* __restrict__ mx,
                                 const double* __restrict__ my, const double* __restrict__ mz,
                                 double Lx, double Ly, double Lz, double alpha, double S,
                                 double qqr2e, double* __restrict__ rho_re,
                                 double* __restrict__ rho_im, KTab* __restrict__ tab,
                                 double* __restrict__ kterm, double* sh) {
  double r = 0.0, im = 0.0;
  const double* pr = part_re + (size_t)k * nparts;
  const double* pi = part_im + (size_t)k * nparts;
  for (int b = threadIdx.x; b < nparts; b += FK_BLOCK) {
    r += pr[b];
    im += pi[b];
  }
  r = block_sum_det<FK_BLOCK>(r, sh);
  im = block_sum_det<FK_BLOCK>(im, sh);
  if (threadIdx.x != 0) return;
  if (rho_re) {
    rho_re[k] = r;
    rho_im[k] = im;
  }
  const double V = Lx * Ly * Lz;
  const double kx = 2 * RBX_PI * mx[k] / Lx;
  const double ky = 2 * RBX_PI * my[k] / Ly;
  const double kz = 2 * RBX_PI * mz[k] / Lz;
  const double k2 = kx * kx + ky * ky + kz * kz;
  if (kterm) {
    const double coef = (2 * RBX_PI * S) / (p * V);
    const double base = coef * (r * r + im * im) / k2;
    const double inner = (1.0 / (4 * alpha)) + (1.0 / k2);
    double* t = kterm + (size_t)k * 8;
    t[0] = base;
    t[1] = base * (1.0 - 2 * kx * kx * inner);
    t[2] = base * (1.0 - 2 * ky * ky * inner);
    t[3] = base * (1.0 - 2 * kz * kz * inner);
    t[4] = base * (-2 * kx * ky * inner);
    t[5] = base * (-2 * kx * kz * inner);
    t[6] = base * (-2 * ky * kz * inner);
  }
  if (tab) {
    const double c = (-4 * RBX_PI * qqr2e * S / p) / (V * k2);
    KTab t;
    t.kx = kx;
    t.ky = ky;
    t.kz = kz;
    t.a = c * r;
    t.b = c * im;
    t.m[0] = (int)mx[k];
    t.m[1] = (int)my[k];
    t.m[2] = (int)mz[k];
    t.m[3] = 0;
    tab[k] = t;
  }
}

__global__ void __launch_bounds__(32)
k_rbe_energy_sum(int p, const double* __restrict__ kterm, EnergySum es) {
  rbe_energy_sum_warp(p, kterm, es, false);
}

// ---------------------------------------------------------------------------
// Force scatter.  Thread per atom; the k table is staged in shared memory.
// Epilogue variants: plain store of F_k, or the fused combine
// F = F_pair - mean + F_k with the second velocity-Verlet half kick.
// ---------------------------------------------------------------------------
constexpr int FRC_TABLE = 512;  // k entries staged per pass

struct ForceEpilogue {
  const double* f_pair_x;  // may be null: store F_k only
  const double* f_pair_y;
  const double* f_pair_z;
  const double* mean;      // may be null
  double* f_out_x;         // total (or k-space only)
  double* f_out_y;
  double* f_out_z;
  double* fk_x;            // optional copy of the k-space part
  double* fk_y;
  double* fk_z;
  double* vx;              // optional half kick
  double* vy;
  double* vz;
  const int* type;
  const double* inv_mass;  // per type
  double half_dt;
};

__device__ __forceinline__ void force_epilogue(const ForceEpilogue& ep, int i, double fx,
                                               double fy, double fz) {
  if (ep.fk_x) {
    ep.fk_x[i] = fx;
    ep.fk_y[i] = fy;
    ep.fk_z[i] = fz;
  }
  if (ep.f_pair_x) {
    double mx = 0, my = 0, mz = 0;
    if (ep.mean) {
      mx = ep.mean[0];
      my = ep.mean[1];
      mz = ep.mean[2];
    }
    fx += ep.f_pair_x[i] - mx;
    fy += ep.f_pair_y[i] - my;
    fz += ep.f_pair_z[i] - mz;
  }
  ep.f_out_x[i] = fx;
  ep.f_out_y[i] = fy;
  ep.f_out_z[i] = fz;
  if (ep.vx) {
    const double im = ep.inv_mass[ep.type[i]] * ep.half_dt;
    ep.vx[i] += fx * im;
    ep.vy[i] += fy * im;
    ep.vz[i] += fz * im;
  }
}

template <int FB>
__global__ void __launch_bounds__(FB)
k_rbe_force_f64(int n, int p, const KTab* __restrict__ tab, const double* __restrict__ q,
                const double* __restrict__ x, const double* __restrict__ y,
                const double* __restrict__ z, ForceEpilogue ep) {
  __shared__ KTab s_tab[FRC_TABLE];
  const int i = blockIdx.x * FB + threadIdx.x;
  const bool live = i < n;
  const double xi = live ? x[i] : 0.0, yi = live ? y[i] : 0.0, zi = live ? z[i] : 0.0;
  double fx = 0, fy = 0, fz = 0;
  for (int k0 = 0; k0 < p; k0 += FRC_TABLE) {
    const int kn = min(FRC_TABLE, p - k0);
    __syncthreads();
    for (int s = threadIdx.x; s < kn; s += FB) s_tab[s] = tab[k0 + s];
    __syncthreads();
    if (live) {
      for (int s = 0; s < kn; ++s) {
        const KTab t = s_tab[s];
        const double dot = t.kx * xi + t.ky * yi + t.kz * zi;
        double sn, cs;
        sincos(dot, &sn, &cs);
        const double f = cs * t.b - sn * t.a;
        fx += f * t.kx;
        fy += f * t.ky;
        fz += f * t.kz;
      }
    }
  }
  if (live) {
    const double qi = q[i];
    force_epilogue(ep, i, fx * qi, fy * qi, fz * qi);
  }
}

// Mixed-form force table entry (FP32 coefficients, integer m).
struct KTabF {
  int m0, m1, m2;
  float a, b, kx, ky, kz;
};

struct ForceMixedArgs {
  int n, p;
  const KTab* tab;
  const uint4* atoms;
  ForceEpilogue ep;
};

template <int FB>
__device__ __forceinline__ void force_mixed_body(const ForceMixedArgs& A, int bx) {
  const int n = A.n, p = A.p;
  const KTab* __restrict__ tab = A.tab;
  const uint4* __restrict__ atoms = A.atoms;
  const ForceEpilogue& ep = A.ep;
  __shared__ KTabF s_tab[FRC_TABLE];
  const int i = bx * FB + threadIdx.x;
  const bool live = i < n;
  const uint4 a = live ? atoms[i] : make_uint4(0, 0, 0, 0);
  const float ang = (float)(2.0 * RBX_PI / 4294967296.0);
  float fx = 0.f, fy = 0.f, fz = 0.f;
  for (int k0 = 0; k0 < p; k0 += FRC_TABLE) {
    const int kn = min(FRC_TABLE, p - k0);
    __syncthreads();
    for (int s = threadIdx.x; s < kn; s += FB) {
      const KTab t = tab[k0 + s];
      KTabF f;
      f.m0 = t.m[0];
      f.m1 = t.m[1];
      f.m2 = t.m[2];
      f.a = (float)t.a;
      f.b = (float)t.b;
      f.kx = (float)t.kx;
      f.ky = (float)t.ky;
      f.kz = (float)t.kz;
      s_tab[s] = f;
    }
    __syncthreads();
    if (live) {
      for (int s = 0; s < kn; ++s) {
        const KTabF t = s_tab[s];
        const unsigned ph = (unsigned)t.m0 * a.x + (unsigned)t.m1 * a.y + (unsigned)t.m2 * a.z;
        float sn, cs;
        __sincosf((float)(int)ph * ang, &sn, &cs);
        const float f = cs * t.b - sn * t.a;
        fx = fmaf(f, t.kx, fx);
        fy = fmaf(f, t.ky, fy);
        fz = fmaf(f, t.kz, fz);
      }
    }
  }
  if (live) {
    const double qi = (double)__uint_as_float(a.w);
    force_epilogue(ep, i, (double)fx * qi, (double)fy * qi, (double)fz * qi);
  }
}

template <int FB>
__global__ void __launch_bounds__(FB) k_rbe_force_mixed(ForceMixedArgs a) {
  force_mixed_body<FB>(a, blockIdx.x);
}

template <int FB>
__global__ void __launch_bounds__(FB)
k_rbe_force_mixed_batch(const ForceMixedArgs* __restrict__ a, const int* __restrict__ start,
                        int nrep) {
  const int r = batch_replica(start, nrep, blockIdx.x);
  force_mixed_body<FB>(a[r], blockIdx.x - __ldg(start + r));
}

// ---------------------------------------------------------------------------
// Philox k-sampler: one thread per sample; per-axis inverse-CDF tables built
// on the host (order m = 0, +1, -1, +2, -2, ...).
// ---------------------------------------------------------------------------
// cdf[t] = w[0] + ... + w[t], accumulated left to right on the host exactly as
// the oracle's linear scan accumulates, so the first t with target < cdf[t]
// (binary search) is the oracle's pick.

constexpr int kSampleSmemTables = 6144;  // staged table entries (48 KB)
constexpr int SAMPLE_BLOCK = 128;

__global__ void __launch_bounds__(SAMPLE_BLOCK)
k_rbe_sample(int p, const double* __restrict__ tables, int c0, int c1, int c2, double t0,
             double t1, double t2, uint32_t key0, uint32_t key1, uint64_t step_arg,
             const int* __restrict__ step_dev, double* __restrict__ mx, double* __restrict__ my,
             double* __restrict__ mz, int* __restrict__ mi, int* __restrict__ status) {
  // the three cumulative tables are staged in shared memory when they fit
  // (dynamic size (c0 + c1 + c2) doubles), so the binary searches run there
  extern __shared__ double s_tab[];
  const int tot = c0 + c1 + c2;
  const bool staged = tot <= kSampleSmemTables;
  if (staged) {
    for (int t = threadIdx.x; t < tot; t += blockDim.x) s_tab[t] = tables[t];
    __syncthreads();
  }
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= p) return;
  // the MD step: a device copy inside a step graph
  const uint64_t step = step_dev ? (uint64_t)(int64_t)*step_dev : step_arg;
  SampleArgs sa{};
  sa.c0 = c0;
  sa.c1 = c1;
  sa.c2 = c2;
  sa.t0 = t0;
  sa.t1 = t1;
  sa.t2 = t2;
  sa.key0 = key0;
  sa.key1 = key1;
  int m[3];
  if (!rbe_draw(s, sa, staged ? s_tab : tables, step, m)) {
    atomicOr(status, 1);
    return;
  }
  if (mx) {
    mx[s] = m[0];
    my[s] = m[1];
    mz[s] = m[2];
  }
  if (mi) {
    mi[3 * s] = m[0];
    mi[3 * s + 1] = m[1];
    mi[3 * s + 2] = m[2];
  }
}

// Integer copy of injected samples (for the mixed kernels).
__global__ void k_m_to_int(int p, const double* __restrict__ mx, const double* __restrict__ my,
                           const double* __restrict__ mz, int* __restrict__ mi) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= p) return;
  mi[3 * s] = (int)mx[s];
  mi[3 * s + 1] = (int)my[s];
  mi[3 * s + 2] = (int)mz[s];
}

// ---------------------------------------------------------------------------
// Exact Ewald over the kmax box (oracle support / statistical reference).
// ---------------------------------------------------------------------------
__global__ void k_ewald_rho(int n, int nk, int kx_max, int ky_max, int kz_max, double Lx,
                            double Ly, double Lz, const double* __restrict__ q,
                            const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, double* __restrict__ re,
                            double* __restrict__ im, double* __restrict__ kvec) {
  __shared__ double sh[FIN_BLOCK / 32];
  const int k = blockIdx.x;
  // k index -> (i, j, l) in ExecuteOnKmax order, skipping the origin.
  const int ny = 2 * ky_max + 1, nz = 2 * kz_max + 1;
  const int center = kx_max * ny * nz + ky_max * nz + kz_max;
  const int flat = k < center ? k : k + 1;
  const int ii = flat / (ny * nz) - kx_max;
  const int jj = (flat / nz) % ny - ky_max;
  const int ll = flat % nz - kz_max;
  const double kx = 2 * RBX_PI * ii / Lx, ky = 2 * RBX_PI * jj / Ly, kz = 2 * RBX_PI * ll / Lz;
  double sr = 0, si = 0;
  for (int j = threadIdx.x; j < n; j += FIN_BLOCK) {
    double s, c;
    sincos(kx * x[j] + ky * y[j] + kz * z[j], &s, &c);
    sr += q[j] * c;
    si += q[j] * s;
  }
  sr = block_sum_det<FIN_BLOCK>(sr, sh);
  si = block_sum_det<FIN_BLOCK>(si, sh);
  if (threadIdx.x == 0) {
    re[k] = sr;
    im[k] = si;
    kvec[3 * k] = kx;
    kvec[3 * k + 1] = ky;
    kvec[3 * k + 2] = kz;
  }
}

__global__ void k_ewald_force(int n, int nk, double V, double alpha, double qqr2e,
                              const double* __restrict__ kvec, const double* __restrict__ re,
                              const double* __restrict__ im, const double* __restrict__ q,
                              const double* __restrict__ x, const double* __restrict__ y,
                              const double* __restrict__ z, double* __restrict__ fx,
                              double* __restrict__ fy, double* __restrict__ fz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double base = -4.0 * RBX_PI * q[i];
  const double ainv = 1.0 / alpha;
  double sx = 0, sy = 0, sz = 0;
  for (int k = 0; k < nk; ++k) {
    const double kx = kvec[3 * k], ky = kvec[3 * k + 1], kz = kvec[3 * k + 2];
    const double k2 = kx * kx + ky * ky + kz * kz;
    double s, c;
    sincos(-(kx * x[i] + ky * y[i] + kz * z[i]), &s, &c);
    double f = base / (V * k2) * exp(-0.25 * k2 * ainv) * (c * im[k] + s * re[k]);
    f *= qqr2e;
    sx += f * kx;
    sy += f * ky;
    sz += f * kz;
  }
  fx[i] = sx;
  fy[i] = sy;
  fz[i] = sz;
}

__global__ void k_ewald_energy(int nk, double V, double alpha, double qqr2e, double qsq,
                               const double* __restrict__ kvec, const double* __restrict__ re,
                               const double* __restrict__ im, double* __restrict__ energy) {
  __shared__ double sh[FIN_BLOCK / 32];
  double e = 0;
  for (int k = threadIdx.x; k < nk; k += FIN_BLOCK) {
    const double kx = kvec[3 * k], ky = kvec[3 * k + 1], kz = kvec[3 * k + 2];
    const double k2 = kx * kx + ky * ky + kz * kz;
    e += exp(-0.25 * k2 / alpha) / k2 * (re[k] * re[k] + im[k] * im[k]);
  }
  e = block_sum_det<FIN_BLOCK>(e, sh);
  if (threadIdx.x == 0) *energy = qqr2e * (2 * RBX_PI / V) * e + qqr2e * (-sqrt(alpha / RBX_PI) * qsq);
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
int rbe_partial_blocks(int n) {
  // about four waves of 256-thread blocks on the 148 SMs, at least 64 atoms each
  const int target = sm_count() * 4;
  int blocks = (n + 63) / 64;
  if (blocks > target) blocks = target;
  return blocks < 1 ? 1 : blocks;
}

// kpt: k-vectors per thread (1, 2, 4 or 8; 32 kpt per block); the partial
// sums do not depend on it.
int launch_rbe_rho_partial_f64(const DBox& b, int n, int p, const double* mx, const double* my,
                               const double* mz, const double* q, const double* x,
                               const double* y, const double* z, double* part_re,
                               double* part_im, int nblocks, cudaStream_t st, int kpt,
                               const SampleArgs* sample) {
  if (n <= 0 || p <= 0) return RBX_OK;
  const int chunk = (n + nblocks - 1) / nblocks;
  dim3 grid(nblocks, (p + 32 * kpt - 1) / (32 * kpt));
  const SampleArgs sa = sample ? *sample : SampleArgs{};
#define RHO_F64(K)                                                                             \
  k_rbe_rho_partial_f64<K><<<grid, RBE_BLOCK, 0, st>>>(n, p, chunk, b.len[0], b.len[1],       \
                                                       b.len[2], mx, my, mz, q, x, y, z,       \
                                                       part_re, part_im, sa)
  switch (kpt) {
    case 1: RHO_F64(1); break;
    case 2: RHO_F64(2); break;
    case 8: RHO_F64(8); break;
    default: RHO_F64(4); break;
  }
#undef RHO_F64
  count_launch();
  return check_launch("rbe_rho_partial_f64");
}

int launch_rbe_rho_partial_mixed(int n, int p, const int* mi, const uint4* atoms,
                                 double* part_re, double* part_im, int nblocks, cudaStream_t st,
                                 int kpt, const SampleArgs* sample) {
  if (n <= 0 || p <= 0) return RBX_OK;
  const int chunk = (n + nblocks - 1) / nblocks;
  dim3 grid(nblocks, (p + 32 * kpt - 1) / (32 * kpt));
  RhoMixedArgs a;
  a.n = n;
  a.p = p;
  a.chunk = chunk;
  a.mi = mi;
  a.atoms = atoms;
  a.part_re = part_re;
  a.part_im = part_im;
  a.sa = sample ? *sample : SampleArgs{};
  a.gx = nblocks;
  if (kpt != 1 && kpt != 2 && kpt != 8) kpt = 4;
  if (batch_recorder())
    return record_phase(PH_RHO, kpt, (int)(grid.x * grid.y), RBE_BLOCK, 0, &a, sizeof a);
#define RHO_MIX(K) k_rbe_rho_partial_mixed<K><<<grid, RBE_BLOCK, 0, st>>>(a)
  switch (kpt) {
    case 1: RHO_MIX(1); break;
    case 2: RHO_MIX(2); break;
    case 8: RHO_MIX(8); break;
    default: RHO_MIX(4); break;
  }
#undef RHO_MIX
  count_launch();
  return check_launch("rbe_rho_partial_mixed");
}

int launch_rbe_finalize(const DBox& b, int p, int nparts, const double* part_re,
                        const double* part_im, const double* mx, const double* my,
                        const double* mz, double alpha, double S, double qqr2e, double qsq,
                        double qsum, double* rho_re, double* rho_im, double* energy,
                        double* virial, KTab* tab, int mean_parts, const double* fpart,
                        int n_atoms, double* mean_out, double* kterm, cudaStream_t st,
                        unsigned* sum_ctr) {
  if (energy && !kterm) {  // no per-k scratch: one block does it all
    k_rbe_finalize<<<1, FIN_WIDE, 0, st>>>(p, nparts, part_re, part_im, mx, my, mz, b.len[0],
                                            b.len[1], b.len[2], alpha, S, qqr2e, qsq, qsum,
                                            rho_re, rho_im, energy, virial, tab, mean_parts, fpart,
                                            (double)n_atoms, mean_out);
    count_launch();
    return check_launch("rbe_finalize");
  }
  const int grid = p + (mean_out ? 3 : 0);
  EnergySum es{nullptr, alpha, b.len[0] * b.len[1] * b.len[2], qqr2e, qsq, qsum, energy, virial};
  // the energy sum in the finalize's last block when a counter is given
  const bool fold = energy && sum_ctr && grid > 0 && p > 0;
  if (grid > 0) {
    FinalizeArgs a;
    a.p = p;
    a.nparts = nparts;
    a.part_re = part_re;
    a.part_im = part_im;
    a.mx = mx;
    a.my = my;
    a.mz = mz;
    a.Lx = b.len[0];
    a.Ly = b.len[1];
    a.Lz = b.len[2];
    a.alpha = alpha;
    a.S = S;
    a.qqr2e = qqr2e;
    a.rho_re = rho_re;
    a.rho_im = rho_im;
    a.tab = tab;
    a.kterm = energy ? kterm : nullptr;
    a.mean_parts = mean_parts;
    a.fpart = fpart;
    a.n_atoms = (double)n_atoms;
    a.mean_out = mean_out;
    a.es = es;
    a.es.ctr = fold ? sum_ctr : nullptr;
    if (batch_recorder()) {
      if (energy && !fold) {
        set_error("rbe_finalize: a batched finalize needs the energy sum folded in");
        return RBX_ERR_INVALID;
      }
      return record_phase(PH_FINALIZE, 0, grid, FK_BLOCK, 0, &a, sizeof a);
    }
    k_rbe_finalize_k<<<grid, FK_BLOCK, 0, st>>>(a);
    count_launch();
    const int rc = check_launch("rbe_finalize_k");
    if (rc) return rc;
  }
  if (energy && !fold) {
    k_rbe_energy_sum<<<1, 32, 0, st>>>(p, kterm, es);
    count_launch();
  }
  return check_launch("rbe_energy_sum");
}

static ForceEpilogue make_ep(const RbeForceOut& o) {
  ForceEpilogue ep;
  ep.f_pair_x = o.f_pair_x;
  ep.f_pair_y = o.f_pair_y;
  ep.f_pair_z = o.f_pair_z;
  ep.mean = o.mean;
  ep.f_out_x = o.f_out_x;
  ep.f_out_y = o.f_out_y;
  ep.f_out_z = o.f_out_z;
  ep.fk_x = o.fk_x;
  ep.fk_y = o.fk_y;
  ep.fk_z = o.fk_z;
  ep.vx = o.vx;
  ep.vy = o.vy;
  ep.vz = o.vz;
  ep.type = o.type;
  ep.inv_mass = o.inv_mass;
  ep.half_dt = o.half_dt;
  return ep;
}

// block: atoms per block (128, 256 or 512); the forces do not depend on it.
int launch_rbe_force_f64(int n, int p, const KTab* tab, const double* q, const double* x,
                         const double* y, const double* z, const RbeForceOut& out,
                         cudaStream_t st, int block) {
  if (n <= 0) return RBX_OK;
  const ForceEpilogue ep = make_ep(out);
  if (block == 128)
    k_rbe_force_f64<128><<<(n + 127) / 128, 128, 0, st>>>(n, p, tab, q, x, y, z, ep);
  else if (block == 512)
    k_rbe_force_f64<512><<<(n + 511) / 512, 512, 0, st>>>(n, p, tab, q, x, y, z, ep);
  else
    k_rbe_force_f64<256><<<(n + 255) / 256, 256, 0, st>>>(n, p, tab, q, x, y, z, ep);
  count_launch();
  return check_launch("rbe_force_f64");
}

int launch_rbe_force_mixed(int n, int p, const KTab* tab, const uint4* atoms,
                           const RbeForceOut& out, cudaStream_t st, int block) {
  if (n <= 0) return RBX_OK;
  ForceMixedArgs a;
  a.n = n;
  a.p = p;
  a.tab = tab;
  a.atoms = atoms;
  a.ep = make_ep(out);
  if (block != 128 && block != 512) block = 256;
  if (batch_recorder())
    return record_phase(PH_FORCE, block, (n + block - 1) / block, block, 0, &a, sizeof a);
  if (block == 128)
    k_rbe_force_mixed<128><<<(n + 127) / 128, 128, 0, st>>>(a);
  else if (block == 512)
    k_rbe_force_mixed<512><<<(n + 511) / 512, 512, 0, st>>>(a);
  else
    k_rbe_force_mixed<256><<<(n + 255) / 256, 256, 0, st>>>(a);
  count_launch();
  return check_launch("rbe_force_mixed");
}

int launch_rho_mixed_batch(int variant, const void* args, const int* start, int nrep, int total,
                           cudaStream_t st) {
  const RhoMixedArgs* a = static_cast<const RhoMixedArgs*>(args);
  switch (variant) {
    case 1: k_rbe_rho_partial_mixed_batch<1><<<total, RBE_BLOCK, 0, st>>>(a, start, nrep); break;
    case 2: k_rbe_rho_partial_mixed_batch<2><<<total, RBE_BLOCK, 0, st>>>(a, start, nrep); break;
    case 8: k_rbe_rho_partial_mixed_batch<8><<<total, RBE_BLOCK, 0, st>>>(a, start, nrep); break;
    default: k_rbe_rho_partial_mixed_batch<4><<<total, RBE_BLOCK, 0, st>>>(a, start, nrep); break;
  }
  count_launch();
  return check_launch("rbe_rho_partial_mixed_batch");
}

int launch_finalize_batch(const void* args, const int* start, int nrep, int total,
                          cudaStream_t st) {
  k_rbe_finalize_k_batch<<<total, FK_BLOCK, 0, st>>>(static_cast<const FinalizeArgs*>(args),
                                                     start, nrep);
  count_launch();
  return check_launch("rbe_finalize_k_batch");
}

int launch_force_mixed_batch(int variant, const void* args, const int* start, int nrep,
                             int total, cudaStream_t st) {
  const ForceMixedArgs* a = static_cast<const ForceMixedArgs*>(args);
  if (variant == 128)
    k_rbe_force_mixed_batch<128><<<total, 128, 0, st>>>(a, start, nrep);
  else if (variant == 512)
    k_rbe_force_mixed_batch<512><<<total, 512, 0, st>>>(a, start, nrep);
  else
    k_rbe_force_mixed_batch<256><<<total, 256, 0, st>>>(a, start, nrep);
  count_launch();
  return check_launch("rbe_force_mixed_batch");
}

int launch_rbe_sample(int p, const double* tables, const int cnt[3], const double tot[3],
                      uint64_t seed, int64_t step, const int* step_dev, double* mx, double* my,
                      double* mz, int* mi, int* status, cudaStream_t st) {
  if (p <= 0) return RBX_OK;
  const int entries = cnt[0] + cnt[1] + cnt[2];
  const size_t smem = entries <= kSampleSmemTables ? sizeof(double) * entries : 0;
  k_rbe_sample<<<(p + SAMPLE_BLOCK - 1) / SAMPLE_BLOCK, SAMPLE_BLOCK, smem, st>>>(
      p, tables, cnt[0], cnt[1], cnt[2], tot[0], tot[1], tot[2], (uint32_t)seed,
      (uint32_t)(seed >> 32), (uint64_t)step, step_dev, mx, my, mz, mi, status);
  count_launch();
  return check_launch("rbe_sample");
}

SampleArgs make_sample_args(const double* tables, const int cnt[3], const double tot[3],
                            uint64_t seed, int64_t step, const int* step_dev, double* mx,
                            double* my, double* mz, int* mi, int* status) {
  SampleArgs sa{};
  sa.tables = tables;
  sa.c0 = cnt[0];
  sa.c1 = cnt[1];
  sa.c2 = cnt[2];
  sa.t0 = tot[0];
  sa.t1 = tot[1];
  sa.t2 = tot[2];
  sa.key0 = (uint32_t)seed;
  sa.key1 = (uint32_t)(seed >> 32);
  sa.step_arg = (uint64_t)step;
  sa.step_dev = step_dev;
  sa.mx = mx;
  sa.my = my;
  sa.mz = mz;
  sa.mi = mi;
  sa.status = status;
  return sa;
}

int launch_m_to_int(int p, const double* mx, const double* my, const double* mz, int* mi,
                    cudaStream_t st) {
  if (p <= 0) return RBX_OK;
  k_m_to_int<<<(p + 127) / 128, 128, 0, st>>>(p, mx, my, mz, mi);
  count_launch();
  return check_launch("m_to_int");
}

int launch_ewald(const DBox& b, int n, const int kmax[3], double alpha, double qqr2e,
                 double qsq, const double* q, const double* x, const double* y, const double* z,
                 double* re, double* im, double* kvec, double* fx, double* fy, double* fz,
                 double* energy, cudaStream_t st) {
  const int nk = (2 * kmax[0] + 1) * (2 * kmax[1] + 1) * (2 * kmax[2] + 1) - 1;
  if (nk <= 0) return RBX_OK;
  k_ewald_rho<<<nk, FIN_BLOCK, 0, st>>>(n, nk, kmax[0], kmax[1], kmax[2], b.len[0], b.len[1],
                                        b.len[2], q, x, y, z, re, im, kvec);
  count_launch();
  int rc = check_launch("ewald_rho");
  if (rc) return rc;
  const double V = b.len[0] * b.len[1] * b.len[2];
  if (n > 0) {
    k_ewald_force<<<(n + 127) / 128, 128, 0, st>>>(n, nk, V, alpha, qqr2e, kvec, re, im, q, x, y,
                                                   z, fx, fy, fz);
    count_launch();
    rc = check_launch("ewald_force");
    if (rc) return rc;
  }
  if (energy) {
    k_ewald_energy<<<1, FIN_BLOCK, 0, st>>>(nk, V, alpha, qqr2e, qsq, kvec, re, im, energy);
    count_launch();
    rc = check_launch("ewald_energy");
  }
  return rc;
}

}  // namespace rbx
