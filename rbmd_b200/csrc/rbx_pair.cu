// rbx_pair.cu -- real-space LJ 12-6 + erfc-Coulomb kernels for sm_100a.
//
// Engine path: one fused kernel per step reads the row-major candidate list
// (cut_off + skin) once, classifies every candidate with the reference's FP64
// list predicates (core r^2 < r_core^2 - EPS, shell r^2 < cut_off^2 - EPS,
// SplitMix64 pair hash % freq == 0 -- FilterRBLNeighborCandidates,
// src/neighbor_list/src/op/rocm/rbl_full_neighbor_list_op.hip.cu:237-304) and
// evaluates the pair force of ComputeLJCutCoulRBLForce
// (src/force/src/lj_cut_coul_kspace_op/rocm/lj_cut_coul_kspace_op.hip.cu:569-683)
// without writing the core/shell lists to HBM.
//
// Mapping: one warp per atom i.  Lanes take 32 candidates at a time; pairs that
// carry a force are compacted into a per-warp shared-memory queue, and the
// force math runs on full 32-pair batches, so the branchy classification and
// the expensive erfc/exp math do not diverge against each other.  Per-atom
// force sums are warp-reduced; per-block force totals (fixed order) feed the
// RBL mean-force removal.
#include <math.h>

#include <atomic>

#include <type_traits>

#include "rbx_common.cuh"
#include "rbx_kernels.h"
#include "rbx_pair_device.cuh"

namespace rbx {

constexpr int PAIR_BLOCK = 256;
constexpr int PAIR_WARPS = PAIR_BLOCK / 32;
constexpr int QCAP = 64;

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}


// LJ 12-6 force/r (lj126_rs, src/force/src/lj_op/rocm/lj_op.hip.cu:40-54) in FP64.
__device__ __forceinline__ double lj_f64(double eps_ij, double s6, double d2) {
  const double d6 = d2 * d2 * d2;
  const double sd6 = s6 / d6;
  return -24.0 * eps_ij * ((2.0 * sd6 - 1.0) * sd6) / d2;
}
// erfc-Coulomb force/r (CoulCutForce_rs_fix, lj_cut_coul_kspace_op.hip.cu:134-161).
__device__ __forceinline__ double coul_f64(double alpha, double sqrt_alpha, double qqr2e,
                                           double qq, double d2) {
  const double dis = sqrt(d2);
  const double g = erfc(sqrt_alpha * dis) / d2 +
                   2.0 * sqrt_alpha * exp(-alpha * d2) / (1.7724538509055160273 * dis);
  return -qqr2e * qq * g / dis;
}
__device__ __forceinline__ float lj_f32(float eps_ij, float s6, float d2) {
  const float d6 = d2 * d2 * d2;
  const float sd6 = s6 / d6;
  return -24.f * eps_ij * ((2.f * sd6 - 1.f) * sd6) / d2;
}
__device__ __forceinline__ float coul_f32(float alpha, float sqrt_alpha, float qqr2e, float qq,
                                          float d2) {
  const float rinv = rsqrtf(d2);
  const float dis = d2 * rinv;
  const float g = erfcf(sqrt_alpha * dis) * (rinv * rinv) +
                  (2.0f / 1.7724538509055160273f) * sqrt_alpha * expf(-alpha * d2) * rinv;
  return -qqr2e * qq * g * rinv;
}

// Per-type-pair LJ tables (eps_ij and sigma_ij^6, ntypes^2 entries each) in
// dynamic shared memory: FP64, then FP32 copies for the mixed form.
struct TypeTables {
  double* eps;
  double* s6;
  float* f_eps;
  float* f_s6;
};

size_t type_table_bytes(int ntypes, bool mixed) {
  return (size_t)ntypes * ntypes * (2 * sizeof(double) + (mixed ? 2 * sizeof(float) : 0));
}

// Carve the tables out of the dynamic shared memory and fill them (all
// threads of the block call this).
__device__ __forceinline__ TypeTables load_type_tables(const PairParams& pp, bool mixed) {
  extern __shared__ __align__(16) unsigned char s_types[];
  const int nt2 = pp.ntypes * pp.ntypes;
  TypeTables t;
  t.eps = reinterpret_cast<double*>(s_types);
  t.s6 = t.eps + nt2;
  t.f_eps = reinterpret_cast<float*>(t.s6 + nt2);
  t.f_s6 = t.f_eps + nt2;
  for (int e = threadIdx.x; e < nt2; e += blockDim.x) {
    const double ep = pp.lj_eps[e], s6 = pp.lj_s6[e];
    t.eps[e] = ep;
    t.s6[e] = s6;
    if (mixed) {
      t.f_eps[e] = (float)ep;
      t.f_s6[e] = (float)s6;
    }
  }
  __syncthreads();
  return t;
}

// Opt a kernel in to the dynamic shared memory its type tables need.
template <typename K>
int type_table_smem(K kern, int ntypes, bool mixed, size_t* bytes) {
  *bytes = type_table_bytes(ntypes, mixed);
  if (*bytes > 48 * 1024 &&
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*bytes) !=
          cudaSuccess) {
    cudaGetLastError();
    set_error("pair kernels: %d atom types need %zu bytes of shared memory", ntypes, *bytes);
    return RBX_ERR_INVALID;
  }
  return RBX_OK;
}

// Block partial of the per-atom forces, accumulated by lane 0 of each warp in
// atom order and combined over warps in warp order.
__device__ __forceinline__ void write_block_partial(double (*s_acc)[3], double* fpart,
                                                    int bx = -1) {
  __syncthreads();
  if (threadIdx.x < 3) {
    double s = 0.0;
    for (int w = 0; w < PAIR_WARPS; ++w) s += s_acc[w][threadIdx.x];
    fpart[(size_t)(bx < 0 ? (int)blockIdx.x : bx) * 3 + threadIdx.x] = s;
  }
}

// ---------------------------------------------------------------------------
// Candidate classification shared by both forms.
//
// The pair vector in fixed point, d = u_j - u_i (wrapped int32), is the exact
// minimum image of the FP64 pair vector to within 3 units of s_d = L_d/2^32
// per coordinate.  |d|^2 is formed in FP32 in units of s^2, s = L_max/2^32
// (on a box with unequal edges each coordinate is first weighted by
// L_d/L_max, which keeps its error below 3 units of s), and each predicate
// "r^2 < C" is decided when |d|^2 lies outside a guard band [lo, hi] around
// C/s^2 that exceeds every rounding and quantisation error; inside the band
// the reference's FP64 expression (CaculateDistance: i minus j, min image, no
// FMA) decides.  The outcome is therefore identical to the FP64 predicate on
// every pair, in both precision forms.
// ---------------------------------------------------------------------------
// Screened classification; *unsure is set when a threshold band is hit.  The
// band around core2_list and the one around rs2 (which lies just above it)
// are merged into one undecided interval, as are d2 values at or below the
// EPS band: each undecided pair is settled by the FP64 predicate, so five
// comparisons classify a pair.
__device__ __forceinline__ Classified classify_screen(const PairParams& pp, float d2s,
                                                      bool* unsure) {
  const bool A = d2s < pp.sc_core.lo;    // certainly d2 < core2_list
  const bool B = d2s <= pp.sc_rs.hi;     // not certainly d2 > rs2
  const bool C = d2s < pp.sc_force.lo;   // certainly d2 < force2_list
  const bool D = d2s < pp.sc_force.hi;   // not certainly d2 >= force2_list
  const bool E = d2s <= pp.sc_eps.hi;    // not certainly d2 > EPS
  *unsure = (!A && B) || (!C && D) || E;
  Classified c;
  c.core_active = A;
  c.shell_window = !B && C;
  return c;
}

__device__ __forceinline__ float fixed_d2(const uint4& ai, const uint4& aj) {
  const float dx = (float)(int)(aj.x - ai.x), dy = (float)(int)(aj.y - ai.y),
              dz = (float)(int)(aj.z - ai.z);
  return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
}
// The same in units of the longest edge's fixed-point step on a box with
// unequal edges (each difference weighted by L_d / L_max).
__device__ __forceinline__ float fixed_d2_weighted(const PairParams& pp, const uint4& ai,
                                                   const uint4& aj) {
  const float dx = (float)(int)(aj.x - ai.x) * pp.sw[0], dy = (float)(int)(aj.y - ai.y) * pp.sw[1],
              dz = (float)(int)(aj.z - ai.z) * pp.sw[2];
  return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
}

// ---------------------------------------------------------------------------
// Fused RBL filter + pair force over split candidate rows.
//
// The list builder writes each candidate row in two segments (see Rows): the
// near segment holds every pair whose build distance is below
// r_core + skin, the far segment (at the back of the row) every other pair.
// Until the next rebuild no atom moves more than skin / 2 from where the list
// was built, so a far pair is never a core pair: whether it carries a force
// this step is decided by its shell-batch hash first, and only the selected
// quarter (freq = 4) is gathered and tested against the shell window.  Near
// pairs are classified in full (fixed-point screen, FP64 predicate inside the
// guard bands) as the reference's FilterRBLNeighborCandidates does
// (rbl_full_neighbor_list_op.hip.cu:237-304).
//
// MIXED = false: plain FP64 (pair vector and force math in FP64 from the FP64
// positions).  MIXED = true: FP32 force math on the exact fixed-point pair
// vector.  SEL selects the batch test: 0 any freq (divisibility by
// multiplication), 1 freq a power of two (mask), 2 freq <= 4 (two bits of a
// partial hash).
//
// One warp per atom i.  A segment is walked in batches of U x 32 candidates:
// the index loads and gathers of a batch are issued before any is consumed,
// classification and the hash are branch-free, and force-carrying pairs are
// appended to a per-warp queue (index plus two flag bits) that is drained 32
// pairs at a time from its tail.
// ---------------------------------------------------------------------------
constexpr int RBL_NEAR_U = 3;  // 32-candidate chunks per near batch
constexpr int RBL_QCAP = 32 + 32 * (RBL_NEAR_U > 4 ? RBL_NEAR_U : 4);  // far batches: 128
constexpr int QF_SHELL = (int)0x80000000;  // shell pair: force times freq
constexpr int QF_CHECK = 0x40000000;       // far pair: shell window still to be tested
constexpr int QF_INDEX = 0x3fffffff;       // atom index (n < 2^30)

// LJ 12-6 force/r in FP32 with one fast reciprocal (mixed form only).
__device__ __forceinline__ float lj_f32_fast(float eps_ij, float s6, float d2) {
  const float r2i = __fdividef(1.0f, d2);
  const float sd6 = s6 * (r2i * r2i * r2i);
  return -24.f * eps_ij * ((2.f * sd6 - 1.f) * sd6) * r2i;
}

template <int SEL>
__device__ __forceinline__ bool batch_selected(unsigned long long key, unsigned long long fmask,
                                               const DivTest& div) {
  if (SEL == 2) return rbl_selected_low2(key, (unsigned)fmask);
  const unsigned long long h = rbl_mix(key);
  return SEL == 1 ? (h & fmask) == 0ULL : divisible(h, div);
}

// Pull the used lines of a split row toward L2 (32 ints = one 128-byte line a lane).
__device__ __forceinline__ void prefetch_row(const Rows& rows, int i, int lane) {
  int nf, nb;
  row_extent(rows, i, nf, nb);
  const int* r = rows.idx + (size_t)i * rows.cap;
  for (int k = lane * 32; k < nf; k += 32 * 32)
    asm volatile("prefetch.global.L2 [%0];" ::"l"(r + k));
  const int b0 = (rows.cap - nb) & ~31;  // rows start on 128-byte lines (cap % 32 == 0)
  for (int k = b0 + lane * 32; k < rows.cap && nb > 0; k += 32 * 32)
    asm volatile("prefetch.global.L2 [%0];" ::"l"(r + k));
}

struct RblArgs {
  PairParams pp;
  int n;
  const uint4* atoms;
  const double *x, *y, *z, *q;
  const int* type;
  const unsigned long long *key_a, *key_b;
  int epoch_arg;
  const int* epoch_dev;
  Rows rows;
  double *fx, *fy, *fz, *fpart;
};

// Block bx of a grid of gx blocks.  (The pointers are parameters, not copies
// of struct fields, so that their __restrict__ qualifiers hold.)
template <bool MIXED, int SEL, bool CUBIC>
__device__ __forceinline__ void rbl_fused_body(
    const PairParams& pp, int n, const uint4* __restrict__ atoms, const double* __restrict__ x,
    const double* __restrict__ y, const double* __restrict__ z, const double* __restrict__ q,
    const int* __restrict__ type, const unsigned long long* __restrict__ key_a,
    const unsigned long long* __restrict__ key_b, int epoch_arg,
    const int* __restrict__ epoch_dev, const Rows& rows, double* __restrict__ fx,
    double* __restrict__ fy, double* __restrict__ fz, double* __restrict__ fpart, int bx,
    int gx) {
  using T = typename std::conditional<MIXED, float, double>::type;
  const int epoch = epoch_dev ? *epoch_dev : epoch_arg;  // device copy inside a step graph
  __shared__ int s_q[PAIR_WARPS][RBL_QCAP];
  __shared__ double s_acc[PAIR_WARPS][3];
  const TypeTables tt = load_type_tables(pp, MIXED);
  const float* const f_eps = tt.f_eps;
  const float* const f_s6 = tt.f_s6;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt = lanemask_lt();
  const unsigned long long fmask = (unsigned long long)(pp.freq - 1);
  const float alpha_f = (float)pp.alpha, sqa_f = (float)pp.sqrt_alpha, qqr2e_f = (float)pp.qqr2e;
  const T freq_t = (T)pp.freq;
  double acc0 = 0, acc1 = 0, acc2 = 0;
  const int nt = pp.ntypes;
  const int wstride = gx * PAIR_WARPS;
  int* const wq = s_q[warp];
  for (int i = bx * PAIR_WARPS + warp; i < n; i += wstride) {
    const uint4 ai = atoms[i];
    const double xi = x[i], yi = y[i], zi = z[i];
    const T qi = MIXED ? (T)__uint_as_float(ai.w) : (T)q[i];
    const int ti = type[i];
    const unsigned long long ea = key_a[i] ^ (unsigned long long)(long long)epoch;
    // a row never holds more than cap entries; a larger count marks an
    // overflowed list (a rebuild inside a step graph), which the host replays
    int nf, nb;
    row_extent(rows, i, nf, nb);
    const int* row = rows.idx + (size_t)i * rows.cap;
    if (i + wstride < n) prefetch_row(rows, i + wstride, lane);
    int qn = 0;
    T fxa = 0, fya = 0, fza = 0;

    // force from queue slot `slot` (all 32 lanes take one pair each)
    auto pair_force = [&](int slot) {
      const int c = wq[slot];
      const int j = c & QF_INDEX;
      const int tj = __ldg(type + j);
      if (MIXED) {
        const uint4 aj = __ldg(atoms + j);  // exact wrapped fixed-point difference r_j - r_i
        const float ex = (float)(int)(aj.x - ai.x), ey = (float)(int)(aj.y - ai.y),
                    ez = (float)(int)(aj.z - ai.z);
        const float vx = ex * pp.sf[0], vy = ey * pp.sf[1], vz = ez * pp.sf[2];
        const float d2 = fmaf(vx, vx, fmaf(vy, vy, vz * vz));
        bool ok = true;
        if (c & QF_CHECK) {  // far pair: inside the shell window this step?
          const float d2s =
              CUBIC ? fmaf(ex, ex, fmaf(ey, ey, ez * ez))
                    : fmaf(ex * pp.sw[0], ex * pp.sw[0],
                           fmaf(ey * pp.sw[1], ey * pp.sw[1], (ez * pp.sw[2]) * (ez * pp.sw[2])));
          bool unsure;
          ok = classify_screen(pp, d2s, &unsure).shell_window;
          if (unsure) ok = classify_exact(exact_d2(pp, x, y, z, i, j), pp).shell_window;
        }
        const float qq = (float)qi * __uint_as_float(aj.w);
        float f = lj_f32_fast(f_eps[ti * nt + tj], f_s6[ti * nt + tj], d2);
        if (qq != 0.f) f += coul_f32(alpha_f, sqa_f, qqr2e_f, qq, d2);
        if (c < 0) f *= (float)freq_t;
        f = ok ? f : 0.f;
        fxa += (T)(f * vx);
        fya += (T)(f * vy);
        fza += (T)(f * vz);
      } else {
        // i minus j with the single-shift minimum image and no FMA: the
        // list predicate's own r^2 (CaculateDistance), so the window test of a
        // far pair is exact; the force takes r_j - r_i = -(dx, dy, dz)
        const double dx = min_image1(__dsub_rn(xi, __ldg(x + j)), pp.box.len[0], pp.box.half[0]);
        const double dy = min_image1(__dsub_rn(yi, __ldg(y + j)), pp.box.len[1], pp.box.half[1]);
        const double dz = min_image1(__dsub_rn(zi, __ldg(z + j)), pp.box.len[2], pp.box.half[2]);
        const double d2 =
            __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
        const bool ok = !(c & QF_CHECK) || classify_exact(d2, pp).shell_window;
        const double qq = (double)qi * __ldg(q + j);
        double f = lj_f64(tt.eps[ti * nt + tj], tt.s6[ti * nt + tj], d2);
        if (qq != 0.0) f += coul_f64(pp.alpha, pp.sqrt_alpha, pp.qqr2e, qq, d2);
        if (c < 0) f *= (double)freq_t;
        f = ok ? f : 0.0;
        fxa -= (T)(f * dx);
        fya -= (T)(f * dy);
        fza -= (T)(f * dz);
      }
    };
    auto drain_full = [&]() {
      __syncwarp();
      while (qn >= 32) {  // full batches from the tail of the queue
        qn -= 32;
        pair_force(qn + lane);
      }
      __syncwarp();
    };

    // near segment: full classification
    for (int k0 = 0; k0 < nf; k0 += 32 * RBL_NEAR_U) {
      int jj[RBL_NEAR_U];
      uint4 aa[RBL_NEAR_U];
      unsigned long long kb[RBL_NEAR_U];
#pragma unroll
      for (int u = 0; u < RBL_NEAR_U; ++u) {
        const int k = k0 + u * 32 + lane;
        jj[u] = k < nf ? __ldg(row + k) : i;
      }
#pragma unroll
      for (int u = 0; u < RBL_NEAR_U; ++u) {
        aa[u] = __ldg(atoms + jj[u]);
        kb[u] = __ldg(key_b + jj[u]);
      }
      unsigned core_bits = 0, shell_bits = 0, sel_bits = 0, unsure_bits = 0;
#pragma unroll
      for (int u = 0; u < RBL_NEAR_U; ++u) {
        const bool valid = jj[u] != i;
        bool unsure;
        const Classified c = classify_screen(
            pp, CUBIC ? fixed_d2(ai, aa[u]) : fixed_d2_weighted(pp, ai, aa[u]), &unsure);
        const bool sel = batch_selected<SEL>(ea ^ kb[u], fmask, pp.div);
        core_bits |= (unsigned)(valid && c.core_active) << u;
        shell_bits |= (unsigned)(valid && c.shell_window) << u;
        sel_bits |= (unsigned)sel << u;
        unsure_bits |= (unsigned)(valid && unsure) << u;
      }
      if (__any_sync(0xffffffffu, unsure_bits != 0)) {  // rare: FP64 predicate decides
#pragma unroll
        for (int u = 0; u < RBL_NEAR_U; ++u) {
          if (unsure_bits & (1u << u)) {
            const Classified c = classify_exact(exact_d2(pp, x, y, z, i, jj[u]), pp);
            core_bits = (core_bits & ~(1u << u)) | ((unsigned)c.core_active << u);
            shell_bits = (shell_bits & ~(1u << u)) | ((unsigned)c.shell_window << u);
          }
        }
      }
      const unsigned push_bits = core_bits | (shell_bits & sel_bits);
#pragma unroll
      for (int u = 0; u < RBL_NEAR_U; ++u) {
        const bool push = (push_bits >> u) & 1u;
        const unsigned m = __ballot_sync(0xffffffffu, push);
        if (push) wq[qn + __popc(m & lt)] = ((core_bits >> u) & 1u) ? jj[u] : (jj[u] | QF_SHELL);
        qn += __popc(m);
      }
      drain_full();
    }

    // far segment: batch hash first; selected pairs are queued with the
    // window test still to do.  The segment is read from the 16-byte boundary
    // at or below its start, four entries a lane (one 128-entry batch per
    // warp load); entries before the segment start are skipped.
    {
      const int fs = rows.cap - nb;  // first far entry
      const int fb = fs & ~3;        // rows start on 128-byte lines (cap % 32 == 0)
      const int4* f4 = reinterpret_cast<const int4*>(row + fb);
      for (int k0 = 0; fb + k0 < rows.cap; k0 += 128) {
        const int p0 = fb + k0 + 4 * lane;  // row position of this lane's first entry
        int4 e = make_int4(i, i, i, i);
        if (p0 < rows.cap) e = __ldg(f4 + (k0 >> 2) + lane);
        const int jj[4] = {p0 >= fs ? e.x : i, p0 + 1 >= fs ? e.y : i, p0 + 2 >= fs ? e.z : i,
                           p0 + 3 >= fs ? e.w : i};
        unsigned long long kb[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) kb[u] = __ldg(key_b + jj[u]);
        unsigned sb = 0;
#pragma unroll
        for (int u = 0; u < 4; ++u)
          sb |= (unsigned)((jj[u] != i) & batch_selected<SEL>(ea ^ kb[u], fmask, pp.div)) << u;
        // queue slots: exclusive prefix over lanes of the per-lane counts (0..4)
        const unsigned c = __popc(sb);
        const unsigned b0 = __ballot_sync(0xffffffffu, c & 1u),
                       b1 = __ballot_sync(0xffffffffu, c & 2u),
                       b2 = __ballot_sync(0xffffffffu, c & 4u);
        int pos = qn + __popc(b0 & lt) + 2 * __popc(b1 & lt) + 4 * __popc(b2 & lt);
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if ((sb >> u) & 1u) wq[pos++] = jj[u] | QF_SHELL | QF_CHECK;
        qn += __popc(b0) + 2 * __popc(b1) + 4 * __popc(b2);
        drain_full();
      }
    }
    if (lane < qn) pair_force(lane);
    __syncwarp();
    const double gx = warp_sum((double)fxa), gy = warp_sum((double)fya),
                 gz = warp_sum((double)fza);
    if (lane == 0) {
      fx[i] = gx;
      fy[i] = gy;
      fz[i] = gz;
      acc0 += gx;
      acc1 += gy;
      acc2 += gz;
    }
  }
  if (lane == 0) {
    s_acc[warp][0] = acc0;
    s_acc[warp][1] = acc1;
    s_acc[warp][2] = acc2;
  }
  if (fpart) write_block_partial(s_acc, fpart, bx);
}

template <bool MIXED, int SEL, bool CUBIC>
__global__ void __launch_bounds__(PAIR_BLOCK, MIXED ? 4 : 3)  // no spills in either form
k_rbl_fused(PairParams pp, int n, const uint4* __restrict__ atoms, const double* __restrict__ x,
            const double* __restrict__ y, const double* __restrict__ z,
            const double* __restrict__ q, const int* __restrict__ type,
            const unsigned long long* __restrict__ key_a,
            const unsigned long long* __restrict__ key_b, int epoch_arg,
            const int* __restrict__ epoch_dev, Rows rows, double* __restrict__ fx,
            double* __restrict__ fy, double* __restrict__ fz, double* __restrict__ fpart) {
  rbl_fused_body<MIXED, SEL, CUBIC>(pp, n, atoms, x, y, z, q, type, key_a, key_b, epoch_arg,
                                    epoch_dev, rows, fx, fy, fz, fpart, blockIdx.x, gridDim.x);
}

// The batched form holds its replica's pointers in registers (the single
// form reads them from the constant bank): one resident block fewer, no spills.
template <bool MIXED, int SEL, bool CUBIC>
__global__ void __launch_bounds__(PAIR_BLOCK, MIXED ? 3 : 2)
k_rbl_fused_batch(const RblArgs* __restrict__ a, const int* __restrict__ start, int nrep) {
  // the replica's arguments in shared memory: read where used, not held in registers
  static_assert(sizeof(RblArgs) % 4 == 0 && sizeof(RblArgs) <= 4 * PAIR_BLOCK, "RblArgs size");
  __shared__ __align__(16) RblArgs s_a;
  const int r = batch_replica(start, nrep, blockIdx.x);
  const int b0 = __ldg(start + r);
  if (threadIdx.x < sizeof(RblArgs) / 4)
    reinterpret_cast<int*>(&s_a)[threadIdx.x] =
        __ldg(reinterpret_cast<const int*>(a + r) + threadIdx.x);
  __syncthreads();
  rbl_fused_body<MIXED, SEL, CUBIC>(s_a.pp, s_a.n, s_a.atoms, s_a.x, s_a.y, s_a.z, s_a.q,
                                    s_a.type, s_a.key_a, s_a.key_b, s_a.epoch_arg, s_a.epoch_dev,
                                    s_a.rows, s_a.fx, s_a.fy, s_a.fz, s_a.fpart, blockIdx.x - b0,
                                    __ldg(start + r + 1) - b0);
}

// ---------------------------------------------------------------------------
// Verlet fused FP64: LJ + erfc-Coulomb for r^2 < cut_off^2 over the candidate
// list (ComputeLJCutCoulForce, lj_cut_coul_kspace_op.hip.cu:256-356), with
// per-block energy and virial partials epart[block][8] =
// {evdwl, ecoul, vxx, vyy, vzz, vxy, vxz, vyz} (ComputeVirial, lj_op.hip.cu:76-88).
// The cutoff test uses the integer screen with the FP64 fallback.
// ---------------------------------------------------------------------------
template <bool CUBIC>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_verlet_fused_f64(PairParams pp, int n, const uint4* __restrict__ atoms,
                   const double* __restrict__ x, const double* __restrict__ y,
                   const double* __restrict__ z, const double* __restrict__ q,
                   const int* __restrict__ type, Rows rows, double* __restrict__ fx,
                   double* __restrict__ fy, double* __restrict__ fz, double* __restrict__ fpart,
                   double* __restrict__ epart) {
  __shared__ struct {
    double dx[PAIR_WARPS][QCAP], dy[PAIR_WARPS][QCAP], dz[PAIR_WARPS][QCAP];
    int j[PAIR_WARPS][QCAP];
  } qu;
  __shared__ double s_acc[PAIR_WARPS][3];
  __shared__ double s_e[PAIR_WARPS][8];
  const TypeTables tt = load_type_tables(pp, false);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt = lanemask_lt();
  double acc0 = 0, acc1 = 0, acc2 = 0;
  double eacc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int nt = pp.ntypes;
  for (int i = blockIdx.x * PAIR_WARPS + warp; i < n; i += gridDim.x * PAIR_WARPS) {
    const uint4 ai = atoms[i];
    const double xi = x[i], yi = y[i], zi = z[i], qi = q[i];
    const int ti = type[i];
    int nf, nb;
    row_extent(rows, i, nf, nb);
    const int cnt = nf + nb;
    const int* row = rows.idx + (size_t)i * rows.cap;
    int qn = 0;
    double fxa = 0, fya = 0, fza = 0;
    double ea[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int k0 = 0;;) {
      const bool more = k0 < cnt;
      if (more) {
        bool push = false;
        int j = 0;
        const int k = k0 + lane;
        if (k < cnt) {
          j = row_at(row, rows.cap, nf, nb, k);
          if (j != i) {
            const uint4 aj = __ldg(atoms + j);
            const float d2s = CUBIC ? fixed_d2(ai, aj) : fixed_d2_weighted(pp, ai, aj);
            int in = d2s < pp.sc_rc.lo ? 1 : (d2s >= pp.sc_rc.hi ? 0 : -1);
            if (in < 0) {
              const double ex = min_image1(__ldg(x + j) - xi, pp.box.len[0], pp.box.half[0]);
              const double ey = min_image1(__ldg(y + j) - yi, pp.box.len[1], pp.box.half[1]);
              const double ez = min_image1(__ldg(z + j) - zi, pp.box.len[2], pp.box.half[2]);
              in = __dadd_rn(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)), __dmul_rn(ez, ez)) <
                   pp.rc2;
            }
            push = in;
          }
        }
        const unsigned m = __ballot_sync(0xffffffffu, push);
        if (push) {
          const int pos = qn + __popc(m & lt);
          qu.dx[warp][pos] = min_image1(__ldg(x + j) - xi, pp.box.len[0], pp.box.half[0]);
          qu.dy[warp][pos] = min_image1(__ldg(y + j) - yi, pp.box.len[1], pp.box.half[1]);
          qu.dz[warp][pos] = min_image1(__ldg(z + j) - zi, pp.box.len[2], pp.box.half[2]);
          qu.j[warp][pos] = j;
        }
        qn += __popc(m);
        k0 += 32;
        __syncwarp();
      }
      while (qn >= 32 || (!more && qn > 0)) {
        if (lane < qn) {
          const int j = qu.j[warp][lane];
          const double ddx = qu.dx[warp][lane], ddy = qu.dy[warp][lane], ddz = qu.dz[warp][lane];
          const double d2 = ddx * ddx + ddy * ddy + ddz * ddz;
          const int tj = __ldg(type + j);
          const double qq = qi * __ldg(q + j);
          const double e_ij = tt.eps[ti * nt + tj], s6 = tt.s6[ti * nt + tj];
          const double d6 = d2 * d2 * d2;
          const double sd6 = s6 / d6;
          double f = -24.0 * e_ij * ((2.0 * sd6 - 1.0) * sd6) / d2;
          ea[0] += 0.5 * (4.0 * e_ij * (s6 / d6 - 1.0) * sd6);
          if (qq != 0.0) {
            const double dis = sqrt(d2);
            const double ec = erfc(pp.sqrt_alpha * dis);
            const double g = ec / d2 + 2.0 * pp.sqrt_alpha * exp(-pp.alpha * d2) /
                                           (1.7724538509055160273 * dis);
            f += -pp.qqr2e * qq * g / dis;
            ea[1] += pp.qqr2e * (0.5 * qq * ec / dis);
          }
          fxa += f * ddx;
          fya += f * ddy;
          fza += f * ddz;
          ea[2] += -0.5 * ddx * ddx * f;
          ea[3] += -0.5 * ddy * ddy * f;
          ea[4] += -0.5 * ddz * ddz * f;
          ea[5] += -0.5 * ddx * ddy * f;
          ea[6] += -0.5 * ddx * ddz * f;
          ea[7] += -0.5 * ddy * ddz * f;
        }
        __syncwarp();
        const int rem = qn > 32 ? qn - 32 : 0;
        if (lane < rem) {
          qu.dx[warp][lane] = qu.dx[warp][32 + lane];
          qu.dy[warp][lane] = qu.dy[warp][32 + lane];
          qu.dz[warp][lane] = qu.dz[warp][32 + lane];
          qu.j[warp][lane] = qu.j[warp][32 + lane];
        }
        __syncwarp();
        qn = rem;
      }
      if (!more) break;
    }
    fxa = warp_sum(fxa);
    fya = warp_sum(fya);
    fza = warp_sum(fza);
#pragma unroll
    for (int c = 0; c < 8; ++c) ea[c] = warp_sum(ea[c]);
    if (lane == 0) {
      fx[i] = fxa;
      fy[i] = fya;
      fz[i] = fza;
      acc0 += fxa;
      acc1 += fya;
      acc2 += fza;
#pragma unroll
      for (int c = 0; c < 8; ++c) eacc[c] += ea[c];
    }
  }
  if (lane == 0) {
    s_acc[warp][0] = acc0;
    s_acc[warp][1] = acc1;
    s_acc[warp][2] = acc2;
    for (int c = 0; c < 8; ++c) s_e[warp][c] = eacc[c];
  }
  if (fpart) write_block_partial(s_acc, fpart);
  if (epart) {
    __syncthreads();
    if (threadIdx.x < 8) {
      double s = 0.0;
      for (int w = 0; w < PAIR_WARPS; ++w) s += s_e[w][threadIdx.x];
      epart[(size_t)blockIdx.x * 8 + threadIdx.x] = s;
    }
  }
}

// ---------------------------------------------------------------------------
// RBL list emitter (same classification as the fused kernels; rows of cap):
// core = list predicate r^2 < r_core^2 - EPS; shell = hashed
// r_core^2 - EPS <= r^2 < cut_off^2 - EPS.  Thread per atom: parity checks and
// the engine's list export, not the per-step path.
// ---------------------------------------------------------------------------
__global__ void k_rbl_lists(PairParams pp, int n, const uint4* __restrict__ atoms,
                            const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z,
                            const unsigned long long* __restrict__ key_a,
                            const unsigned long long* __restrict__ key_b, int epoch, Rows rows,
                            int* __restrict__ core_count, int* __restrict__ core,
                            int* __restrict__ shell_count, int* __restrict__ shell) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long ea = key_a[i] ^ (unsigned long long)(long long)epoch;
  int nc = 0, ns = 0;
  int nf, nb;
  row_extent(rows, i, nf, nb);
  const int cap = rows.cap;
  const int* row = rows.idx + (size_t)i * cap;
  for (int t = 0; t < nf + nb; ++t) {
    const int j = row_at(row, cap, nf, nb, t);
    if (j == i) continue;
    const double d2 = exact_d2(pp, x, y, z, i, j);
    if (d2 < pp.core2_list)
      core[(size_t)i * cap + nc++] = j;
    else if (d2 < pp.force2_list && rbl_selected(ea, key_b[j], pp.div))
      shell[(size_t)i * cap + ns++] = j;
  }
  core_count[i] = nc;
  shell_count[i] = ns;
}

__global__ void k_rbl_keys(int n, const int* __restrict__ gid, unsigned long long* __restrict__ a,
                           unsigned long long* __restrict__ b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  a[i] = rbl_key_a(gid[i]);
  b[i] = rbl_key_b(gid[i]);
}

// ---------------------------------------------------------------------------
// Drop-in ops with the reference data layouts.
// ---------------------------------------------------------------------------
// The drop-in ops take the reference's rbmd::Real (T): double under
// ENABLE_DOUBLE, float in the default build.  Every membership test (list
// predicates, force windows) is evaluated in T with the reference's own
// expression, so a pair is kept or dropped exactly as the reference build of
// the same precision keeps or drops it; force values are then computed in
// FP64 from the T inputs.
//
// Single-shift minimum image of MinImageDistance (box.h:51-73): the half-edge
// test compares against box._length * 0.5, which C++ evaluates in double.
template <typename T>
__device__ __forceinline__ T ref_min_image(T d, T len) {
  if (fabs((double)d) > (double)len * 0.5) d -= (d > 0 ? len : -len);
  return d;
}
// CaculateDistance (full_neighbor_list_op.h:98-106): i minus j, the squares
// by POW and summed left to right.  In double POW(d, 2) is the product d * d.
__device__ __forceinline__ double ref_list_d2(double dx, double dy, double dz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}
__device__ __forceinline__ float ref_list_d2(float dx, float dy, float dz) {
  return __fadd_rn(__fadd_rn(powf(dx, 2.f), powf(dy, 2.f)), powf(dz, 2.f));
}
template <typename T>
struct RefLen {
  T len[3];
};
template <typename T>
RefLen<T> ref_len(const DBox& b) {
  RefLen<T> r;
  for (int d = 0; d < 3; ++d) r.len[d] = (T)b.len[d];
  return r;
}

// FilterRBLNeighborCandidates semantics (rbl_full_neighbor_list_op.hip.cu:237-304).
template <typename T>
__global__ void k_ref_rbl_filter(T core2, T force2, int n, const int* __restrict__ gid,
                                 const T* __restrict__ x, const T* __restrict__ y,
                                 const T* __restrict__ z, const int* __restrict__ cstart,
                                 const int* __restrict__ cend, const int* __restrict__ cand,
                                 const int* __restrict__ core_cap,
                                 const int* __restrict__ core_start, int* __restrict__ core_end,
                                 int* __restrict__ core, int shell_cap, int* __restrict__ shell,
                                 int* __restrict__ shell_num, int* __restrict__ required,
                                 RefLen<T> b, int* __restrict__ realloc, DivTest div, int epoch) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long ea = rbl_key_a(gid[i]) ^ (unsigned long long)(long long)epoch;
  int nc = 0, ns = 0;
  const int out0 = core_start[i], ccap = core_cap[i];
  const T xi = x[i], yi = y[i], zi = z[i];
  for (int pos = cstart[i]; pos < cend[i]; ++pos) {
    const int j = cand[pos];
    if (j == i) continue;
    const T d2 = ref_list_d2(ref_min_image<T>(xi - x[j], b.len[0]),
                             ref_min_image<T>(yi - y[j], b.len[1]),
                             ref_min_image<T>(zi - z[j], b.len[2]));
    if (d2 < core2) {
      if (nc < ccap)
        core[out0 + nc] = j;
      else
        atomicOr(realloc, 1);
      ++nc;
    } else if (d2 < force2 && rbl_selected(ea, rbl_key_b(gid[j]), div)) {
      if (ns < shell_cap) shell[(size_t)ns * n + i] = j;
      ++ns;
    }
  }
  core_end[i] = out0 + (nc < ccap ? nc : ccap);
  shell_num[i] = ns < shell_cap ? ns : shell_cap;
  atomicMax(required, ns);
}

// Pair vector r_j - r_i in T with the minimum image, and its r^2 as the
// reference's force helpers form it (lj_op.hip.cu:40-54).
template <typename T>
struct RefPair {
  T dx, dy, dz, d2;
};
template <typename T>
__device__ __forceinline__ RefPair<T> ref_pair(const RefLen<T>& b, T xi, T yi, T zi, T xj, T yj,
                                               T zj) {
  RefPair<T> p;
  p.dx = ref_min_image<T>(xj - xi, b.len[0]);
  p.dy = ref_min_image<T>(yj - yi, b.len[1]);
  p.dz = ref_min_image<T>(zj - zi, b.len[2]);
  p.d2 = p.dx * p.dx + p.dy * p.dy + p.dz * p.dz;
  return p;
}

// LJCutCoulRBLForce semantics, warp per atom over core CSR + sample-major shell.
template <typename T>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_ref_pair_rbl(RefLen<T> b, T rs, T rc, int n, int pice, double alpha, double sqa, double qqr2e,
               const int* __restrict__ type, const T* __restrict__ sigma,
               const T* __restrict__ eps, const int* __restrict__ start,
               const int* __restrict__ end, const int* __restrict__ core,
               const int* __restrict__ shell, const int* __restrict__ shell_num,
               const T* __restrict__ q, const T* __restrict__ x, const T* __restrict__ y,
               const T* __restrict__ z, T* __restrict__ fx, T* __restrict__ fy,
               T* __restrict__ fz) {
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * PAIR_WARPS + (threadIdx.x >> 5);
  if (i >= n) return;
  const T rs2 = rs * rs, rc2 = rc * rc, eps_t = (T)RBX_EPSILON;
  const int ti = type[i];
  const T xi = x[i], yi = y[i], zi = z[i];
  const double qi = q[i], si = sigma[ti], ei = eps[ti];
  double s[3] = {0, 0, 0}, c[3] = {0, 0, 0};
  const int a = start[i], e = end[i], ns = shell_num[i];
  for (int t = a + lane; t < e; t += 32) {
    const int j = core[t];
    const RefPair<T> p = ref_pair<T>(b, xi, yi, zi, x[j], y[j], z[j]);
    if (p.d2 < rs2 && p.d2 > eps_t) {
      const double dx = p.dx, dy = p.dy, dz = p.dz, d2 = dx * dx + dy * dy + dz * dz;
      const double sij = (si + (double)sigma[type[j]]) / 2, eij = sqrt(ei * (double)eps[type[j]]);
      double f = lj_f64(eij, pow(sij, 6.0), d2);
      const double qq = qi * (double)q[j];
      if (qq != 0.0) f += coul_f64(alpha, sqa, qqr2e, qq, d2);
      s[0] += f * dx;
      s[1] += f * dy;
      s[2] += f * dz;
    }
  }
  for (int t = lane; t < ns; t += 32) {
    const int j = shell[(size_t)t * n + i];
    const RefPair<T> p = ref_pair<T>(b, xi, yi, zi, x[j], y[j], z[j]);
    if (p.d2 < rc2 && p.d2 > rs2) {
      const double dx = p.dx, dy = p.dy, dz = p.dz, d2 = dx * dx + dy * dy + dz * dz;
      const double sij = (si + (double)sigma[type[j]]) / 2, eij = sqrt(ei * (double)eps[type[j]]);
      double f = lj_f64(eij, pow(sij, 6.0), d2);
      const double qq = qi * (double)q[j];
      if (qq != 0.0) f += coul_f64(alpha, sqa, qqr2e, qq, d2);
      f *= (double)pice;
      c[0] += f * dx;
      c[1] += f * dy;
      c[2] += f * dz;
    }
  }
  for (int d = 0; d < 3; ++d) {
    s[d] = warp_sum(s[d]);
    c[d] = warp_sum(c[d]);
  }
  if (lane == 0) {
    fx[i] = (T)(s[0] + c[0]);
    fy[i] = (T)(s[1] + c[1]);
    fz[i] = (T)(s[2] + c[2]);
  }
}

// LJCutCoulForce semantics (Verlet), warp per atom, per-atom virial columns
// and per-atom energies epart[2*n] for a deterministic reduction.
template <typename T>
__global__ void __launch_bounds__(PAIR_BLOCK)
k_ref_pair_verlet(RefLen<T> b, T cut_off, int n, double alpha, double sqa, double qqr2e,
                  const int* __restrict__ type, const T* __restrict__ sigma,
                  const T* __restrict__ eps, const int* __restrict__ start,
                  const int* __restrict__ end, const int* __restrict__ nbrs,
                  const T* __restrict__ q, const T* __restrict__ x, const T* __restrict__ y,
                  const T* __restrict__ z, T* __restrict__ fx, T* __restrict__ fy,
                  T* __restrict__ fz, T* __restrict__ vir, double* __restrict__ epart) {
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * PAIR_WARPS + (threadIdx.x >> 5);
  if (i >= n) return;
  const T cut2 = cut_off * cut_off;
  const int ti = type[i];
  const T xi = x[i], yi = y[i], zi = z[i];
  const double qi = q[i];
  double a[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int t = start[i] + lane; t < end[i]; t += 32) {
    const int j = nbrs[t];
    const RefPair<T> p = ref_pair<T>(b, xi, yi, zi, x[j], y[j], z[j]);
    if (!(p.d2 < cut2)) continue;
    const double dx = p.dx, dy = p.dy, dz = p.dz, d2 = dx * dx + dy * dy + dz * dz;
    const double sij = ((double)sigma[ti] + (double)sigma[type[j]]) / 2,
                 eij = sqrt((double)eps[ti] * (double)eps[type[j]]);
    const double s6 = pow(sij, 6.0), d6 = d2 * d2 * d2, sd6 = s6 / d6;
    double f = -24 * eij * ((2 * sd6 - 1) * sd6) / d2;
    a[3] += 0.5 * (4 * eij * (s6 / d6 - 1) * sd6);
    const double qq = qi * (double)q[j];
    if (qq != 0.0) {
      const double dis = sqrt(d2), ec = erfc(sqa * dis);
      f += -qqr2e * qq * (ec / d2 + 2 * sqa * exp(-alpha * d2) / (1.7724538509055160273 * dis)) / dis;
      a[4] += qqr2e * (0.5 * qq * ec / dis);
    }
    a[0] += f * dx;
    a[1] += f * dy;
    a[2] += f * dz;
    a[5] += -0.5 * dx * dx * f;
    a[6] += -0.5 * dy * dy * f;
    a[7] += -0.5 * dz * dz * f;
    a[8] += -0.5 * dx * dy * f;
    a[9] += -0.5 * dx * dz * f;
    a[10] += -0.5 * dy * dz * f;
  }
  for (int c = 0; c < 11; ++c) a[c] = warp_sum(a[c]);
  if (lane == 0) {
    fx[i] = (T)a[0];
    fy[i] = (T)a[1];
    fz[i] = (T)a[2];
    if (epart) {
      epart[i] = a[3];
      epart[(size_t)n + i] = a[4];
    }
    if (vir)
      for (int c = 0; c < 6; ++c) vir[(size_t)c * n + i] = (T)a[5 + c];
  }
}

// Deterministic column sums: out[c] = scale * sum_i cols[c*n + i] (one block per column).
template <typename T>
__global__ void k_reduce_cols(int n, const T* __restrict__ cols, double* __restrict__ out,
                              double scale) {
  __shared__ double sh[8];
  double s = 0.0;
  const T* col = cols + (size_t)blockIdx.x * n;
  for (int i = threadIdx.x; i < n; i += 256) s += col[i];
  s = block_sum_det<256>(s, sh);
  if (threadIdx.x == 0) out[blockIdx.x] = s * scale;
}

__global__ void k_sum_i32(int n, const int* __restrict__ src, long long* __restrict__ out) {
  long long s = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    s += src[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd((unsigned long long*)out, (unsigned long long)s);
}

template <typename T>
__global__ void k_sub_mean(int n, T* __restrict__ fx, T* __restrict__ fy, T* __restrict__ fz,
                           const double* __restrict__ mean) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  fx[i] = (T)((double)fx[i] - mean[0]);
  fy[i] = (T)((double)fy[i] - mean[1]);
  fz[i] = (T)((double)fz[i] - mean[2]);
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
#define RBX_TRY_K(expr)     \
  do {                      \
    const int _rc = (expr); \
    if (_rc) return _rc;    \
  } while (0)

IntScreen make_screen(double C, double L, double band) {
  // |d|^2 s^2 < C  <=>  |d|^2 < C / s^2, s = L / 2^32; band in r^2 units
  const double scale = 18446744073709551616.0 / (L * L);
  IntScreen t;
  t.lo = (float)((C - band) * scale);
  t.hi = (float)((C + band) * scale);
  return t;
}

int rbl_fused_blocks(int n) {
  // capacity of the per-block partial buffers: enough for rbl_fused_grid at up
  // to 16 waves of 8 resident blocks per SM, so a grid is never cut short of a
  // whole number of waves
  const int target = sm_count() * 8 * 16;
  int b = (n + PAIR_WARPS - 1) / PAIR_WARPS;
  if (b > target) b = target;
  return b < 1 ? 1 : b;
}

namespace {
using RblKernel = void (*)(PairParams, int, const uint4*, const double*, const double*,
                           const double*, const double*, const int*, const unsigned long long*,
                           const unsigned long long*, int, const int*, Rows, double*, double*,
                           double*, double*);
using RblBatchKernel = void (*)(const RblArgs*, const int*, int);

// The instantiation a launch uses: the batch test from freq, the unweighted
// distance screen on cubic boxes; variant = (mixed * 3 + sel) * 2 + cubic.
int rbl_variant(bool mixed, int freq, bool cubic) {
  const bool pow2 = freq >= 1 && (freq & (freq - 1)) == 0;
  const int sel = pow2 ? (freq <= 4 ? 2 : 1) : 0;
  return ((mixed ? 3 : 0) + sel) * 2 + (cubic ? 1 : 0);
}
RblKernel rbl_kernel(int v) {
  static RblKernel const table[12] = {
      k_rbl_fused<false, 0, false>, k_rbl_fused<false, 0, true>, k_rbl_fused<false, 1, false>,
      k_rbl_fused<false, 1, true>,  k_rbl_fused<false, 2, false>, k_rbl_fused<false, 2, true>,
      k_rbl_fused<true, 0, false>,  k_rbl_fused<true, 0, true>,  k_rbl_fused<true, 1, false>,
      k_rbl_fused<true, 1, true>,   k_rbl_fused<true, 2, false>, k_rbl_fused<true, 2, true>};
  return table[v];
}
RblBatchKernel rbl_batch_kernel(int v) {
  static RblBatchKernel const table[12] = {
      k_rbl_fused_batch<false, 0, false>, k_rbl_fused_batch<false, 0, true>,
      k_rbl_fused_batch<false, 1, false>, k_rbl_fused_batch<false, 1, true>,
      k_rbl_fused_batch<false, 2, false>, k_rbl_fused_batch<false, 2, true>,
      k_rbl_fused_batch<true, 0, false>,  k_rbl_fused_batch<true, 0, true>,
      k_rbl_fused_batch<true, 1, false>,  k_rbl_fused_batch<true, 1, true>,
      k_rbl_fused_batch<true, 2, false>,  k_rbl_fused_batch<true, 2, true>};
  return table[v];
}
RblKernel rbl_choose(bool mixed, int freq, bool cubic) {
  return rbl_kernel(rbl_variant(mixed, freq, cubic));
}
}  // namespace

int rbl_fused_grid(bool mixed, int freq, int n, int cap, int max_blocks, int waves, int ntypes) {
  // waves of resident blocks (default 8): with several waves the block
  // scheduler evens out the per-atom work
  (void)cap;
  const int kRblWaves = waves > 0 ? waves : 8;
  const RblKernel k = rbl_choose(mixed, freq, true);  // occupancy of the cubic form
  size_t smem = 0;
  int occ = 0;
  if (type_table_smem(k, ntypes, mixed, &smem) != RBX_OK ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, PAIR_BLOCK, smem) != cudaSuccess ||
      occ < 1) {
    cudaGetLastError();
    occ = 1;
  }
  int b = kRblWaves * occ * sm_count();
  const int need = (n + PAIR_WARPS - 1) / PAIR_WARPS;
  if (b > need) b = need;
  if (b > max_blocks) b = max_blocks;
  return b < 1 ? 1 : b;
}

int launch_rbl_fused(bool mixed, const PairParams& pp, int n, const uint4* atoms,
                     const double* x, const double* y, const double* z, const double* q,
                     const int* type, const unsigned long long* key_a,
                     const unsigned long long* key_b, int epoch, const int* epoch_dev,
                     const Rows& rows, double* fx, double* fy, double* fz, double* fpart,
                     int nblocks, cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  if (n > QF_INDEX) {
    set_error("rbl_fused: at most %d atoms", QF_INDEX);
    return RBX_ERR_INVALID;
  }
  const int v = rbl_variant(mixed, pp.freq, pp.cubic != 0);
  const RblKernel k = rbl_kernel(v);
  size_t smem = 0;
  RBX_TRY_K(type_table_smem(k, pp.ntypes, mixed, &smem));
  RblArgs a;
  a.pp = pp;
  a.n = n;
  a.atoms = atoms;
  a.x = x;
  a.y = y;
  a.z = z;
  a.q = q;
  a.type = type;
  a.key_a = key_a;
  a.key_b = key_b;
  a.epoch_arg = epoch;
  a.epoch_dev = epoch_dev;
  a.rows = rows;
  a.fx = fx;
  a.fy = fy;
  a.fz = fz;
  a.fpart = fpart;
  if (batch_recorder()) {
    RBX_TRY_K(type_table_smem(rbl_batch_kernel(v), pp.ntypes, mixed, &smem));
    return record_phase(PH_RBL, v, nblocks, PAIR_BLOCK, smem, &a, sizeof a);
  }
  k<<<nblocks, PAIR_BLOCK, smem, st>>>(pp, n, atoms, x, y, z, q, type, key_a, key_b, epoch,
                                    epoch_dev, rows, fx, fy, fz, fpart);
  count_launch();
  return check_launch(mixed ? "rbl_fused_mixed" : "rbl_fused_f64");
}

int launch_rbl_batch(int variant, const void* args, const int* start, int nrep, int total,
                     size_t smem, cudaStream_t st) {
  rbl_batch_kernel(variant)<<<total, PAIR_BLOCK, smem, st>>>(static_cast<const RblArgs*>(args),
                                                             start, nrep);
  count_launch();
  return check_launch("rbl_fused_batch");
}

int launch_verlet_fused_f64(const PairParams& pp, int n, const uint4* atoms, const double* x,
                            const double* y, const double* z, const double* q, const int* type,
                            const Rows& rows, double* fx, double* fy, double* fz, double* fpart,
                            double* epart, int nblocks, cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  size_t smem = 0;
  if (pp.cubic) {
    RBX_TRY_K(type_table_smem(k_verlet_fused_f64<true>, pp.ntypes, false, &smem));
    k_verlet_fused_f64<true><<<nblocks, PAIR_BLOCK, smem, st>>>(pp, n, atoms, x, y, z, q, type,
                                                                rows, fx, fy, fz, fpart, epart);
  } else {
    RBX_TRY_K(type_table_smem(k_verlet_fused_f64<false>, pp.ntypes, false, &smem));
    k_verlet_fused_f64<false><<<nblocks, PAIR_BLOCK, smem, st>>>(pp, n, atoms, x, y, z, q, type,
                                                                 rows, fx, fy, fz, fpart, epart);
  }
  count_launch();
  return check_launch("verlet_fused_f64");
}

int launch_rbl_lists(const PairParams& pp, int n, const uint4* atoms, const double* x,
                     const double* y, const double* z, const unsigned long long* key_a,
                     const unsigned long long* key_b, int epoch, const Rows& rows,
                     int* core_count, int* core, int* shell_count, int* shell,
                     cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_rbl_lists<<<(n + 127) / 128, 128, 0, st>>>(pp, n, atoms, x, y, z, key_a, key_b, epoch, rows,
                                               core_count, core, shell_count, shell);
  count_launch();
  return check_launch("rbl_lists");
}

int launch_rbl_keys(int n, const int* gid, unsigned long long* key_a, unsigned long long* key_b,
                    cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_rbl_keys<<<(n + 255) / 256, 256, 0, st>>>(n, gid, key_a, key_b);
  count_launch();
  return check_launch("rbl_keys");
}

template <typename T>
int launch_ref_rbl_filter_t(T core2, T force2, int n, const int* gid, const T* x, const T* y,
                            const T* z, const int* cstart, const int* cend, const int* cand,
                            const int* core_cap, const int* core_start, int* core_end, int* core,
                            int shell_cap, int* shell, int* shell_num, int* required,
                            const DBox& b, int* realloc, const DivTest& div, int epoch,
                            cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_ref_rbl_filter<T><<<(n + 127) / 128, 128, 0, st>>>(
      core2, force2, n, gid, x, y, z, cstart, cend, cand, core_cap, core_start, core_end, core,
      shell_cap, shell, shell_num, required, ref_len<T>(b), realloc, div, epoch);
  count_launch();
  return check_launch("ref_rbl_filter");
}
int launch_ref_rbl_filter(double core2, double force2, int n, const int* gid, const double* x,
                          const double* y, const double* z, const int* cstart, const int* cend,
                          const int* cand, const int* core_cap, const int* core_start,
                          int* core_end, int* core, int shell_cap, int* shell, int* shell_num,
                          int* required, const DBox& b, int* realloc, const DivTest& div,
                          int epoch, cudaStream_t st) {
  return launch_ref_rbl_filter_t<double>(core2, force2, n, gid, x, y, z, cstart, cend, cand,
                                         core_cap, core_start, core_end, core, shell_cap, shell,
                                         shell_num, required, b, realloc, div, epoch, st);
}
int launch_ref_rbl_filter(float core2, float force2, int n, const int* gid, const float* x,
                          const float* y, const float* z, const int* cstart, const int* cend,
                          const int* cand, const int* core_cap, const int* core_start,
                          int* core_end, int* core, int shell_cap, int* shell, int* shell_num,
                          int* required, const DBox& b, int* realloc, const DivTest& div,
                          int epoch, cudaStream_t st) {
  return launch_ref_rbl_filter_t<float>(core2, force2, n, gid, x, y, z, cstart, cend, cand,
                                        core_cap, core_start, core_end, core, shell_cap, shell,
                                        shell_num, required, b, realloc, div, epoch, st);
}

template <typename T>
int launch_ref_pair_rbl_t(const DBox& b, T rs, T rc, int n, int pice_num, double alpha,
                          double qqr2e, const int* type, const T* sigma, const T* eps,
                          const int* start, const int* end, const int* core, const int* shell,
                          const int* shell_num, const T* q, const T* x, const T* y, const T* z,
                          T* fx, T* fy, T* fz, cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_ref_pair_rbl<T><<<(n + PAIR_WARPS - 1) / PAIR_WARPS, PAIR_BLOCK, 0, st>>>(
      ref_len<T>(b), rs, rc, n, pice_num, alpha, sqrt(alpha), qqr2e, type, sigma, eps, start,
      end, core, shell, shell_num, q, x, y, z, fx, fy, fz);
  count_launch();
  return check_launch("ref_pair_rbl");
}
int launch_ref_pair_rbl(const DBox& b, double rs, double rc, int n, int pice_num, double alpha,
                        double qqr2e, const int* type, const double* sigma, const double* eps,
                        const int* start, const int* end, const int* core, const int* shell,
                        const int* shell_num, const double* q, const double* x, const double* y,
                        const double* z, double* fx, double* fy, double* fz, cudaStream_t st) {
  return launch_ref_pair_rbl_t<double>(b, rs, rc, n, pice_num, alpha, qqr2e, type, sigma, eps,
                                       start, end, core, shell, shell_num, q, x, y, z, fx, fy, fz,
                                       st);
}
int launch_ref_pair_rbl(const DBox& b, float rs, float rc, int n, int pice_num, double alpha,
                        double qqr2e, const int* type, const float* sigma, const float* eps,
                        const int* start, const int* end, const int* core, const int* shell,
                        const int* shell_num, const float* q, const float* x, const float* y,
                        const float* z, float* fx, float* fy, float* fz, cudaStream_t st) {
  return launch_ref_pair_rbl_t<float>(b, rs, rc, n, pice_num, alpha, qqr2e, type, sigma, eps,
                                      start, end, core, shell, shell_num, q, x, y, z, fx, fy, fz,
                                      st);
}

template <typename T>
int launch_ref_pair_verlet_t(const DBox& b, T cut_off, int n, double alpha, double qqr2e,
                             const int* type, const T* sigma, const T* eps, const int* start,
                             const int* end, const int* nbrs, const T* q, const T* x, const T* y,
                             const T* z, T* fx, T* fy, T* fz, T* flat_virial, double* epart,
                             cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_ref_pair_verlet<T><<<(n + PAIR_WARPS - 1) / PAIR_WARPS, PAIR_BLOCK, 0, st>>>(
      ref_len<T>(b), cut_off, n, alpha, sqrt(alpha), qqr2e, type, sigma, eps, start, end, nbrs,
      q, x, y, z, fx, fy, fz, flat_virial, epart);
  count_launch();
  return check_launch("ref_pair_verlet");
}
int launch_ref_pair_verlet(const DBox& b, double cut_off, int n, double alpha, double qqr2e,
                           const int* type, const double* sigma, const double* eps,
                           const int* start, const int* end, const int* nbrs, const double* q,
                           const double* x, const double* y, const double* z, double* fx,
                           double* fy, double* fz, double* flat_virial, double* epart,
                           cudaStream_t st) {
  return launch_ref_pair_verlet_t<double>(b, cut_off, n, alpha, qqr2e, type, sigma, eps, start,
                                          end, nbrs, q, x, y, z, fx, fy, fz, flat_virial, epart,
                                          st);
}
int launch_ref_pair_verlet(const DBox& b, float cut_off, int n, double alpha, double qqr2e,
                           const int* type, const float* sigma, const float* eps,
                           const int* start, const int* end, const int* nbrs, const float* q,
                           const float* x, const float* y, const float* z, float* fx,
                           float* fy, float* fz, float* flat_virial, double* epart,
                           cudaStream_t st) {
  return launch_ref_pair_verlet_t<float>(b, cut_off, n, alpha, qqr2e, type, sigma, eps, start,
                                         end, nbrs, q, x, y, z, fx, fy, fz, flat_virial, epart,
                                         st);
}

template <typename T>
int launch_reduce_cols_t(int n, int ncols, const T* cols, double* out, double scale,
                         cudaStream_t st) {
  if (ncols <= 0) return RBX_OK;
  k_reduce_cols<T><<<ncols, 256, 0, st>>>(n, cols, out, scale);
  count_launch();
  return check_launch("reduce_cols");
}
int launch_reduce_cols(int n, int ncols, const double* cols, double* out, double scale,
                       cudaStream_t st) {
  return launch_reduce_cols_t<double>(n, ncols, cols, out, scale, st);
}
int launch_reduce_cols(int n, int ncols, const float* cols, double* out, double scale,
                       cudaStream_t st) {
  return launch_reduce_cols_t<float>(n, ncols, cols, out, scale, st);
}
int launch_sum_i32(int n, const int* src, long long* out, cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_sum_i32<<<grid_for(n, 256, sm_count() * 4), 256, 0, st>>>(n, src, out);
  count_launch();
  return check_launch("sum_i32");
}

template <typename T>
int launch_sub_mean_t(int n, T* fx, T* fy, T* fz, const double* mean, cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_sub_mean<T><<<(n + 255) / 256, 256, 0, st>>>(n, fx, fy, fz, mean);
  count_launch();
  return check_launch("sub_mean");
}
int launch_sub_mean(int n, double* fx, double* fy, double* fz, const double* mean,
                    cudaStream_t st) {
  return launch_sub_mean_t<double>(n, fx, fy, fz, mean, st);
}
int launch_sub_mean(int n, float* fx, float* fy, float* fz, const double* mean,
                    cudaStream_t st) {
  return launch_sub_mean_t<float>(n, fx, fy, fz, mean, st);
}

}  // namespace rbx
