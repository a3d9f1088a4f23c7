// rbx_rbsog.cu -- RBSOG k-space (random-batch sum of Gaussians) and the
// VERLET-SOG real-space pair force.
//
// RBMD's ComputeRBSOG (src/force/src/kspace_calculator.cpp:1331-1543) sums
// the far-field Gaussians over P sampled k-vectors, drawn from
// p(m) ~ G^(m) |k|^2 on |m|^2 > 1 with G^(m) = sum_l coef_l exp(-b^(2l)
// sigma^2 |k|^2 / 2), plus the six |m| = 1 vectors directly:
//   F_i = q_i sum_k c_k (cos(k.r_i) Im rho_k - sin(k.r_i) Re rho_k) k,
//   c_k = -(S / P) qqr2e / (V |k|^2)  (sampled),  -qqr2e G^(k) / V  (direct),
// (ComputeRBSOGSampleForceKernel :955-1012, ComputeRBSOGDirectForceKernel
// :1224-1277), energy (S / (2 P V)) qqr2e |rho|^2 / |k|^2 and
// qqr2e G^(k) |rho|^2 / (2 V) plus the self term.  The structure factor and
// the force scatter are the RBE kernels (rbx_rbe.cu) over P + 6 vectors; this
// file adds the sampler, the per-k coefficients and the energy sum.
//
// The reference samples with a Metropolis chain on the host (RBSOGSampleKSpace,
// :1142-1329).  Here the density is sampled exactly on the device: since
// |k|^2 = sum_d k_d^2 and each Gaussian factorises over the axes,
// G^(m)|k|^2 = sum_(l,d) coef_l k_d^2 g_l(m_d) prod_(d' != d) g_l(m_d'), a
// mixture of separable densities; a Philox draw picks the component (l, d)
// from its weight, then one inverse-CDF draw per axis, and |m|^2 <= 1 is
// rejected.  Same stationary density, independent draws, deterministic per
// (seed, step, sample).
#include <math.h>

#include "rbx_common.cuh"
#include "rbx_kernels.h"
#include "rbx_pair_device.cuh"

namespace rbx {

namespace {
constexpr int SOG_SAMPLE_BLOCK = 128;
constexpr int SOG_FK_BLOCK = 128;
constexpr int SOG_PAIR_BLOCK = 128;

// first index t with target < cdf[t] (cdf ascending), else cnt - 1
__device__ __forceinline__ int cdf_search(const double* cdf, int cnt, double target) {
  int lo = 0, hi = cnt - 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (target < cdf[mid])
      hi = mid;
    else
      lo = mid + 1;
  }
  return lo;
}

__device__ __forceinline__ double u53(uint32_t hi, uint32_t lo) {
  return (double)(((((uint64_t)hi) << 32) | lo) >> 11) * (1.0 / 9007199254740992.0);
}

__global__ void __launch_bounds__(SOG_SAMPLE_BLOCK)
k_rbsog_sample(int p, RbsogTables t, uint32_t key0, uint32_t key1, uint64_t step_arg,
               const int* __restrict__ step_dev, double* __restrict__ mx, double* __restrict__ my,
               double* __restrict__ mz, int* __restrict__ mi, int* __restrict__ status) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= p) return;
  const uint64_t step = step_dev ? (uint64_t)(int64_t)*step_dev : step_arg;
  for (int a = 0; a < 64; ++a) {
    uint32_t c[4] = {(uint32_t)s, (uint32_t)(2 * a), (uint32_t)step, (uint32_t)(step >> 32)};
    philox4x32_10(c, key0, key1);
    uint32_t d[4] = {(uint32_t)s, (uint32_t)(2 * a + 1), (uint32_t)step, (uint32_t)(step >> 32)};
    philox4x32_10(d, key0, key1);
    const int comp = cdf_search(t.comp_cdf, t.ncomp, u53(c[0], c[1]) * t.comp_tot);
    const int l = comp / 3, dd = comp - 3 * l;
    const double u[3] = {u53(c[2], c[3]), u53(d[0], d[1]), u53(d[2], d[3])};
    int m[3];
    for (int ax = 0; ax < 3; ++ax) {
      const int ti = (l * 3 + ax) * 2 + (ax == dd ? 1 : 0);
      const int e = cdf_search(t.tables + t.off[ti], t.cnt[ti], u[ax] * t.tot[ti]);
      m[ax] = e == 0 ? 0 : ((e & 1) ? (e + 1) / 2 : -(e / 2));
    }
    if (m[0] * m[0] + m[1] * m[1] + m[2] * m[2] > 1) {
      mx[s] = m[0];
      my[s] = m[1];
      mz[s] = m[2];
      if (mi) {
        mi[3 * s] = m[0];
        mi[3 * s + 1] = m[1];
        mi[3 * s + 2] = m[2];
      }
      return;
    }
  }
  atomicOr(status, 1);
}

// G^(k) = sum_l coef_l exp(-b^(2l) sigma^2 |k|^2 / 2) (KSpaceCalculator::Gaussian
// and Gaussian_modify, kspace_calculator.cpp:1559-1590).
__device__ double sog_ghat(const double* __restrict__ coef, int mmax, double b2, double sig2,
                           double k2) {
  double sum = 0.0, bl = 1.0;
  for (int l = 0; l < mmax; ++l) {
    sum += coef[l] * exp(-(bl * sig2) * k2 / 2.0);
    bl *= b2;
  }
  return sum;
}

constexpr int SOG_CHAIN_BLOCK = 256;
constexpr int SOG_CHAIN_CHUNK = 1024;
constexpr uint32_t SOG_NPT_STREAM = 0x4e505400u;  // Philox counter word of the NPT uniforms

// The NPT gather chain (RBSOGSampleKSpace, kspace_calculator.cpp:1242-1301):
// an independence Metropolis chain over the samples themselves, with target
// G_npt(m) |k|^4 and proposal density G(m) |k|^2 (the density the samples
// follow).  Chunks of 1024 samples: every thread forms ratios and uniforms
// into shared memory, then thread 0 walks the chunk.  Accepting i when
// u_i r_cur < r_i is u_i < min(1, r_i / r_cur) without the division.
__global__ void __launch_bounds__(SOG_CHAIN_BLOCK)
k_rbsog_npt_chain(int p, const double* __restrict__ mx, const double* __restrict__ my,
                  const double* __restrict__ mz, double Lx, double Ly, double Lz, SogGauss g,
                  uint32_t key0, uint32_t key1, uint64_t step_arg, const int* __restrict__ step_dev,
                  int* __restrict__ idx, int* __restrict__ mult) {
  __shared__ double s_r[SOG_CHAIN_CHUNK], s_u[SOG_CHAIN_CHUNK];
  const uint64_t step = step_dev ? (uint64_t)(int64_t)*step_dev : step_arg;
  int cur = 0;
  double rcur = 0.0;
  for (int base = 0; base < p; base += SOG_CHAIN_CHUNK) {
    const int m = min(SOG_CHAIN_CHUNK, p - base);
    __syncthreads();  // thread 0 is done with the previous chunk
    for (int t = threadIdx.x; t < m; t += SOG_CHAIN_BLOCK) {
      const int i = base + t;
      const double kx = 2 * RBX_PI * mx[i] / Lx, ky = 2 * RBX_PI * my[i] / Ly,
                   kz = 2 * RBX_PI * mz[i] / Lz;
      const double k2 = kx * kx + ky * ky + kz * kz;
      s_r[t] = sog_ghat(g.coef_npt, g.mmax, g.b2, g.sig2, k2) * (k2 * k2) /
               (sog_ghat(g.coef, g.mmax, g.b2, g.sig2, k2) * k2);
      uint32_t c[4] = {(uint32_t)i, SOG_NPT_STREAM, (uint32_t)step, (uint32_t)(step >> 32)};
      philox4x32_10(c, key0, key1);
      s_u[t] = u53(c[0], c[1]);
      mult[i] = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int t = 0; t < m; ++t) {
        const int i = base + t;
        const double r = s_r[t];
        if (i == 0) {
          rcur = r;
        } else if (s_u[t] * rcur < r) {
          mult[cur] = i - cur;
          cur = i;
          rcur = r;
        }
        if (idx) idx[i] = cur;
      }
    }
  }
  if (threadIdx.x == 0 && p > 0) mult[cur] = p - cur;
}

// Block k < p: rho(k) from the partial sums (fixed order), the force-table
// entry with c_k = (wa_k / |k|^2 + wb_k) / V and the energy term
// (ea_k / |k|^2 + eb_k) |rho|^2; blocks p..p+2: mean of the pair-force sums.
// With vir, the per-k virial terms (ComputeRBSOGSampleVirialKernel :1133-1190,
// ComputeRBSOGDirectVirialKernel :1308-1355): the energy term on the
// diagonal plus the NPT term g_k k_a k_b.
__global__ void __launch_bounds__(SOG_FK_BLOCK)
k_rbsog_finalize(int p, int nparts, const double* __restrict__ part_re,
                 const double* __restrict__ part_im, const double* __restrict__ mx,
                 const double* __restrict__ my, const double* __restrict__ mz, double Lx,
                 double Ly, double Lz, const double4* __restrict__ w,
                 double* __restrict__ rho_re, double* __restrict__ rho_im,
                 KTab* __restrict__ tab, double* __restrict__ kterm, int mean_parts,
                 const double* __restrict__ fpart, double n_atoms, double* __restrict__ mean_out,
                 SogVirial vir) {
  __shared__ double sh[SOG_FK_BLOCK / 32];
  const int blk = blockIdx.x;
  if (blk >= p) {
    const int d = blk - p;
    double s = 0.0;
    for (int b = threadIdx.x; b < mean_parts; b += SOG_FK_BLOCK) s += fpart[(size_t)b * 3 + d];
    s = block_sum_det<SOG_FK_BLOCK>(s, sh);
    if (threadIdx.x == 0) mean_out[d] = s / n_atoms;
    return;
  }
  const int k = blk;
  double r = 0.0, im = 0.0;
  for (int b = threadIdx.x; b < nparts; b += SOG_FK_BLOCK) {
    r += part_re[(size_t)k * nparts + b];
    im += part_im[(size_t)k * nparts + b];
  }
  r = block_sum_det<SOG_FK_BLOCK>(r, sh);
  im = block_sum_det<SOG_FK_BLOCK>(im, sh);
  if (threadIdx.x != 0) return;
  if (rho_re) {
    rho_re[k] = r;
    rho_im[k] = im;
  }
  const double V = Lx * Ly * Lz;
  const double kx = 2 * RBX_PI * mx[k] / Lx, ky = 2 * RBX_PI * my[k] / Ly,
               kz = 2 * RBX_PI * mz[k] / Lz;
  const double k2 = kx * kx + ky * ky + kz * kz;
  const double4 wk = w[k];
  const double r2 = r * r + im * im;
  if (kterm) kterm[k] = (wk.z / k2 + wk.w) * r2;
  if (vir.vterm) {
    const double e = (wk.z / k2 + wk.w) * r2;
    const double gk = k < vir.psamp ? vir.mult[k] * vir.vw[k] * r2 / (k2 * k2) : vir.vw[k] * r2;
    double* v = vir.vterm + 6 * (size_t)k;
    v[0] = e + gk * kx * kx;
    v[1] = e + gk * ky * ky;
    v[2] = e + gk * kz * kz;
    v[3] = gk * kx * ky;
    v[4] = gk * kx * kz;
    v[5] = gk * ky * kz;
  }
  if (tab) {
    const double c = (wk.x / k2 + wk.y) / V;
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

// Energy: one warp adds the per-k terms in increasing k, then the self term;
// the virial terms likewise when vterm is given.
__global__ void __launch_bounds__(32)
k_rbsog_energy_sum(int p, const double* __restrict__ kterm, double self_energy,
                   double* __restrict__ energy, const double* __restrict__ vterm,
                   double* __restrict__ virial) {
  if (energy) {
    double t = 0.0;
    for (int k = threadIdx.x; k < p; k += 32) t += kterm[k];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) *energy = t + self_energy;
  }
  if (vterm) {
    for (int c = 0; c < 6; ++c) {
      double t = 0.0;
      for (int k = threadIdx.x; k < p; k += 32) t += vterm[6 * (size_t)k + c];
      for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
      if (threadIdx.x == 0) virial[c] = t;
    }
  }
}

// VERLET-SOG pair force (ComputeLJCutCoulForceUserKernel with lj126 and
// CoulCutForceUser, lj_cut_coul_kspace_op.hip.cu:196-254, 357-470): for
// r^2 < cut_off^2, the LJ 12-6 force plus the short-range SOG Coulomb force
// -qqr2e qi qj (1/r^3 + sum_(i<6) c_i r^(2i)); energy 4 eps (s6/r6 - 1) s6/r6 / 2
// and qqr2e qi qj (1/r - sum_l w_l exp(-r^2 / (2 sigma^2 b^(2l)))) / 2.  A warp
// per atom over its candidate row, FP64, per-atom sums in lane order.
// VIRIAL: the per-atom virial flat_virial[c * n + i] of ComputeVirial
// (lj_op.hip.cu:76-88), -r_a r_b f / 2 summed over the atom's pairs.
template <bool ENERGY, bool VIRIAL>
__global__ void __launch_bounds__(SOG_PAIR_BLOCK)
k_verlet_sog(SogPairParams sp, int n, const double* __restrict__ x, const double* __restrict__ y,
             const double* __restrict__ z, const double* __restrict__ q,
             const int* __restrict__ type, const int* __restrict__ cand_count,
             const int* __restrict__ cand, int cap, double* __restrict__ fx,
             double* __restrict__ fy, double* __restrict__ fz, double* __restrict__ epart,
             double* __restrict__ vir) {
  __shared__ double se[2][SOG_PAIR_BLOCK / 32];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int i = blockIdx.x * (SOG_PAIR_BLOCK / 32) + wib;
  double elj = 0.0, ecl = 0.0;
  if (i < n) {
    const double xi = x[i], yi = y[i], zi = z[i], qi = q[i];
    const int ti = type[i];
    const double cut2 = sp.cut_off * sp.cut_off;
    const int cnt = min(cand_count[i], cap);
    double f[3] = {0, 0, 0}, v[6] = {0, 0, 0, 0, 0, 0};
    for (int t = lane; t < cnt; t += 32) {
      const int j = cand[(size_t)i * cap + t];
      double dx = x[j] - xi, dy = y[j] - yi, dz = z[j] - zi;
      dx = min_image1(dx, sp.box.len[0], sp.box.half[0]);
      dy = min_image1(dy, sp.box.len[1], sp.box.half[1]);
      dz = min_image1(dz, sp.box.len[2], sp.box.half[2]);
      const double d2 = dx * dx + dy * dy + dz * dz;
      if (!(d2 < cut2)) continue;
      const int pt = ti * sp.ntypes + type[j];
      const double eps = sp.lj_eps[pt], s6 = sp.lj_s6[pt];
      const double d6 = d2 * d2 * d2;
      const double sd6 = s6 / d6;
      const double flj = -24 * eps * ((2 * sd6 - 1) * sd6) / d2;
      const double r2inv = 1.0 / d2, rinv = sqrt(r2inv), r3inv = rinv * r2inv;
      const double pre = sp.qqr2e * qi * q[j];
      const double poly =
          sp.taylor[0] +
          d2 * (sp.taylor[1] +
                d2 * (sp.taylor[2] + d2 * (sp.taylor[3] + d2 * (sp.taylor[4] + d2 * sp.taylor[5]))));
      const double fcl = -pre * (r3inv + poly);
      const double fp = flj + fcl;
      f[0] += fp * dx;
      f[1] += fp * dy;
      f[2] += fp * dz;
      if (VIRIAL) {
        v[0] += -0.5 * dx * dx * fp;
        v[1] += -0.5 * dy * dy * fp;
        v[2] += -0.5 * dz * dz * fp;
        v[3] += -0.5 * dx * dy * fp;
        v[4] += -0.5 * dx * dz * fp;
        v[5] += -0.5 * dy * dz * fp;
      }
      if (ENERGY) {
        elj += 0.5 * (4 * eps * (s6 / d6 - 1) * sd6);
        double sume = sp.norm * sp.w0 * exp(-d2 / (2.0 * sp.sigma * sp.sigma));
        double bl = 1.0;
        for (int l = 1; l < sp.mmax; ++l) {
          bl *= sp.b;
          sume += sp.norm * (1.0 / bl) * exp(-d2 / (2 * sp.sigma * sp.sigma * bl * bl));
        }
        ecl += 0.5 * pre * (rinv - sume);
      }
    }
    for (int d = 0; d < 3; ++d) f[d] = warp_sum(f[d]);
    if (VIRIAL)
      for (int c = 0; c < 6; ++c) v[c] = warp_sum(v[c]);
    if (lane == 0) {
      fx[i] = f[0];
      fy[i] = f[1];
      fz[i] = f[2];
      if (VIRIAL)
        for (int c = 0; c < 6; ++c) vir[(size_t)c * n + i] = v[c];
    }
  }
  if (ENERGY) {
    elj = warp_sum(elj);
    ecl = warp_sum(ecl);
    if (lane == 0) {
      se[0][wib] = elj;
      se[1][wib] = ecl;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
      double s = 0.0;
      for (int w = 0; w < SOG_PAIR_BLOCK / 32; ++w) s += se[threadIdx.x][w];
      epart[(size_t)blockIdx.x * 2 + threadIdx.x] = s;
    }
  }
}
// Mixed form of the VERLET-SOG force: the pair vector is the exact wrapped
// difference of the fixed-point records scaled by L / 2^32 per axis, the LJ
// and short-range SOG terms are FP32 (cut decided on the FP32 r^2), each lane
// sums its pairs in FP32 and the warp reduces in FP64.
__global__ void __launch_bounds__(SOG_PAIR_BLOCK)
k_verlet_sog_mixed(SogPairParams sp, float sfx, float sfy, float sfz, int n,
                   const uint4* __restrict__ atoms, const int* __restrict__ type,
                   const int* __restrict__ cand_count, const int* __restrict__ cand, int cap,
                   double* __restrict__ fx, double* __restrict__ fy, double* __restrict__ fz) {
  extern __shared__ __align__(16) float s_tab[];  // eps_ij, then sigma_ij^6 (ntypes^2 each)
  const int nt2 = sp.ntypes * sp.ntypes;
  float* const s_eps = s_tab;
  float* const s_s6 = s_tab + nt2;
  for (int t = threadIdx.x; t < nt2; t += SOG_PAIR_BLOCK) {
    s_eps[t] = (float)sp.lj_eps[t];
    s_s6[t] = (float)sp.lj_s6[t];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int i = blockIdx.x * (SOG_PAIR_BLOCK / 32) + wib;
  if (i >= n) return;
  const uint4 ai = atoms[i];
  const int ti = type[i];
  const float qi = __uint_as_float(ai.w);
  const float cut2 = (float)(sp.cut_off * sp.cut_off);
  const float qe = (float)sp.qqr2e;
  float c[6];
  for (int k = 0; k < 6; ++k) c[k] = (float)sp.taylor[k];
  const int cnt = min(cand_count[i], cap);
  float f0 = 0.f, f1 = 0.f, f2 = 0.f;
  for (int t = lane; t < cnt; t += 32) {
    const int j = cand[(size_t)i * cap + t];
    const uint4 aj = __ldg(atoms + j);
    const float dx = (float)(int)(aj.x - ai.x) * sfx, dy = (float)(int)(aj.y - ai.y) * sfy,
                dz = (float)(int)(aj.z - ai.z) * sfz;
    const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    if (!(d2 < cut2)) continue;
    const int pt = ti * sp.ntypes + __ldg(type + j);
    const float r2inv = 1.0f / d2;
    const float sd6 = s_s6[pt] * (r2inv * r2inv * r2inv);
    const float flj = -24.f * s_eps[pt] * ((2.f * sd6 - 1.f) * sd6) * r2inv;
    const float rinv = rsqrtf(d2);
    const float poly = c[0] + d2 * (c[1] + d2 * (c[2] + d2 * (c[3] + d2 * (c[4] + d2 * c[5]))));
    const float f = flj - qe * qi * __uint_as_float(aj.w) * (rinv * r2inv + poly);
    f0 = fmaf(f, dx, f0);
    f1 = fmaf(f, dy, f1);
    f2 = fmaf(f, dz, f2);
  }
  const double g0 = warp_sum((double)f0), g1 = warp_sum((double)f1), g2 = warp_sum((double)f2);
  if (lane == 0) {
    fx[i] = g0;
    fy[i] = g1;
    fz[i] = g2;
  }
}
}  // namespace

int launch_rbsog_sample(int p, const RbsogTables& t, uint64_t seed, uint64_t step,
                        const int* step_dev, double* mx, double* my, double* mz, int* mi,
                        int* status, cudaStream_t st) {
  if (p <= 0) return RBX_OK;
  k_rbsog_sample<<<(p + SOG_SAMPLE_BLOCK - 1) / SOG_SAMPLE_BLOCK, SOG_SAMPLE_BLOCK, 0, st>>>(
      p, t, (uint32_t)seed, (uint32_t)(seed >> 32), step, step_dev, mx, my, mz, mi, status);
  count_launch();
  return check_launch("rbsog_sample");
}

int launch_rbsog_finalize(const DBox& b, int p, int nparts, const double* part_re,
                          const double* part_im, const double* mx, const double* my,
                          const double* mz, const double4* w, double* rho_re, double* rho_im,
                          KTab* tab, double* kterm, double self_energy, double* energy,
                          int mean_parts, const double* fpart, int n_atoms, double* mean_out,
                          cudaStream_t st, const SogVirial* vir) {
  const int grid = p + (mean_out ? 3 : 0);
  const SogVirial v = vir ? *vir : SogVirial{0, nullptr, nullptr, nullptr, nullptr};
  if (grid > 0) {
    k_rbsog_finalize<<<grid, SOG_FK_BLOCK, 0, st>>>(
        p, nparts, part_re, part_im, mx, my, mz, b.len[0], b.len[1], b.len[2], w, rho_re, rho_im,
        tab, energy ? kterm : nullptr, mean_parts, fpart, (double)n_atoms, mean_out, v);
    count_launch();
    const int rc = check_launch("rbsog_finalize");
    if (rc) return rc;
  }
  if (energy || v.vterm) {
    k_rbsog_energy_sum<<<1, 32, 0, st>>>(p, kterm, self_energy, energy, v.vterm, v.out);
    count_launch();
    return check_launch("rbsog_energy_sum");
  }
  return RBX_OK;
}

int launch_rbsog_npt_chain(const DBox& b, int p, const double* mx, const double* my,
                           const double* mz, const SogGauss& g, uint64_t seed, uint64_t step,
                           const int* step_dev, int* idx, int* mult, cudaStream_t st) {
  if (p <= 0) return RBX_OK;
  k_rbsog_npt_chain<<<1, SOG_CHAIN_BLOCK, 0, st>>>(p, mx, my, mz, b.len[0], b.len[1], b.len[2],
                                                   g, (uint32_t)seed, (uint32_t)(seed >> 32),
                                                   step, step_dev, idx, mult);
  count_launch();
  return check_launch("rbsog_npt_chain");
}

int verlet_sog_blocks(int n) { return (n + SOG_PAIR_BLOCK / 32 - 1) / (SOG_PAIR_BLOCK / 32); }

int launch_verlet_sog(const SogPairParams& sp, int n, const double* x, const double* y,
                      const double* z, const double* q, const int* type, const int* cand_count,
                      const int* cand, int cap, double* fx, double* fy, double* fz, double* epart,
                      cudaStream_t st, double* flat_virial) {
  if (n <= 0) return RBX_OK;
  const int grid = verlet_sog_blocks(n);
  auto go = [&](auto kern) {
    kern<<<grid, SOG_PAIR_BLOCK, 0, st>>>(sp, n, x, y, z, q, type, cand_count, cand, cap, fx, fy,
                                          fz, epart, flat_virial);
  };
  if (epart)
    flat_virial ? go(k_verlet_sog<true, true>) : go(k_verlet_sog<true, false>);
  else
    flat_virial ? go(k_verlet_sog<false, true>) : go(k_verlet_sog<false, false>);
  count_launch();
  return check_launch("verlet_sog");
}

}  // namespace rbx

namespace rbx {
int launch_verlet_sog_mixed(const SogPairParams& sp, const float sf[3], int n, const uint4* atoms,
                            const int* type, const int* cand_count, const int* cand, int cap,
                            double* fx, double* fy, double* fz, cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  const size_t smem = (size_t)2 * sp.ntypes * sp.ntypes * sizeof(float);
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(k_verlet_sog_mixed, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess) {
    cudaGetLastError();
    set_error("VERLET-SOG mixed form: %d atom types need %zu bytes of shared memory",
              sp.ntypes, smem);
    return RBX_ERR_INVALID;
  }
  k_verlet_sog_mixed<<<verlet_sog_blocks(n), SOG_PAIR_BLOCK, smem, st>>>(
      sp, sf[0], sf[1], sf[2], n, atoms, type, cand_count, cand, cap, fx, fy, fz);
  count_launch();
  return check_launch("verlet_sog_mixed");
}
}  // namespace rbx
