/*
 * rbx_oracle.c -- FP64 host restatement of RBMD 2.0's RBE + LJ/erfc-Coulomb
 * hot path (see rbx_oracle.h).  TEST INFRASTRUCTURE: used only by tests/, the
 * smoke check and bench.py's CPU-baseline leg, as the checker.
 *
 * Compiled with -ffp-contract=off so that every distance predicate rounds
 * exactly like the reference's `POW(dx,2)+POW(dy,2)+POW(dz,2)`
 * (src/neighbor_list/src/op/full_neighbor_list_op.h:98-106).
 *
 * Citations are relative to the RBMD 2.0 source tree.
 */
#include "rbx_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* EPSILON under USE_DOUBLE (src/common/rbmd_define.h:46-50). */
#define ORC_EPSILON 0.0001

static inline double box_len(const orc_box* b, int d) { return b->hi[d] - b->lo[d]; }

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ========================================================================== */
/* k-space                                                                    */
/* ========================================================================== */

/* ComputeRbeGaussianSum, src/force/src/kspace_calculator.cpp:68-78:
 * S = prod_d H_d - 1, H_d = sqrt(alpha L_d^2/pi) * sum_{m=-10..10} exp(-alpha L_d^2 m^2). */
double orc_rbe_gauss_sum(const orc_box* box, double alpha) {
  double h[3] = {0.0, 0.0, 0.0};
  for (int d = 0; d < 3; ++d) {
    const double L = box_len(box, d);
    const double factor = -(alpha * L * L);
    for (int m = -10; m <= 10; ++m) h[d] += exp((double)(m * m) * factor);
    h[d] *= sqrt(-(factor) / M_PI);
  }
  return h[0] * h[1] * h[2] - 1.0;
}

/* ComputePnumberChargeStructureFactorOpt,
 * src/force/src/kspace_calculator_op/rocm/kspace_calculator_op.hip.cu:238-289:
 * Re rho_p = sum_j q_j cos(k_p.r_j), Im rho_p = sum_j q_j sin(k_p.r_j), k = 2 pi m / L. */
void orc_rbe_structure_factor(int n, int p, const orc_box* box, const double* q,
                              const double* x, const double* y, const double* z,
                              const double* mx, const double* my,
                              const double* mz, double* re, double* im) {
  const double Lx = box_len(box, 0), Ly = box_len(box, 1), Lz = box_len(box, 2);
#pragma omp parallel for schedule(dynamic, 1)
  for (int k = 0; k < p; ++k) {
    const double kx = 2 * M_PI * mx[k] / Lx;
    const double ky = 2 * M_PI * my[k] / Ly;
    const double kz = 2 * M_PI * mz[k] / Lz;
    double sr = 0.0, si = 0.0;
    for (int j = 0; j < n; ++j) {
      const double dot = kx * x[j] + ky * y[j] + kz * z[j];
      sr += q[j] * cos(dot);
      si += q[j] * sin(dot);
    }
    re[k] = sr;
    im[k] = si;
  }
}

/* ComputeRBEForce + RBEForce, kspace_calculator_op.hip.cu:98-125, 678-738:
 * F_i = (S/P) sum_p [-4 pi q_i qqr2e / (V k^2)] (cos(k.r_i) Im - sin(k.r_i) Re) k. */
void orc_rbe_force(int n, int p, const orc_box* box, double S, double qqr2e,
                   const double* re, const double* im, const double* q,
                   const double* mx, const double* my, const double* mz,
                   const double* x, const double* y, const double* z,
                   double* fx, double* fy, double* fz) {
  const double Lx = box_len(box, 0), Ly = box_len(box, 1), Lz = box_len(box, 2);
  const double volume = Lx * Ly * Lz;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    double sx = 0.0, sy = 0.0, sz = 0.0;
    const double factor_a = -4 * M_PI * q[i];
    for (int k = 0; k < p; ++k) {
      const double Kx = 2 * M_PI * mx[k] / Lx;
      const double Ky = 2 * M_PI * my[k] / Ly;
      const double Kz = 2 * M_PI * mz[k] / Lz;
      const double k2 = Kx * Kx + Ky * Ky + Kz * Kz;
      const double dot = Kx * x[i] + Ky * y[i] + Kz * z[i];
      double f = (factor_a / (volume * k2)) * (cos(dot) * im[k] - sin(dot) * re[k]);
      f *= qqr2e;
      sx += f * Kx;
      sy += f * Ky;
      sz += f * Kz;
    }
    fx[i] = sx * S / p;
    fy[i] = sy * S / p;
    fz[i] = sz * S / p;
  }
}

/* ComputeRBEVirial0, kspace_calculator_op.hip.cu:573-674 (the path the op uses):
 * E = qqr2e [ (2 pi S/(P V)) sum |rho|^2/k^2 - sqrt(alpha) sum q^2/sqrt(pi)
 *             - (pi/2) Q^2/(alpha V) ],
 * W_ab = qqr2e (2 pi S/(P V)) sum (|rho|^2/k^2)(delta_ab - 2 k_a k_b (1/(4 alpha) + 1/k^2)).
 * Summed in sample order (the reference's float atomics have no fixed order). */
void orc_rbe_energy_virial(int p, const orc_box* box, double alpha, double S,
                           double qqr2e, double qsq, double qsum,
                           const double* re, const double* im,
                           const double* mx, const double* my,
                           const double* mz, double* virial6, double* energy) {
  const double Lx = box_len(box, 0), Ly = box_len(box, 1), Lz = box_len(box, 2);
  const double V = Lx * Ly * Lz;
  const double coef = (2 * M_PI * S) / (p * V);
  double e = 0.0, w[6] = {0, 0, 0, 0, 0, 0};
  for (int k = 0; k < p; ++k) {
    const double kx = 2 * M_PI * mx[k] / Lx;
    const double ky = 2 * M_PI * my[k] / Ly;
    const double kz = 2 * M_PI * mz[k] / Lz;
    const double k2 = kx * kx + ky * ky + kz * kz;
    const double rho2 = re[k] * re[k] + im[k] * im[k];
    e += coef * rho2 / k2;
    const double base = coef * rho2 / k2;
    const double inner = (1.0 / (4 * alpha)) + (1.0 / k2);
    w[0] += base * (1.0 - 2 * kx * kx * inner);
    w[1] += base * (1.0 - 2 * ky * ky * inner);
    w[2] += base * (1.0 - 2 * kz * kz * inner);
    w[3] += base * (-2 * kx * ky * inner);
    w[4] += base * (-2 * kx * kz * inner);
    w[5] += base * (-2 * ky * kz * inner);
  }
  const double MY_PIS = 1.77245385090551602729, MY_PI2 = 1.57079632679489661923;
  e -= sqrt(alpha) * qsq / MY_PIS + MY_PI2 * qsum * qsum / (alpha * V);
  *energy = e * qqr2e;
  for (int j = 0; j < 6; ++j) virial6[j] = w[j] * qqr2e;
}

/* Exact Ewald over the kmax box, the ordering of ExecuteOnKmax /
 * ComputeKspaceEnergy (kspace_calculator.cpp:816-895). */
int orc_ewald_num_k(const int kmax[3]) {
  return (2 * kmax[0] + 1) * (2 * kmax[1] + 1) * (2 * kmax[2] + 1) - 1;
}

void orc_ewald_kvectors(const int kmax[3], const orc_box* box, double* kx,
                        double* ky, double* kz) {
  int idx = 0;
  for (int i = -kmax[0]; i <= kmax[0]; ++i)
    for (int j = -kmax[1]; j <= kmax[1]; ++j)
      for (int k = -kmax[2]; k <= kmax[2]; ++k) {
        if (i == 0 && j == 0 && k == 0) continue;
        kx[idx] = 2 * M_PI * i / box_len(box, 0);
        ky[idx] = 2 * M_PI * j / box_len(box, 1);
        kz[idx] = 2 * M_PI * k / box_len(box, 2);
        ++idx;
      }
}

/* ComputeKspaceChargeStructureFactor, kspace_calculator_op.hip.cu:176-213. */
void orc_ewald_structure_factor(int n, int nk, const double* q,
                                const double* x, const double* y,
                                const double* z, const double* kx,
                                const double* ky, const double* kz, double* re,
                                double* im) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int k = 0; k < nk; ++k) {
    double sr = 0.0, si = 0.0;
    for (int j = 0; j < n; ++j) {
      const double dot = kx[k] * x[j] + ky[k] * y[j] + kz[k] * z[j];
      sr += q[j] * cos(dot);
      si += q[j] * sin(dot);
    }
    re[k] = sr;
    im[k] = si;
  }
}

/* ComputeEwaldForceFlat, kspace_calculator_op.hip.cu:334-403. */
void orc_ewald_force(int n, int nk, const orc_box* box, double alpha,
                     double qqr2e, const double* kx, const double* ky,
                     const double* kz, const double* re, const double* im,
                     const double* q, const double* x, const double* y,
                     const double* z, double* fx, double* fy, double* fz) {
  const double volume = box_len(box, 0) * box_len(box, 1) * box_len(box, 2);
  const double alpha_inv = 1.0 / alpha;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    const double base = -4.0 * M_PI * q[i];
    double sx = 0, sy = 0, sz = 0;
    for (int k = 0; k < nk; ++k) {
      const double k2 = kx[k] * kx[k] + ky[k] * ky[k] + kz[k] * kz[k];
      const double dot = -(kx[k] * x[i] + ky[k] * y[i] + kz[k] * z[i]);
      const double fb = exp(-0.25 * k2 * alpha_inv);
      double f = base / (volume * k2) * fb * (cos(dot) * im[k] + sin(dot) * re[k]);
      f *= qqr2e;
      sx += f * kx[k];
      sy += f * ky[k];
      sz += f * kz[k];
    }
    fx[i] = sx;
    fy[i] = sy;
    fz[i] = sz;
  }
}

/* ComputeKspaceEnergy + ComputeSelfEnergy, kspace_calculator.cpp:816-907. */
double orc_ewald_energy(int nk, const orc_box* box, double alpha, double qqr2e,
                        double qsq, const double* kx, const double* ky,
                        const double* kz, const double* re, const double* im) {
  const double volume = box_len(box, 0) * box_len(box, 1) * box_len(box, 2);
  double e = 0.0;
  for (int k = 0; k < nk; ++k) {
    const double k2 = kx[k] * kx[k] + ky[k] * ky[k] + kz[k] * kz[k];
    e += exp(-0.25 * k2 / alpha) / k2 * (re[k] * re[k] + im[k] * im[k]);
  }
  e = qqr2e * (2 * M_PI / volume) * e;
  return e + qqr2e * (-sqrt(alpha / M_PI) * qsq);
}

/* ========================================================================== */
/* k-vector samplers                                                          */
/* ========================================================================== */

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
 * as 1, 2, 3", SC'11): 10 rounds of two 32x32->64 multiplies with Weyl key
 * schedule.  The project's on-device k-sampler uses the same function. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2],
                       uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c0 = hi1 ^ c1 ^ k0;
    c1 = lo1;
    c2 = hi0 ^ c3 ^ k1;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

/* Discrete Gaussian weights of the RBE importance density along one axis:
 * P(m) ~ exp(-(2 pi m / L)^2 / (4 alpha)) (RBEPSample.h:98-105), tabulated in
 * the order m = 0, +1, -1, +2, -2, ... until the weight drops below 1e-20. */
static int rbe_axis_table(double L, double alpha, double* w, int max_entries,
                          double* total) {
  const double c = (M_PI * M_PI) / (alpha * L * L);
  int cnt = 0;
  double z = 0.0;
  for (int m = 0;; ++m) {
    const double v = exp(-c * (double)m * (double)m);
    if (m > 0 && v < 1e-20) break;
    if (cnt + (m == 0 ? 1 : 2) > max_entries) return -1;
    if (m == 0) {
      w[cnt++] = v;
      z += v;
    } else {
      w[cnt++] = v;
      w[cnt++] = v;
      z += v;
      z += v;
    }
  }
  *total = z;
  return cnt;
}

static inline int rbe_table_pick(const double* w, int cnt, double total, uint64_t u53) {
  const double target = (double)u53 * (1.0 / 9007199254740992.0) * total;
  double acc = 0.0;
  int idx = cnt - 1;
  for (int t = 0; t < cnt; ++t) {
    acc += w[t];
    if (target < acc) {
      idx = t;
      break;
    }
  }
  /* idx 0 -> m = 0; odd 2k-1 -> +k; even 2k -> -k */
  if (idx == 0) return 0;
  return (idx & 1) ? (idx + 1) / 2 : -(idx / 2);
}

/* Counter-based RBE k-sampler (the project's replacement of RBEPSample's
 * Metropolis-Hastings chain, RBEPSample.h:150-188): i.i.d. draws from the same
 * discrete density, excluding m = (0,0,0).  Counter = (sample, 2*attempt+b,
 * step_lo, step_hi), key = (seed_lo, seed_hi); three 53-bit uniforms per
 * attempt drive an inverse-CDF pick per axis.  Returns 0, or -1 if a sample
 * needed more than 64 attempts or a table overflowed. */
int orc_rbe_sample_philox(int p, const orc_box* box, double alpha,
                          uint64_t seed, int64_t step, double* mx, double* my,
                          double* mz) {
  enum { MAXT = 4096 };
  static double w[3][MAXT];
  double tot[3];
  int cnt[3];
  for (int d = 0; d < 3; ++d) {
    cnt[d] = rbe_axis_table(box_len(box, d), alpha, w[d], MAXT, &tot[d]);
    if (cnt[d] < 0) return -1;
  }
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  const uint64_t ustep = (uint64_t)step;
  for (int s = 0; s < p; ++s) {
    int ok = 0;
    for (int a = 0; a < 64 && !ok; ++a) {
      uint32_t o[8];
      const uint32_t c0[4] = {(uint32_t)s, (uint32_t)(2 * a), (uint32_t)ustep,
                              (uint32_t)(ustep >> 32)};
      const uint32_t c1[4] = {(uint32_t)s, (uint32_t)(2 * a + 1),
                              (uint32_t)ustep, (uint32_t)(ustep >> 32)};
      orc_philox4x32_10(c0, key, o);
      orc_philox4x32_10(c1, key, o + 4);
      int m[3];
      for (int d = 0; d < 3; ++d) {
        const uint64_t u = (((uint64_t)o[2 * d] << 32) | o[2 * d + 1]) >> 11;
        m[d] = rbe_table_pick(w[d], cnt[d], tot[d], u);
      }
      if (m[0] != 0 || m[1] != 0 || m[2] != 0) {
        mx[s] = m[0];
        my[s] = m[1];
        mz[s] = m[2];
        ok = 1;
      }
    }
    if (!ok) return -1;
  }
  return 0;
}

/* -- restatement of the reference's MH chain (statistical comparison only) -- */
typedef struct {
  uint64_t s;
} orc_rng;
static inline uint64_t rng_next(orc_rng* r) { /* SplitMix64 stream */
  uint64_t z = (r->s += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
static inline double rng_uniform(orc_rng* r) {
  return (double)(rng_next(r) >> 11) * (1.0 / 9007199254740992.0);
}

/* FetchSample_1D, RBEPSample.h:124-148 (Box-Muller, U1 >= 1e-6). */
static double mh_gauss(orc_rng* r, double sigma) {
  double u1;
  do {
    u1 = rng_uniform(r);
  } while (u1 < 1e-6);
  const double u2 = rng_uniform(r);
  return sigma * sqrt(-2.0 * log(u1)) * cos(2 * M_PI * u2);
}

typedef struct {
  double alpha, L[3], H[3];
} mh_ctx;

/* Distribution_P, RBEPSample.h:98-105. */
static double mh_P(const mh_ctx* c, double x, int d) {
  const double t = 2 * M_PI * x / c->L[d];
  return exp(-(t * t) / (4 * c->alpha)) / c->H[d];
}
/* Distribution_q, RBEPSample.h:107-122. */
static double mh_q(const mh_ctx* c, double x, int d) {
  const double s = sqrt(c->alpha * c->L[d] * c->L[d] / (M_PI * M_PI));
  if (x == 0 || fabs(x) < 1.0e-13) return erf(0.5 / s);
  return (erf((0.5 + fabs(x)) / s) - erf((fabs(x) - 0.5) / s)) / 2;
}
/* MH_Algorithm, RBEPSample.h:70-97. */
static double mh_step(const mh_ctx* c, orc_rng* r, double m, double sigma, int d) {
  const double mw = round(mh_gauss(r, sigma));
  double prob = (mh_P(c, mw, d) / mh_P(c, m, d)) * (mh_q(c, m, d) / mh_q(c, mw, d));
  if (prob > 1.0) prob = 1.0;
  const double u = rng_uniform(r);
  return (u <= prob) ? mw : m;
}

/* Fetch_P_Sample, RBEPSample.h:150-188, with sigma from
 * KSpaceCalculator::RBEInit (kspace_calculator.cpp:697-700). */
void orc_rbe_sample_mh(int p, const orc_box* box, double alpha, uint64_t seed,
                       double* mx, double* my, double* mz) {
  mh_ctx c;
  c.alpha = alpha;
  double sig[3];
  for (int d = 0; d < 3; ++d) {
    c.L[d] = box_len(box, d);
    const double factor = -(alpha * c.L[d] * c.L[d]);
    c.H[d] = 0.0;
    for (int m = -10; m <= 10; ++m) c.H[d] += exp((double)(m * m) * factor);
    c.H[d] *= sqrt(-factor / M_PI);
    sig[d] = sqrt(alpha / 2.0) * c.L[d] / M_PI;
  }
  orc_rng r = {seed};
  const double eps = 1e-6;
  double x0[3];
  do {
    for (int d = 0; d < 3; ++d) x0[d] = round(mh_gauss(&r, sig[d]));
  } while (fabs(x0[0]) < eps && fabs(x0[1]) < eps && fabs(x0[2]) < eps);
  mx[0] = x0[0];
  my[0] = x0[1];
  mz[0] = x0[2];
  for (int i = 1; i < p; i++) {
    double x1[3];
    for (int d = 0; d < 3; ++d) x1[d] = mh_step(&c, &r, x0[d], sig[d], d);
    mx[i] = x1[0];
    my[i] = x1[1];
    mz[i] = x1[2];
    x0[0] = x1[0];
    x0[1] = x1[1];
    x0[2] = x1[2];
    if (fabs(x1[0]) < eps && fabs(x1[1]) < eps && fabs(x1[2]) < eps) {
      i = i - 1;
      continue;
    }
  }
}

/* ========================================================================== */
/* Geometry, cells and neighbor lists                                         */
/* ========================================================================== */

/* MinImageDistance single shift, box.h:51-73. */
static inline void min_image(const orc_box* b, double* dx, double* dy, double* dz) {
  const double Lx = box_len(b, 0), Ly = box_len(b, 1), Lz = box_len(b, 2);
  if (fabs(*dx) > Lx * 0.5) *dx -= (*dx > 0 ? Lx : -Lx);
  if (fabs(*dy) > Ly * 0.5) *dy -= (*dy > 0 ? Ly : -Ly);
  if (fabs(*dz) > Lz * 0.5) *dz -= (*dz > 0 ? Lz : -Lz);
}

/* MinImageDistance_while, box.h:75-97. */
static inline void min_image_while(const orc_box* b, double* dx, double* dy, double* dz) {
  const double Lx = box_len(b, 0), Ly = box_len(b, 1), Lz = box_len(b, 2);
  /* bounded form of the while loop: nearest image by rint */
  if (fabs(*dx) > Lx * 0.5) *dx -= Lx * rint(*dx / Lx);
  if (fabs(*dy) > Ly * 0.5) *dy -= Ly * rint(*dy / Ly);
  if (fabs(*dz) > Lz * 0.5) *dz -= Lz * rint(*dz / Lz);
}

/* CaculateDistance, full_neighbor_list_op.h:98-106 (i minus j, squared terms
 * summed left to right without fused multiply-add). */
double orc_dist2(const orc_box* box, double xi, double yi, double zi, double xj,
                 double yj, double zj) {
  double dx = xi - xj, dy = yi - yj, dz = zi - zj;
  min_image(box, &dx, &dy, &dz);
  return dx * dx + dy * dy + dz * dz;
}

/* LinkedCell::Build (linked_cell.cpp:251-411) without halo: per-dimension cell
 * count floor(L / neighbor_cutoff). */
int orc_cell_grid(const orc_box* box, double neighbor_cutoff, int dims[3]) {
  for (int d = 0; d < 3; ++d) {
    const double nd = floor(box_len(box, d) / neighbor_cutoff);
    if (!(nd >= 1.0)) return -1;
    dims[d] = (int)nd;
  }
  return dims[0] * dims[1] * dims[2];
}

/* AssignAtomsToCell (linked_cell_op.hip.cu:57-138, halo width 0), stable sort
 * by cell (SortAtomsByCellKey, linked_cell.cpp:485-560) and cell ranges
 * (ComputeCellRangesIndices, linked_cell_op.hip.cu:142-164).
 * perm[new] = old index; cell_of_sorted[new] = cell id. */
int orc_cells_sort(int n, const orc_box* box, double neighbor_cutoff,
                   const double* x, const double* y, const double* z,
                   int* perm, int* cell_of_sorted, int* cell_start,
                   int* cell_end) {
  int dims[3];
  const int ncell = orc_cell_grid(box, neighbor_cutoff, dims);
  if (ncell <= 0) return -1;
  double clen[3], crecip[3];
  for (int d = 0; d < 3; ++d) {
    clen[d] = box_len(box, d) / dims[d];
    crecip[d] = 1.0 / clen[d];
  }
  int* cell = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  const double* pos[3] = {x, y, z};
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    int c[3];
    for (int d = 0; d < 3; ++d) {
      int v = (int)floor((pos[d][i] - box->lo[d]) * crecip[d]);
      v = v < 0 ? 0 : v;
      v = v > dims[d] - 1 ? dims[d] - 1 : v;
      c[d] = v;
    }
    /* one-cell correction against the cell bounds lo + c*len */
    int cc[3];
    int inside = 1;
    for (int d = 0; d < 3; ++d) {
      const double cmin = c[d] * clen[d] + box->lo[d];
      const double cmax = (c[d] + 1) * clen[d] + box->lo[d];
      if (!(cmin <= pos[d][i] && pos[d][i] < cmax)) inside = 0;
    }
    if (!inside) {
      for (int d = 0; d < 3; ++d) {
        const double cmin = c[d] * clen[d] + box->lo[d];
        const double cmax = (c[d] + 1) * clen[d] + box->lo[d];
        cc[d] = c[d];
        if (pos[d][i] < cmin)
          cc[d]--;
        else if (pos[d][i] >= cmax)
          cc[d]++;
        cc[d] = cc[d] < 0 ? 0 : (cc[d] > dims[d] - 1 ? dims[d] - 1 : cc[d]);
      }
      int ok = 1;
      for (int d = 0; d < 3; ++d) {
        const double cmin = cc[d] * clen[d] + box->lo[d];
        const double cmax = (cc[d] + 1) * clen[d] + box->lo[d];
        if (!(cmin <= pos[d][i] && pos[d][i] < cmax)) ok = 0;
      }
      if (ok) {
        c[0] = cc[0];
        c[1] = cc[1];
        c[2] = cc[2];
      }
    }
    cell[i] = (c[2] * dims[1] + c[1]) * dims[0] + c[0];
  }
  /* stable counting sort by cell id */
  for (int c = 0; c < ncell; ++c) cell_start[c] = 0;
  for (int i = 0; i < n; ++i) cell_start[cell[i]]++;
  int acc = 0;
  for (int c = 0; c < ncell; ++c) {
    const int t = cell_start[c];
    cell_start[c] = acc;
    cell_end[c] = acc;
    acc += t;
  }
  for (int i = 0; i < n; ++i) {
    const int pos_new = cell_end[cell[i]]++;
    perm[pos_new] = i;
    cell_of_sorted[pos_new] = cell[i];
  }
  free(cell);
  return ncell;
}

/* ComputeFullNeighborStencilCellOnTheFly (full_neighbor_list_op.hip.cu:19-85)
 * for a whole-domain grid: stencil index s -> offsets (s%3-1, (s/3)%3-1, s/9-1). */
static inline int stencil_cell(const int dims[3], int cell_idx, int s) {
  const int ox = s % 3 - 1, oy = (s / 3) % 3 - 1, oz = s / 9 - 1;
  const int cz = cell_idx / (dims[0] * dims[1]);
  const int cy = (cell_idx - cz * dims[0] * dims[1]) / dims[0];
  const int cx = cell_idx - dims[0] * (cy + dims[1] * cz);
  int nx = (cx + ox) % dims[0];
  if (nx < 0) nx += dims[0];
  int ny = (cy + oy) % dims[1];
  if (ny < 0) ny += dims[1];
  int nz = (cz + oz) % dims[2];
  if (nz < 0) nz += dims[2];
  return (nz * dims[1] + ny) * dims[0] + nx;
}

/* GenerateFullNeighborListNoWarp (full_neighbor_list_op.hip.cu:227-288) over
 * sorted atoms: j != i with dist2 < neighbor_cutoff^2.  Row i of nbrs holds up
 * to cap entries; count[i] is the true count.  Returns the largest count. */
int64_t orc_full_list(int n, const orc_box* box, double neighbor_cutoff,
                      const double* x, const double* y, const double* z,
                      const int* cell_of, const int* cell_start,
                      const int* cell_end, int cap, int* count, int* nbrs) {
  int dims[3];
  if (orc_cell_grid(box, neighbor_cutoff, dims) <= 0) return -1;
  const double cut2 = neighbor_cutoff * neighbor_cutoff;
  int64_t maxc = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(max : maxc)
  for (int i = 0; i < n; ++i) {
    int cnt = 0;
    int seen[27], nseen = 0;
    for (int s = 0; s < 27; ++s) {
      const int nc = stencil_cell(dims, cell_of[i], s);
      /* fewer than three cells along an axis: the stencil wraps onto a cell
       * it has visited (the reference's WrapFullNeighborStencilIndex then
       * lists those pairs twice); each pair is listed once here */
      int dup = 0;
      for (int k = 0; k < nseen; ++k) dup |= seen[k] == nc;
      if (dup) continue;
      seen[nseen++] = nc;
      for (int j = cell_start[nc]; j < cell_end[nc]; ++j) {
        if (j == i) continue;
        const double d2 = orc_dist2(box, x[i], y[i], z[i], x[j], y[j], z[j]);
        if (d2 < cut2) {
          if (cnt < cap && nbrs) nbrs[(size_t)i * cap + cnt] = j;
          ++cnt;
        }
      }
    }
    count[i] = cnt;
    if (cnt > maxc) maxc = cnt;
  }
  return maxc;
}

/* RblFullNeighborListBuilder::GetRblParams (rbl_full_neighbor_list_builder.cpp:193-228). */
int orc_rbl_params(int n_global, const orc_box* box, double r_core,
                   double cut_off, int sample_num, int* rs_num, int* rc_num) {
  const double volume = box_len(box, 0) * box_len(box, 1) * box_len(box, 2);
  const double rho = (double)n_global / volume;
  const double coeff = 1.0 + (0.05 / rho - 0.05);
  const int icoeff = (int)round(coeff);
  const int rs = (int)(icoeff * rho * ceil(4.0 / 3.0 * M_PI * pow(r_core, 3)) + 1);
  const int rc = (int)(icoeff * rho * ceil(4.0 / 3.0 * M_PI * pow(cut_off, 3)) + 1);
  if (rs_num) *rs_num = rs;
  if (rc_num) *rc_num = rc;
  const int shell = rc - rs;
  return shell <= sample_num ? 1 : (int)ceil((double)shell / (double)sample_num);
}

/* MixRblSampleKey (rbl_full_neighbor_list_op.hip.cu:6-11): SplitMix64 finaliser. */
uint64_t orc_rbl_mix(uint64_t v) {
  v += 0x9e3779b97f4a7c15ULL;
  v = (v ^ (v >> 30)) * 0xbf58476d1ce4e5b9ULL;
  v = (v ^ (v >> 27)) * 0x94d049bb133111ebULL;
  return v ^ (v >> 31);
}

/* RblShellSampleSelected (rbl_full_neighbor_list_op.hip.cu:13-30). */
int orc_rbl_selected(int freq, int epoch, int gid_i, int gid_j) {
  if (freq <= 1) return 1;
  uint64_t key = (uint64_t)(int64_t)epoch;
  key ^= orc_rbl_mix((uint64_t)(int64_t)gid_i);
  key ^= orc_rbl_mix((uint64_t)(int64_t)gid_j + 0xd1b54a32d192ed03ULL);
  return orc_rbl_mix(key) % (uint64_t)freq == 0ULL;
}

/* FilterRBLNeighborCandidates (rbl_full_neighbor_list_op.hip.cu:237-304) with
 * the host capacity loops run to completion (FilterCandidateList,
 * rbl_full_neighbor_list_builder.cpp:416-471): core = r^2 < r_core^2 - EPS,
 * sampled shell = r^2 < cut_off^2 - EPS and selected.  Row layout as cand. */
void orc_rbl_filter(int n, const orc_box* box, double r_core, double cut_off,
                    int freq, int epoch, const int* gid, const double* x,
                    const double* y, const double* z, int cap,
                    const int* cand_count, const int* cand, int* core_count,
                    int* core, int* shell_count, int* shell) {
  const double core2 = r_core * r_core - ORC_EPSILON;
  const double force2 = cut_off * cut_off - ORC_EPSILON;
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < n; ++i) {
    int nc = 0, ns = 0;
    const int* row = cand + (size_t)i * cap;
    for (int t = 0; t < cand_count[i]; ++t) {
      const int j = row[t];
      if (j == i) continue;
      const double d2 = orc_dist2(box, x[i], y[i], z[i], x[j], y[j], z[j]);
      if (d2 < core2) {
        core[(size_t)i * cap + nc++] = j;
      } else if (d2 < force2 && orc_rbl_selected(freq, epoch, gid[i], gid[j])) {
        shell[(size_t)i * cap + ns++] = j;
      }
    }
    core_count[i] = nc;
    shell_count[i] = ns;
  }
}

/* ========================================================================== */
/* Pair forces                                                                */
/* ========================================================================== */

/* lj126_rs / lj126_rcs (src/force/src/lj_op/rocm/lj_op.hip.cu:40-73) and
 * CoulCutForce_rs_fix / _rcs_fix (lj_cut_coul_kspace_op.hip.cu:134-194). */
static inline double lj_force(double eps_ij, double sigma_ij, double d2) {
  const double s6 = pow(sigma_ij, 6.0);
  const double d6 = pow(d2, 3.0);
  const double sd6 = s6 / d6;
  return -24 * eps_ij * ((2 * sd6 - 1) * sd6) / d2;
}
static inline double coul_force(double alpha, double qqr2e, double qi, double qj,
                                double d2) {
  const double dis = sqrt(d2);
  const double erfcx = sqrt(alpha) * dis;
  const double g = (1.0 - erf(erfcx)) / d2 +
                   2 * sqrt(alpha) * exp(-alpha * d2) / (sqrt(M_PI) * dis);
  return -qqr2e * qi * qj * g / dis;
}

/* ComputeLJCutCoulRBLForce (lj_cut_coul_kspace_op.hip.cu:569-683). */
void orc_pair_force_rbl(int n, const orc_box* box, double r_core, double cut_off,
                        int freq, double alpha, double qqr2e, const int* type,
                        const double* sigma, const double* eps, const double* q,
                        const double* x, const double* y, const double* z,
                        int cap, const int* core_count, const int* core,
                        const int* shell_count, const int* shell, double* fx,
                        double* fy, double* fz) {
  const double rs2 = r_core * r_core, rc2 = cut_off * cut_off;
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < n; ++i) {
    const int ti = type[i];
    const double eps_i = eps[ti], sig_i = sigma[ti], qi = q[i];
    double sx = 0, sy = 0, sz = 0, cx = 0, cy = 0, cz = 0;
    for (int t = 0; t < core_count[i]; ++t) {
      const int j = core[(size_t)i * cap + t];
      const int tj = type[j];
      const double eps_ij = sqrt(eps_i * eps[tj]);
      const double sig_ij = (sig_i + sigma[tj]) / 2;
      double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
      min_image(box, &dx, &dy, &dz);
      const double d2 = dx * dx + dy * dy + dz * dz;
      double f = 0.0;
      if (d2 < rs2 && d2 > ORC_EPSILON)
        f = lj_force(eps_ij, sig_ij, d2) + coul_force(alpha, qqr2e, qi, q[j], d2);
      sx += f * dx;
      sy += f * dy;
      sz += f * dz;
    }
    for (int t = 0; t < shell_count[i]; ++t) {
      const int j = shell[(size_t)i * cap + t];
      const int tj = type[j];
      const double eps_ij = sqrt(eps_i * eps[tj]);
      const double sig_ij = (sig_i + sigma[tj]) / 2;
      double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
      min_image(box, &dx, &dy, &dz);
      const double d2 = dx * dx + dy * dy + dz * dz;
      double f = 0.0;
      if (d2 < rc2 && d2 > rs2)
        f = freq * lj_force(eps_ij, sig_ij, d2) +
            freq * coul_force(alpha, qqr2e, qi, q[j], d2);
      cx += f * dx;
      cy += f * dy;
      cz += f * dz;
    }
    fx[i] = sx + cx;
    fy[i] = sy + cy;
    fz[i] = sz + cz;
  }
}

/* ComputeSpecialLJCutCoulRBLForce (src/force/src/cvff_op/rocm/cvff_op.hip.cu:401-533),
 * CVFF's RBL pair force: LJ from the type-pair tables 48 eps sigma^12 and
 * 24 eps sigma^6 (CVFF::Init, cvff.cpp:855-870; LJForceFromTypePair :387-398),
 * both multiplied by the special-bond weight of the pair, and the erfc
 * Coulomb minus (1 - weight) times the bare Coulomb -qqr2e qi qj / r^3 (not
 * multiplied by pice_num in the shell).  The weight of partner gid g in row i
 * (LookupSpecialWeight :79-110): w12 / w13 / w14 by its position against the
 * cumulative counts nspecial[i][0..2] (clamped as LoadSpecialCounts :51-77),
 * 1 when g is absent. */
static double special_weight(const int* ns, const int* row, int maxs, int g, double w12,
                             double w13, double w14) {
  int n12 = ns[0] < 0 ? 0 : ns[0], n13 = ns[1] < 0 ? 0 : ns[1], n14 = ns[2] < 0 ? 0 : ns[2];
  if (n12 > n13) n13 = n12;
  if (n13 > n14) n14 = n13;
  if (n14 > maxs) n14 = maxs;
  if (n13 > n14) n13 = n14;
  if (n12 > n13) n12 = n13;
  for (int k = 0; k < n14; ++k)
    if (row[k] == g) return k < n12 ? w12 : (k < n13 ? w13 : w14);
  return 1.0;
}

void orc_pair_force_rbl_special(int n, const orc_box* box, double r_core, double cut_off,
                                int freq, double alpha, double qqr2e, const int* type,
                                int ntypes, const double* lj12, const double* lj6,
                                const int* gid, const double* q, const double* x,
                                const double* y, const double* z, int cap,
                                const int* core_count, const int* core, const int* shell_count,
                                const int* shell, const int* nspecial, const int* special,
                                int maxs, double w12, double w13, double w14, double* fx,
                                double* fy, double* fz) {
  const double rs2 = r_core * r_core, rc2 = cut_off * cut_off;
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < n; ++i) {
    const int ti = type[i];
    const double qi = q[i];
    double f3[3] = {0, 0, 0};
    for (int pass = 0; pass < 2; ++pass) {
      const int cnt = pass == 0 ? core_count[i] : shell_count[i];
      const int* lst = pass == 0 ? core : shell;
      const double lo = pass == 0 ? ORC_EPSILON : rs2, hi = pass == 0 ? rs2 : rc2;
      const double mult = pass == 0 ? 1.0 : (double)freq;
      for (int t = 0; t < cnt; ++t) {
        const int j = lst[(size_t)i * cap + t];
        if (j == i) continue;
        const int pair = ti * ntypes + type[j];
        double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
        min_image_while(box, &dx, &dy, &dz);
        const double d2 = dx * dx + dy * dy + dz * dz;
        double flj = 0.0;
        if (d2 > lo && d2 < hi) {
          const double r2inv = 1.0 / d2, r6inv = r2inv * r2inv * r2inv;
          flj = -mult * r2inv * r6inv * (lj12[pair] * r6inv - lj6[pair]);
        }
        const double w = special ? special_weight(nspecial + 3 * (size_t)i,
                                                  special + (size_t)i * maxs, maxs, gid[j],
                                                  w12, w13, w14)
                                 : 1.0;
        double fc = 0.0, bare = 0.0;
        if (d2 < hi && d2 > lo) {
          const double dis = sqrt(d2);
          const double g = (1.0 - erf(sqrt(alpha) * dis)) / d2 +
                           2 * sqrt(alpha) * exp(-alpha * d2) / (sqrt(M_PI) * dis);
          bare = -qqr2e * qi * q[j] / pow(dis, 3.0);
          fc = -mult * qqr2e * qi * q[j] * g / dis;
        }
        const double f = w * flj + (fc - (1 - w) * bare);
        f3[0] += f * dx;
        f3[1] += f * dy;
        f3[2] += f * dz;
      }
    }
    fx[i] = f3[0];
    fy[i] = f3[1];
    fz[i] = f3[2];
  }
}

/* LJCutCoulKspace::ComputeLJRBL mean-force removal (lj_cut_coul_kspace.cpp:537-563)
 * + FixRBLForce (src/force/src/force_op/rocm/force_op.hip.cu:9-45). */
void orc_fix_rbl(int n, double* fx, double* fy, double* fz, double mean_out[3]) {
  double s[3] = {0, 0, 0};
  for (int i = 0; i < n; ++i) {
    s[0] += fx[i];
    s[1] += fy[i];
    s[2] += fz[i];
  }
  const double mx = s[0] / n, my = s[1] / n, mz = s[2] / n;
  for (int i = 0; i < n; ++i) {
    fx[i] -= mx;
    fy[i] -= my;
    fz[i] -= mz;
  }
  if (mean_out) {
    mean_out[0] = mx;
    mean_out[1] = my;
    mean_out[2] = mz;
  }
}

/* ComputeLJCutCoulForce (lj_cut_coul_kspace_op.hip.cu:256-356) with lj126
 * (lj_op.hip.cu:18-38), CoulCutForce (lj_cut_coul_kspace_op.hip.cu:108-132)
 * and ComputeVirial (lj_op.hip.cu:76-88); virial summed over atoms in index
 * order (Force::ReduceVirial, force.h:24-41). */
void orc_pair_force_verlet(int n, const orc_box* box, double cut_off,
                           double alpha, double qqr2e, const int* type,
                           const double* sigma, const double* eps,
                           const double* q, const double* x, const double* y,
                           const double* z, int cap, const int* count,
                           const int* nbrs, double* fx, double* fy, double* fz,
                           double* virial6, double* evdwl, double* ecoul) {
  const double cut2 = cut_off * cut_off;
  double* vir = (double*)calloc((size_t)6 * (n > 0 ? n : 1), sizeof(double));
  double* elj = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
  double* ecl = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < n; ++i) {
    const int ti = type[i];
    double sx = 0, sy = 0, sz = 0, el = 0, ec = 0, w[6] = {0, 0, 0, 0, 0, 0};
    for (int t = 0; t < count[i]; ++t) {
      const int j = nbrs[(size_t)i * cap + t];
      const int tj = type[j];
      const double eps_ij = sqrt(eps[ti] * eps[tj]);
      const double sig_ij = (sigma[ti] + sigma[tj]) / 2;
      double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
      min_image(box, &dx, &dy, &dz);
      const double d2 = dx * dx + dy * dy + dz * dz;
      double flj = 0, elj_p = 0, fc = 0, ec_p = 0;
      if (d2 < cut2) {
        const double s6 = pow(sig_ij, 6.0);
        const double d6 = pow(d2, 3.0);
        const double sd6 = s6 / d6;
        flj = -24 * eps_ij * ((2 * sd6 - 1) * sd6) / d2;
        elj_p = 0.5 * (4 * eps_ij * (s6 / d6 - 1) * sd6);
        const double dis = sqrt(d2);
        const double erfc_v = erfc(sqrt(alpha) * dis);
        const double g = erfc_v / d2 + 2 * sqrt(alpha) * exp(-alpha * d2) / (sqrt(M_PI) * dis);
        fc = -qqr2e * q[i] * q[j] * g / dis;
        ec_p = qqr2e * (0.5 * q[i] * q[j] * erfc_v / dis);
      }
      const double f = flj + fc;
      sx += f * dx;
      sy += f * dy;
      sz += f * dz;
      el += elj_p;
      ec += ec_p;
      w[0] += -0.5 * dx * dx * f;
      w[1] += -0.5 * dy * dy * f;
      w[2] += -0.5 * dz * dz * f;
      w[3] += -0.5 * dx * dy * f;
      w[4] += -0.5 * dx * dz * f;
      w[5] += -0.5 * dy * dz * f;
    }
    fx[i] = sx;
    fy[i] = sy;
    fz[i] = sz;
    elj[i] = el;
    ecl[i] = ec;
    for (int c = 0; c < 6; ++c) vir[(size_t)c * n + i] = w[c];
  }
  double tw[6] = {0, 0, 0, 0, 0, 0}, te = 0, tc = 0;
  for (int i = 0; i < n; ++i) {
    for (int c = 0; c < 6; ++c) tw[c] += vir[(size_t)c * n + i];
    te += elj[i];
    tc += ecl[i];
  }
  if (virial6)
    for (int c = 0; c < 6; ++c) virial6[c] = tw[c];
  if (evdwl) *evdwl = te;
  if (ecoul) *ecoul = tc;
  free(vir);
  free(elj);
  free(ecl);
}

/* DisplacementSq + max reduction (base_neighbor_list_builder.cpp:102-116, 270-283). */
double orc_max_disp2(int n, const orc_box* box, const double* x,
                     const double* y, const double* z, const double* x0,
                     const double* y0, const double* z0) {
  double m = 0.0;
#pragma omp parallel for schedule(static) reduction(max : m)
  for (int i = 0; i < n; ++i) {
    double dx = x[i] - x0[i], dy = y[i] - y0[i], dz = z[i] - z0[i];
    min_image_while(box, &dx, &dy, &dz);
    const double d2 = dx * dx + dy * dy + dz * dz;
    if (d2 > m) m = d2;
  }
  return m;
}

/* ========================================================================== */
/* Whole MD step on the host (CPU baseline): NVEensemble::Solve               */
/* (src/simulate_pipeline/src/nve_ensemble.cpp:59-91) with LJCutCoulKspace::   */
/* Execute (lj_cut_coul_kspace.cpp:464-471), RBL or Verlet real space.         */
/* ========================================================================== */
struct orc_engine {
  int n, ntypes, use_rbl, p, sample_num, freq, cap, rebuilds, have_cache;
  orc_box box;
  double sigma[64], eps[64], mass[64];
  double cut_off, r_core, skin, alpha, qqr2e, dt, S, qsq, qsum;
  uint64_t seed;
  int epoch;
  int *gid, *type, *perm, *cell, *cstart, *cend, *cand_count, *cand, *core_count, *core,
      *shell_count, *shell, *itmp;
  double *q, *x, *y, *z, *vx, *vy, *vz, *fx, *fy, *fz, *x0, *y0, *z0, *tmp;
  double *kfx, *kfy, *kfz, *mx, *my, *mz, *re, *im;
  int ncell;
  /* Nose-Hoover chain (NVT) */
  int nh_on;
  long long nh_num_steps;
  double nh_t_start, nh_t_stop, nh_t_freq, nh_kb, nh_mvv2e, nh_tdof;
  double eta[3], eta_dot[4], eta_dotdot[3], eta_mass[3], temperature, t_target, ke_target;
  /* unit style: force/mass*time -> velocity */
  double fmt2v;
  /* SHAKE clusters by gid (centre second) */
  int shake_nc, max_gid;
  int *shake_gid, *where;
  double shake_b1sq, shake_b2sq, shake_b12sq;
  double *xs, *ys, *zs;
  int shake_failures;
};

orc_engine* orc_engine_create(int n, const orc_box* box, int ntypes,
                              const double* sigma, const double* eps,
                              const double* mass, double cut_off, double r_core,
                              double skin, int neighbor_sample_num,
                              double alpha, int kspace_p, double qqr2e,
                              double dt, uint64_t seed, int use_rbl) {
  if (n <= 0 || ntypes <= 0 || ntypes > 64) return NULL;
  orc_engine* e = (orc_engine*)calloc(1, sizeof(orc_engine));
  e->n = n;
  e->ntypes = ntypes;
  e->box = *box;
  for (int t = 0; t < ntypes; ++t) {
    e->sigma[t] = sigma[t];
    e->eps[t] = eps[t];
    e->mass[t] = mass[t];
  }
  e->cut_off = cut_off;
  e->r_core = r_core;
  e->skin = skin;
  e->sample_num = neighbor_sample_num;
  e->alpha = alpha;
  e->p = kspace_p;
  e->qqr2e = qqr2e;
  e->dt = dt;
  e->seed = seed;
  e->use_rbl = use_rbl;
  e->fmt2v = 1.0;
  e->freq = orc_rbl_params(n, box, r_core, cut_off, neighbor_sample_num, NULL, NULL);
  e->S = orc_rbe_gauss_sum(box, alpha);
  int dims[3];
  e->ncell = orc_cell_grid(box, cut_off + skin, dims);
  const size_t N = (size_t)n;
#define A(ptr, T, cnt) ptr = (T*)calloc((cnt), sizeof(T))
  A(e->gid, int, N); A(e->type, int, N); A(e->perm, int, N); A(e->cell, int, N);
  A(e->itmp, int, N); A(e->cand_count, int, N); A(e->core_count, int, N);
  A(e->shell_count, int, N);
  A(e->cstart, int, e->ncell > 0 ? e->ncell : 1); A(e->cend, int, e->ncell > 0 ? e->ncell : 1);
  A(e->q, double, N); A(e->x, double, N); A(e->y, double, N); A(e->z, double, N);
  A(e->vx, double, N); A(e->vy, double, N); A(e->vz, double, N);
  A(e->fx, double, N); A(e->fy, double, N); A(e->fz, double, N);
  A(e->x0, double, N); A(e->y0, double, N); A(e->z0, double, N); A(e->tmp, double, N);
  A(e->kfx, double, N); A(e->kfy, double, N); A(e->kfz, double, N);
  A(e->mx, double, kspace_p); A(e->my, double, kspace_p); A(e->mz, double, kspace_p);
  A(e->re, double, kspace_p); A(e->im, double, kspace_p);
#undef A
  return e;
}

void orc_engine_destroy(orc_engine* e) {
  if (!e) return;
  void* ptrs[] = {e->gid, e->type, e->perm, e->cell, e->itmp, e->cand_count, e->core_count,
                  e->shell_count, e->cstart, e->cend, e->q, e->x, e->y, e->z, e->vx, e->vy,
                  e->vz, e->fx, e->fy, e->fz, e->x0, e->y0, e->z0, e->tmp, e->kfx, e->kfy,
                  e->kfz, e->mx, e->my, e->mz, e->re, e->im, e->cand, e->core, e->shell};
  for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); ++i) free(ptrs[i]);
  free(e->shake_gid);
  free(e->where);
  free(e->xs);
  free(e->ys);
  free(e->zs);
  free(e);
}

int orc_engine_set_state(orc_engine* e, const int* gid, const int* type,
                         const double* q, const double* x, const double* y,
                         const double* z, const double* vx, const double* vy,
                         const double* vz) {
  const size_t N = (size_t)e->n;
  memcpy(e->gid, gid, N * sizeof(int));
  memcpy(e->type, type, N * sizeof(int));
  memcpy(e->q, q, N * sizeof(double));
  memcpy(e->x, x, N * sizeof(double));
  memcpy(e->y, y, N * sizeof(double));
  memcpy(e->z, z, N * sizeof(double));
  memcpy(e->vx, vx, N * sizeof(double));
  memcpy(e->vy, vy, N * sizeof(double));
  memcpy(e->vz, vz, N * sizeof(double));
  e->qsq = 0;
  e->qsum = 0;
  for (int i = 0; i < e->n; ++i) {
    e->qsq += q[i] * q[i];
    e->qsum += q[i];
  }
  e->have_cache = 0;
  e->epoch = 0;
  return 0;
}

static void permute_d(double* a, const int* perm, double* tmp, int n) {
  for (int i = 0; i < n; ++i) tmp[i] = a[perm[i]];
  memcpy(a, tmp, sizeof(double) * (size_t)n);
}
static void permute_i(int* a, const int* perm, int* tmp, int n) {
  for (int i = 0; i < n; ++i) tmp[i] = a[perm[i]];
  memcpy(a, tmp, sizeof(int) * (size_t)n);
}

static int engine_rebuild(orc_engine* e) {
  const int n = e->n;
  if (orc_cells_sort(n, &e->box, e->cut_off + e->skin, e->x, e->y, e->z, e->perm, e->cell,
                     e->cstart, e->cend) <= 0)
    return -1;
  double* arrs[] = {e->q, e->x, e->y, e->z, e->vx, e->vy, e->vz, e->fx, e->fy, e->fz};
  for (size_t a = 0; a < sizeof(arrs) / sizeof(arrs[0]); ++a) permute_d(arrs[a], e->perm, e->tmp, n);
  permute_i(e->gid, e->perm, e->itmp, n);
  permute_i(e->type, e->perm, e->itmp, n);
  const int64_t maxc = orc_full_list(n, &e->box, e->cut_off + e->skin, e->x, e->y, e->z,
                                     e->cell, e->cstart, e->cend, 0, e->cand_count, NULL);
  if (maxc < 0) return -1;
  const int cap = (int)(maxc > 0 ? maxc : 1);
  if (cap > e->cap) {
    free(e->cand);
    free(e->core);
    free(e->shell);
    e->cand = (int*)malloc(sizeof(int) * (size_t)n * cap);
    e->core = (int*)malloc(sizeof(int) * (size_t)n * cap);
    e->shell = (int*)malloc(sizeof(int) * (size_t)n * cap);
    e->cap = cap;
  }
  orc_full_list(n, &e->box, e->cut_off + e->skin, e->x, e->y, e->z, e->cell, e->cstart,
                e->cend, e->cap, e->cand_count, e->cand);
  memcpy(e->x0, e->x, sizeof(double) * (size_t)n);
  memcpy(e->y0, e->y, sizeof(double) * (size_t)n);
  memcpy(e->z0, e->z, sizeof(double) * (size_t)n);
  e->have_cache = 1;
  e->rebuilds++;
  return 0;
}

int orc_engine_compute_forces(orc_engine* e, int epoch) {
  const int n = e->n;
  const double thr = e->skin * 0.5;
  int need = !e->have_cache || e->skin <= 0.0;
  if (!need) {
    const double md2 = orc_max_disp2(n, &e->box, e->x, e->y, e->z, e->x0, e->y0, e->z0);
    need = md2 > thr * thr;
  }
  if (need && engine_rebuild(e) != 0) return -1;
  if (e->use_rbl) {
    orc_rbl_filter(n, &e->box, e->r_core, e->cut_off, e->freq, epoch, e->gid, e->x, e->y, e->z,
                   e->cap, e->cand_count, e->cand, e->core_count, e->core, e->shell_count,
                   e->shell);
    orc_pair_force_rbl(n, &e->box, e->r_core, e->cut_off, e->freq, e->alpha, e->qqr2e, e->type,
                       e->sigma, e->eps, e->q, e->x, e->y, e->z, e->cap, e->core_count, e->core,
                       e->shell_count, e->shell, e->fx, e->fy, e->fz);
    orc_fix_rbl(n, e->fx, e->fy, e->fz, NULL);
  } else {
    orc_pair_force_verlet(n, &e->box, e->cut_off, e->alpha, e->qqr2e, e->type, e->sigma, e->eps,
                          e->q, e->x, e->y, e->z, e->cap, e->cand_count, e->cand, e->fx, e->fy,
                          e->fz, NULL, NULL, NULL);
  }
  if (e->p > 0) {
    if (orc_rbe_sample_philox(e->p, &e->box, e->alpha, e->seed, epoch, e->mx, e->my, e->mz) != 0)
      return -1;
    orc_rbe_structure_factor(n, e->p, &e->box, e->q, e->x, e->y, e->z, e->mx, e->my, e->mz,
                             e->re, e->im);
    orc_rbe_force(n, e->p, &e->box, e->S, e->qqr2e, e->re, e->im, e->q, e->mx, e->my, e->mz,
                  e->x, e->y, e->z, e->kfx, e->kfy, e->kfz);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      e->fx[i] += e->kfx[i];
      e->fy[i] += e->kfy[i];
      e->fz[i] += e->kfz[i];
    }
  }
  return 0;
}

/* UpdateVelocity (update_velocity_op.hip.cu:5-28, fmt2v = 1) and
 * UpdatePositionFlag + ApplyPBC (update_position_op.hip.cu:22-46, box.h:133-169). */
static void engine_kick(orc_engine* e) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < e->n; ++i) {
    const double m = e->mass[e->type[i]];
    e->vx[i] += 0.5 * e->fx[i] / m * e->dt * e->fmt2v;
    e->vy[i] += 0.5 * e->fy[i] / m * e->dt * e->fmt2v;
    e->vz[i] += 0.5 * e->fz[i] / m * e->dt * e->fmt2v;
  }
}

void orc_engine_set_fmt2v(orc_engine* e, double fmt2v) { e->fmt2v = fmt2v; }

/* ---- SHAKE / RATTLE of rigid 3-atom clusters ---------------------------- */
/* ShakeA / ShakeB of RBMD (shake_controller_op.hip.cu:19-389, 391-660),
 * restated: MinImageDistanceVec (box.h:115-131) = a - b with
 * d -= L rint(d / L). */
static void shk_sub(const orc_box* b, const double* a, const double* c, double* o) {
  for (int k = 0; k < 3; ++k) {
    const double L = box_len(b, k);
    o[k] = a[k] - c[k];
    o[k] -= L * rint(o[k] * (1.0 / L));
  }
}
static double shk_dot(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
static double shk_inv3(const double a[3][3], double ai[3][3]) {
  const double d = a[0][0] * a[1][1] * a[2][2] + a[0][1] * a[1][2] * a[2][0] +
                   a[0][2] * a[1][0] * a[2][1] - a[0][0] * a[1][2] * a[2][1] -
                   a[0][1] * a[1][0] * a[2][2] - a[0][2] * a[1][1] * a[2][0];
  const double r = 1 / d;
  ai[0][0] = r * (a[1][1] * a[2][2] - a[1][2] * a[2][1]);
  ai[0][1] = -r * (a[0][1] * a[2][2] - a[0][2] * a[2][1]);
  ai[0][2] = r * (a[0][1] * a[1][2] - a[0][2] * a[1][1]);
  ai[1][0] = -r * (a[1][0] * a[2][2] - a[1][2] * a[2][0]);
  ai[1][1] = r * (a[0][0] * a[2][2] - a[0][2] * a[2][0]);
  ai[1][2] = -r * (a[0][0] * a[1][2] - a[0][2] * a[1][0]);
  ai[2][0] = r * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
  ai[2][1] = -r * (a[0][0] * a[2][1] - a[0][1] * a[2][0]);
  ai[2][2] = r * (a[0][0] * a[1][1] - a[0][1] * a[1][0]);
  return d;
}

int orc_engine_set_shake(orc_engine* e, int nc, const int* cluster_gids, double bond,
                         double angle_deg) {
  free(e->shake_gid);
  free(e->where);
  e->shake_gid = NULL;
  e->where = NULL;
  e->shake_nc = 0;
  if (nc <= 0 || !(bond > 0)) return 0;
  int mg = 0;
  for (int i = 0; i < e->n; ++i) mg = e->gid[i] > mg ? e->gid[i] : mg;
  e->max_gid = mg;
  e->shake_gid = (int*)malloc(sizeof(int) * 3 * (size_t)nc);
  memcpy(e->shake_gid, cluster_gids, sizeof(int) * 3 * (size_t)nc);
  e->where = (int*)malloc(sizeof(int) * ((size_t)mg + 1));
  if (!e->xs) {
    e->xs = (double*)malloc(sizeof(double) * (size_t)e->n);
    e->ys = (double*)malloc(sizeof(double) * (size_t)e->n);
    e->zs = (double*)malloc(sizeof(double) * (size_t)e->n);
  }
  const double a = angle_deg / 180.0 * M_PI;
  e->shake_b1sq = e->shake_b2sq = bond * bond;
  const double b12 = sqrt(bond * bond + bond * bond - 2.0 * bond * bond * cos(a));
  e->shake_b12sq = b12 * b12;
  e->shake_nc = nc;
  e->shake_failures = 0;
  return 0;
}

int orc_engine_shake_failures(const orc_engine* e) { return e->shake_failures; }

static void shk_index(orc_engine* e) {
  for (int i = 0; i < e->n; ++i) e->where[e->gid[i]] = i;
}

static void shake_a(orc_engine* e) {
  shk_index(e);
  for (int c = 0; c < e->shake_nc; ++c) {
    int id[3];
    double po[3][3], pu[3][3], im[3];
    for (int k = 0; k < 3; ++k) {
      id[k] = e->where[e->shake_gid[3 * c + k]];
      po[k][0] = e->xs[id[k]];
      po[k][1] = e->ys[id[k]];
      po[k][2] = e->zs[id[k]];
      pu[k][0] = e->x[id[k]];
      pu[k][1] = e->y[id[k]];
      pu[k][2] = e->z[id[k]];
      im[k] = 1 / e->mass[e->type[id[k]]];
    }
    double r01[3], r12[3], r20[3], s10[3], s21[3], s02[3];
    shk_sub(&e->box, po[1], po[0], r01);
    shk_sub(&e->box, po[2], po[1], r12);
    shk_sub(&e->box, po[0], po[2], r20);
    shk_sub(&e->box, pu[0], pu[1], s10);
    shk_sub(&e->box, pu[1], pu[2], s21);
    shk_sub(&e->box, pu[2], pu[0], s02);
    const double r01sq = shk_dot(r01, r01), r02sq = shk_dot(r20, r20), r12sq = shk_dot(r12, r12);
    const double s01sq = shk_dot(s10, s10), s02sq = shk_dot(s02, s02), s12sq = shk_dot(s21, s21);
    double A[3][3], Ai[3][3];
    A[0][0] = 2 * (im[0] + im[1]) * shk_dot(s10, r01);
    A[0][1] = -2 * im[1] * shk_dot(s10, r12);
    A[0][2] = -2 * im[0] * shk_dot(s10, r20);
    A[1][0] = -2 * im[1] * shk_dot(s21, r01);
    A[1][1] = 2 * (im[1] + im[2]) * shk_dot(s21, r12);
    A[1][2] = -2 * im[2] * shk_dot(s21, r20);
    A[2][0] = -2 * im[0] * shk_dot(s02, r01);
    A[2][1] = -2 * im[2] * shk_dot(s02, r12);
    A[2][2] = 2 * (im[0] + im[2]) * shk_dot(s02, r20);
    const double det = shk_inv3(A, Ai);
    const double r0120 = shk_dot(r01, r20), r0112 = shk_dot(r01, r12), r2012 = shk_dot(r20, r12);
    /* coefficients of l01^2, l20^2, l12^2, l01 l20, l01 l12, l20 l12 */
    const double Q[3][6] = {
        {(im[0] + im[1]) * (im[0] + im[1]) * r01sq, im[0] * im[0] * r02sq, im[1] * im[1] * r12sq,
         -2 * (im[0] + im[1]) * im[0] * r0120, -2 * (im[0] + im[1]) * im[1] * r0112,
         2 * im[0] * im[1] * r2012},
        {im[1] * im[1] * r01sq, im[2] * im[2] * r02sq, (im[1] + im[2]) * (im[1] + im[2]) * r12sq,
         2 * im[1] * im[2] * r0120, -2 * (im[1] + im[2]) * im[1] * r0112,
         -2 * (im[1] + im[2]) * im[2] * r2012},
        {im[0] * im[0] * r01sq, (im[0] + im[2]) * (im[0] + im[2]) * r02sq, im[2] * im[2] * r12sq,
         -2 * (im[0] + im[2]) * im[0] * r0120, 2 * im[0] * im[2] * r0112,
         -2 * (im[0] + im[2]) * im[2] * r2012}};
    const double rhs0[3] = {e->shake_b1sq - s01sq, e->shake_b2sq - s12sq,
                            e->shake_b12sq - s02sq};
    double l01 = 0, l20 = 0, l12 = 0;
    int done = 0, overflow = 0, it = 0;
    while (!done && it < 5000) {
      const double t[6] = {l01 * l01, l20 * l20, l12 * l12, l01 * l20, l01 * l12, l20 * l12};
      double bq[3];
      for (int r = 0; r < 3; ++r) {
        double quad = Q[r][0] * t[0];
        for (int m = 1; m < 6; ++m) quad += Q[r][m] * t[m];
        bq[r] = rhs0[r] - quad;
      }
      const double n01 = Ai[0][0] * bq[0] + Ai[0][1] * bq[1] + Ai[0][2] * bq[2];
      const double n12 = Ai[1][0] * bq[0] + Ai[1][1] * bq[1] + Ai[1][2] * bq[2];
      const double n20 = Ai[2][0] * bq[0] + Ai[2][1] * bq[1] + Ai[2][2] * bq[2];
      done = fabs(n01 - l01) <= 1e-5 && fabs(n20 - l20) <= 1e-5 && fabs(n12 - l12) <= 1e-5;
      l01 = n01;
      l20 = n20;
      l12 = n12;
      if (isnan(l01) || isnan(l20) || isnan(l12) || fabs(l01) > 1e20 || fabs(l20) > 1e20 ||
          fabs(l12) > 1e20)
        done = overflow = 1;
      ++it;
    }
    if (!done || overflow || fabs(det) < 1e-4) e->shake_failures++;
    double* pos[3] = {e->x, e->y, e->z};
    double* vel[3] = {e->vx, e->vy, e->vz};
    for (int k = 0; k < 3; ++k) {
      const double d[3] = {l01 * r01[k] * im[0] - l20 * r20[k] * im[0],
                           l12 * r12[k] * im[1] - l01 * r01[k] * im[1],
                           l20 * r20[k] * im[2] - l12 * r12[k] * im[2]};
      const double L = box_len(&e->box, k);
      for (int a2 = 0; a2 < 3; ++a2) {
        vel[k][id[a2]] += d[a2] / e->dt;
        double p = pu[a2][k] + d[a2];
        if (p >= e->box.hi[k]) p -= L;
        if (p < e->box.lo[k]) p += L;
        pos[k][id[a2]] = p;
      }
    }
  }
}

static void shake_b(orc_engine* e) {
  shk_index(e);
  for (int c = 0; c < e->shake_nc; ++c) {
    int id[3];
    double p[3][3], v[3][3], im[3];
    for (int k = 0; k < 3; ++k) {
      id[k] = e->where[e->shake_gid[3 * c + k]];
      p[k][0] = e->x[id[k]];
      p[k][1] = e->y[id[k]];
      p[k][2] = e->z[id[k]];
      v[k][0] = e->vx[id[k]];
      v[k][1] = e->vy[id[k]];
      v[k][2] = e->vz[id[k]];
      im[k] = 1 / e->mass[e->type[id[k]]];
    }
    double r01[3], r12[3], r20[3], sv10[3], sv21[3], sv02[3];
    shk_sub(&e->box, p[1], p[0], r01);
    shk_sub(&e->box, p[2], p[1], r12);
    shk_sub(&e->box, p[0], p[2], r20);
    for (int k = 0; k < 3; ++k) {
      sv10[k] = v[0][k] - v[1][k];
      sv21[k] = v[1][k] - v[2][k];
      sv02[k] = v[2][k] - v[0][k];
    }
    double A[3][3], Ai[3][3];
    A[0][0] = (im[1] + im[0]) * shk_dot(r01, r01);
    A[0][1] = -im[1] * shk_dot(r01, r12);
    A[0][2] = -im[0] * shk_dot(r01, r20);
    A[1][0] = A[0][1];
    A[1][1] = (im[1] + im[2]) * shk_dot(r12, r12);
    A[1][2] = -im[2] * shk_dot(r20, r12);
    A[2][0] = A[0][2];
    A[2][1] = A[1][2];
    A[2][2] = (im[0] + im[2]) * shk_dot(r20, r20);
    const double c3[3] = {-shk_dot(sv10, r01), -shk_dot(sv21, r12), -shk_dot(sv02, r20)};
    if (fabs(shk_inv3(A, Ai)) < 1e-4) e->shake_failures++;
    double l[3];
    for (int r = 0; r < 3; ++r) l[r] = Ai[r][0] * c3[0] + Ai[r][1] * c3[1] + Ai[r][2] * c3[2];
    double* vel[3] = {e->vx, e->vy, e->vz};
    for (int k = 0; k < 3; ++k) {
      vel[k][id[0]] = v[0][k] + (l[0] * r01[k] * im[0] - l[2] * r20[k] * im[0]);
      vel[k][id[1]] = v[1][k] + (l[1] * r12[k] * im[1] - l[0] * r01[k] * im[1]);
      vel[k][id[2]] = v[2][k] + (l[2] * r20[k] * im[2] - l[1] * r12[k] * im[2]);
    }
  }
}
/* ShakeAOp / ShakeBOp at op level (shake_controller_op.hip.cu:1188-1238) for
 * atoms i = 0..n-1 with global ids gid[i], on caller arrays:
 * A: from the positions p (in the box) and velocities v before the step and
 * the forces f, the half kick and drift of the unconstrained update, then the
 * constraint; writes p (wrapped into the box, image counters img[3][n]
 * updated) and v.  B: RATTLE of v at positions p with the forces f of the new
 * positions after the second half kick; writes v.  Clusters are (H, O, H)
 * global-id triples; the constraint geometry is bond / angle_deg.  Returns
 * the number of clusters whose iteration failed. */
static void shk_view(orc_engine* e, int n, const orc_box* box, const int* gid, const int* type,
                     const double* mass, int ntypes, double dt, double fmt2v) {
  memset(e, 0, sizeof(*e));
  e->n = n;
  e->box = *box;
  e->dt = dt;
  e->fmt2v = fmt2v;
  e->gid = (int*)gid;
  e->type = (int*)type;
  for (int t = 0; t < ntypes && t < 64; ++t) e->mass[t] = mass[t];
}

int orc_shake_a_op(int n, const orc_box* box, const int* gid, const int* type, const double* mass,
                   int ntypes, double dt, double fmt2v, int nc, const int* clusters, double bond,
                   double angle_deg, double* px, double* py, double* pz, double* vx, double* vy,
                   double* vz, const double* fx, const double* fy, const double* fz, int* img) {
  orc_engine e;
  shk_view(&e, n, box, gid, type, mass, ntypes, dt, fmt2v);
  e.x = px; e.y = py; e.z = pz;
  e.vx = vx; e.vy = vy; e.vz = vz;
  e.fx = (double*)fx; e.fy = (double*)fy; e.fz = (double*)fz;
  if (orc_engine_set_shake(&e, nc, clusters, bond, angle_deg) != 0) return -1;
  engine_kick(&e);
  memcpy(e.xs, px, sizeof(double) * (size_t)n);
  memcpy(e.ys, py, sizeof(double) * (size_t)n);
  memcpy(e.zs, pz, sizeof(double) * (size_t)n);
  const double L[3] = {box_len(box, 0), box_len(box, 1), box_len(box, 2)};
  double* pos[3] = {px, py, pz};
  const double* vel[3] = {vx, vy, vz};
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) {
      double s = pos[d][i] + vel[d][i] * dt;
      if (s >= box->hi[d]) { s -= L[d]; if (img) img[d * n + i]++; }
      if (s < box->lo[d]) { s += L[d]; if (img) img[d * n + i]--; }
      pos[d][i] = s;
    }
  shake_a(&e);
  const int fails = e.shake_failures;
  free(e.shake_gid);
  free(e.where);
  free(e.xs);
  free(e.ys);
  free(e.zs);
  return fails;
}

int orc_shake_b_op(int n, const orc_box* box, const int* gid, const int* type, const double* mass,
                   int ntypes, double dt, double fmt2v, int nc, const int* clusters, double bond,
                   double angle_deg, const double* px, const double* py, const double* pz,
                   double* vx, double* vy, double* vz, const double* fx, const double* fy,
                   const double* fz) {
  orc_engine e;
  shk_view(&e, n, box, gid, type, mass, ntypes, dt, fmt2v);
  e.x = (double*)px; e.y = (double*)py; e.z = (double*)pz;
  e.vx = vx; e.vy = vy; e.vz = vz;
  e.fx = (double*)fx; e.fy = (double*)fy; e.fz = (double*)fz;
  if (orc_engine_set_shake(&e, nc, clusters, bond, angle_deg) != 0) return -1;
  engine_kick(&e);
  shake_b(&e);
  const int fails = e.shake_failures;
  free(e.shake_gid);
  free(e.where);
  free(e.xs);
  free(e.ys);
  free(e.zs);
  return fails;
}

static void engine_drift(orc_engine* e) {
  const double L[3] = {box_len(&e->box, 0), box_len(&e->box, 1), box_len(&e->box, 2)};
#pragma omp parallel for schedule(static)
  for (int i = 0; i < e->n; ++i) {
    double* p[3] = {&e->x[i], &e->y[i], &e->z[i]};
    const double v[3] = {e->vx[i], e->vy[i], e->vz[i]};
    for (int d = 0; d < 3; ++d) {
      double s = *p[d] + v[d] * e->dt;
      if (s >= e->box.hi[d]) s -= L[d];
      if (s < e->box.lo[d]) s += L[d];
      *p[d] = s;
    }
  }
}

/* ---- Nose-Hoover chain thermostat -------------------------------------- */
/* NoseHooverController (src/simulate_pipeline/src/controller/pressure_controller/
 * nose_hoover_controller.cpp): chain of 3, one sub-cycle, no drag.
 * Temperature: ComputeTemperature (update_temperature_op.hip.cu:7-29) and
 * SampleCurrentTemperatureState (:256-287), summed here in atom order. */
static double nh_temperature(const orc_engine* e) {
  double s = 0;
  for (int i = 0; i < e->n; ++i)
    s += e->nh_mvv2e * e->mass[e->type[i]] *
         (e->vx[i] * e->vx[i] + e->vy[i] * e->vy[i] + e->vz[i] * e->vz[i]);
  return 0.5 * s / (e->nh_tdof * e->nh_kb / 2.0);
}

/* ComputeTempTarget (:473-497). */
static void nh_temp_target(orc_engine* e, long long step) {
  double t = e->nh_t_start;
  if (e->nh_t_stop != e->nh_t_start) {
    double delta = (double)step;
    if (delta != 0.0) delta = delta / (double)e->nh_num_steps;
    t = e->nh_t_start + delta * (e->nh_t_stop - e->nh_t_start);
  }
  e->t_target = t;
  e->ke_target = e->nh_tdof * e->nh_kb * t;
}

/* NHCTempIntegrate (:732-840) with the velocity rescale it contains. */
static void nh_chain(orc_engine* e) {
  const double dt8 = 0.125 * e->dt, dt4 = 0.25 * e->dt, dthalf = 0.5 * e->dt;
  const double tf2 = e->nh_t_freq * e->nh_t_freq;
  double ke = e->nh_tdof * e->nh_kb * e->temperature;
  e->eta_mass[0] = e->nh_tdof * e->nh_kb * e->t_target / tf2;
  for (int c = 1; c < 3; ++c) e->eta_mass[c] = e->nh_kb * e->t_target / tf2;
  e->eta_dotdot[0] = e->eta_mass[0] > 0.0 ? (ke - e->ke_target) / e->eta_mass[0] : 0.0;
  for (int c = 2; c > 0; --c) {
    const double x = exp(-dt8 * e->eta_dot[c + 1]);
    e->eta_dot[c] = (e->eta_dot[c] * x + e->eta_dotdot[c] * dt4) * x;
  }
  const double x1 = exp(-dt8 * e->eta_dot[1]);
  e->eta_dot[0] = (e->eta_dot[0] * x1 + e->eta_dotdot[0] * dt4) * x1;
  const double f = exp(-dthalf * e->eta_dot[0]);
  for (int i = 0; i < e->n; ++i) {
    e->vx[i] *= f;
    e->vy[i] *= f;
    e->vz[i] *= f;
  }
  e->temperature = e->temperature * f * f;
  ke = e->nh_tdof * e->nh_kb * e->temperature;
  e->eta_dotdot[0] = e->eta_mass[0] > 0.0 ? (ke - e->ke_target) / e->eta_mass[0] : 0.0;
  for (int c = 0; c < 3; ++c) e->eta[c] += dthalf * e->eta_dot[c];
  e->eta_dot[0] = (e->eta_dot[0] * x1 + e->eta_dotdot[0] * dt4) * x1;
  for (int c = 1; c < 3; ++c) {
    const double x = exp(-dt8 * e->eta_dot[c + 1]);
    e->eta_dot[c] *= x;
    e->eta_dotdot[c] = (e->eta_mass[c - 1] * e->eta_dot[c - 1] * e->eta_dot[c - 1] -
                        e->nh_kb * e->t_target) / e->eta_mass[c];
    e->eta_dot[c] = (e->eta_dot[c] + e->eta_dotdot[c] * dt4) * x;
  }
}

/* Init + SetUp (:89-250, :415-471); t_damp <= 0 switches it off. */
int orc_engine_set_nose_hoover(orc_engine* e, double t_start, double t_stop, double t_damp,
                               long long num_steps, double kb, double mvv2e, double tdof) {
  if (!(t_damp > 0)) {
    e->nh_on = 0;
    return 0;
  }
  e->nh_on = 1;
  e->nh_t_start = t_start;
  e->nh_t_stop = t_stop;
  e->nh_t_freq = 1.0 / t_damp;
  e->nh_num_steps = num_steps;
  e->nh_kb = kb;
  e->nh_mvv2e = mvv2e;
  e->nh_tdof = tdof > 0 ? tdof : 3.0 * e->n - 3.0;
  for (int c = 0; c < 3; ++c) e->eta[c] = e->eta_dot[c] = e->eta_dotdot[c] = 0.0;
  e->eta_dot[3] = 0.0;
  e->temperature = nh_temperature(e);
  nh_temp_target(e, 0);
  const double tf2 = e->nh_t_freq * e->nh_t_freq;
  e->eta_mass[0] = e->nh_tdof * kb * e->t_target / tf2;
  for (int c = 1; c < 3; ++c) e->eta_mass[c] = kb * e->t_target / tf2;
  for (int c = 1; c < 3; ++c)
    e->eta_dotdot[c] = (e->eta_mass[c - 1] * e->eta_dot[c - 1] * e->eta_dot[c - 1] -
                        kb * e->t_target) / e->eta_mass[c];
  return 0;
}

void orc_engine_get_thermostat(const orc_engine* e, double* temperature, double* eta,
                               double* eta_dot) {
  if (temperature) *temperature = e->temperature;
  for (int c = 0; c < 3; ++c) {
    if (eta) eta[c] = e->eta[c];
    if (eta_dot) eta_dot[c] = e->eta_dot[c];
  }
}

/* NVEensemble::Solve, or NVTensemble::Solve with NOSE_HOOVER (nvt_ensemble.cpp:128-160):
 * InitialIntegrate = target + chain + kick + drift; force; FinalIntegrate =
 * kick + temperature + chain. */
int orc_engine_step(orc_engine* e, int nsteps) {
  if (!e->have_cache) {
    if (orc_engine_compute_forces(e, e->epoch) != 0) return -1;
  }
  for (int s = 0; s < nsteps; ++s) {
    if (e->nh_on) {
      nh_temp_target(e, (long long)e->epoch + 1);
      nh_chain(e);
    }
    engine_kick(e);
    if (e->shake_nc) {
      memcpy(e->xs, e->x, sizeof(double) * (size_t)e->n);
      memcpy(e->ys, e->y, sizeof(double) * (size_t)e->n);
      memcpy(e->zs, e->z, sizeof(double) * (size_t)e->n);
    }
    engine_drift(e);
    if (e->shake_nc) shake_a(e);
    e->epoch++;
    if (orc_engine_compute_forces(e, e->epoch) != 0) return -1;
    engine_kick(e);
    if (e->shake_nc) shake_b(e);
    if (e->nh_on) {
      e->temperature = nh_temperature(e);
      nh_chain(e);
    }
  }
  return 0;
}

int orc_engine_get(orc_engine* e, int* gid, double* x, double* y, double* z,
                   double* vx, double* vy, double* vz, double* fx, double* fy,
                   double* fz) {
  const size_t N = (size_t)e->n;
  if (gid) memcpy(gid, e->gid, N * sizeof(int));
  if (x) memcpy(x, e->x, N * sizeof(double));
  if (y) memcpy(y, e->y, N * sizeof(double));
  if (z) memcpy(z, e->z, N * sizeof(double));
  if (vx) memcpy(vx, e->vx, N * sizeof(double));
  if (vy) memcpy(vy, e->vy, N * sizeof(double));
  if (vz) memcpy(vz, e->vz, N * sizeof(double));
  if (fx) memcpy(fx, e->fx, N * sizeof(double));
  if (fy) memcpy(fy, e->fy, N * sizeof(double));
  if (fz) memcpy(fz, e->fz, N * sizeof(double));
  return 0;
}

int orc_engine_rebuilds(const orc_engine* e) { return e->rebuilds; }

/* ========================================================================== */
/* RBSOG k-space and VERLET-SOG real space                                    */
/* ========================================================================== */
/* rbsog_level presets (src/force/include/rbsog_level_preset.h:14-38). */
static const double kSogB[5] = {2.0, 1.62976708826776469, 1.48783512395703226,
                                1.32070036405934420, 1.21812525709410644};
static const double kSogSig[5] = {5.027010924194599, 3.633717409009413, 2.662784519725113,
                                  2.277149356440992, 1.774456369233284};
static const int kSogM[5] = {6, 16, 30, 64, 102};

typedef struct {
  int mmax;
  double b, sigma, w0, S, S_npt, self_coeff, taylor[6];
  double coef[128], coef_npt[128];
  int dm[18];
  double dfb[6], dfb_npt[6];
} orc_sog;

static double sog_g1(double r) { return exp(-r * r / 2.0) / sqrt(2 * M_PI); }

/* G^(m) = sum_l coef_l exp(-(b^2)^l sigma^2 k^2 / 2) (KSpaceCalculator::Gaussian,
 * kspace_calculator.cpp:1559-1573) */
static double sog_ghat(const orc_sog* s, const double* coef, double k2) {
  double sum = 0.0;
  for (int l = 0; l < s->mmax; ++l)
    sum += coef[l] * exp(-(pow(s->b * s->b, l + 0.0) * s->sigma * s->sigma) * k2 / 2.0);
  return sum;
}

/* RBSOGInit + RBSOGSetup (:988-1140), Compute_W01 (RBEPSample.h:19-34),
 * direct vectors and self term of ComputeRBSOG (:1423-1535), LJCoulSOGInit
 * (lj_cut_coul_kspace.cpp:651-711).  S keeps the reference's l = 0-only
 * high-k sum (its stop value is never reset between Gaussians). */
static int sog_setup(int level, double cut_off, const orc_box* box, orc_sog* s) {
  if (level < 0 || level > 4) return -1;
  memset(s, 0, sizeof(*s));
  s->b = kSogB[level];
  s->sigma = kSogSig[level] * cut_off / 10.0;
  s->mmax = kSogM[level];
  const double L[3] = {box_len(box, 0), box_len(box, 1), box_len(box, 2)};
  const double b = s->b, logb = log(b), r0 = cut_off / s->sigma;
  double acc = 0.0;
  for (int i = 1; i < 200; ++i) acc += pow(b, -i + 0.0) * sog_g1(pow(b, -i + 0.0) * r0);
  s->w0 = (1.0 / sog_g1(r0)) * ((1.0 / (2 * logb * r0)) - acc);
  const double sig2 = s->sigma * s->sigma, sig4 = sig2 * sig2;
  s->coef[0] = 4 * M_PI * logb * s->w0 * sig2;
  s->coef_npt[0] = 8 * M_PI * logb * s->w0 * sig4;
  for (int l = 1; l < s->mmax; ++l) {
    s->coef[l] = s->coef[l - 1] * (b * b);
    s->coef_npt[l] = s->coef_npt[l - 1] * (b * b * b * b);
  }
  double low = 0.0, low_npt = 0.0;
  const int ijk[4][3] = {{0, 0, 0}, {0, 0, 1}, {0, 1, 0}, {1, 0, 0}};
  for (int t = 0; t < 4; ++t) {
    double K[3], k2 = 0.0;
    for (int d = 0; d < 3; ++d) {
      K[d] = (2 * M_PI / L[d]) * (ijk[t][d] + 0.00);
      k2 += pow((ijk[t][d] + 0.00) * 2 * M_PI / L[d], 2);
    }
    const double K2 = K[0] * K[0] + K[1] * K[1] + K[2] * K[2];
    low += 2 * sog_ghat(s, s->coef, k2) * K2;
    low_npt += 2 * sog_ghat(s, s->coef_npt, k2) * (K2 * K2);
  }
  const double prd = fmax(L[0], fmax(L[1], L[2]));
  double sum = 0.0, sum_npt = 0.0, bound = 1.0, sl = sqrt(2.0) * s->sigma;
  for (int l = 0; l < s->mmax; ++l) {
    if (l > 0) sl *= b;
    double H[3] = {0, 0, 0}, Y[3] = {0, 0, 0}, Z[3] = {0, 0, 0};
    for (int j = 1; bound > 1e-12; ++j) {
      for (int d = 0; d < 3; ++d) {
        const double kd = M_PI * j / L[d];
        const double e = exp(-(kd * sl * kd * sl));
        H[d] += 2 * e;
        Y[d] += 2 * e * (4 * kd * kd);
        Z[d] += 2 * e * (16 * kd * kd * kd * kd);
      }
      const double km = M_PI * j / prd, km2 = km * km;
      bound = exp(4 * l * logb - km2 * (sl * sl)) * (km2 * km2) * sig4;
    }
    for (int d = 0; d < 3; ++d) H[d] += 1;
    sum += s->coef[l] * (Y[0] * H[1] * H[2] + H[0] * Y[1] * H[2] + H[0] * H[1] * Y[2]);
    sum_npt += s->coef_npt[l] * (Z[0] * H[1] * H[2] + H[0] * Z[1] * H[2] + H[0] * H[1] * Z[2] +
                                 2 * Y[0] * Y[1] * H[2] + 2 * Y[0] * H[1] * Y[2] +
                                 2 * H[0] * Y[1] * Y[2]);
  }
  s->S = sum - low;
  s->S_npt = sum_npt - low_npt;
  int nd = 0;
  for (int i = -1; i <= 1; ++i)
    for (int j = -1; j <= 1; ++j)
      for (int k = -1; k <= 1; ++k) {
        if ((i == 0 && j == 0 && k == 0) || i * i + j * j + k * k > 1) continue;
        const double Kx = (2 * M_PI / L[0]) * (i + 0.00), Ky = (2 * M_PI / L[1]) * (j + 0.00),
                     Kz = (2 * M_PI / L[2]) * (k + 0.00);
        s->dm[3 * nd] = i;
        s->dm[3 * nd + 1] = j;
        s->dm[3 * nd + 2] = k;
        s->dfb_npt[nd] = sog_ghat(s, s->coef_npt, Kx * Kx + Ky * Ky + Kz * Kz);
        s->dfb[nd++] = sog_ghat(s, s->coef, Kx * Kx + Ky * Ky + Kz * Kz);
      }
  s->self_coeff = (logb / (sqrt(2 * M_PI) * s->sigma)) *
                  (s->w0 + (1 - pow(b, -s->mmax + 0.0)) / (b - 1));
  const double ct = logb / (sig2 * sqrt(2 * M_PI * sig2));
  const double fact[6] = {1, 1, 2, 6, 24, 120};
  for (int i = 0; i < 6; ++i) {
    double ss = 0.0;
    for (int j = 0; j < s->mmax; ++j) {
      const double bl = pow(b, j + 0.0);
      const double w = j == 0 ? s->w0 : (1.0 / bl) * (1.0 / bl) * (1.0 / bl);
      ss += w * (1.0 / fact[i]) * pow(1.0 / (2.0 * sig2 * bl * bl), i + 0.0);
    }
    s->taylor[i] = pow(-1.0, i + 1.0) * 2.0 * ct * ss;
  }
  return 0;
}

int orc_rbsog_params(int level, double cut_off, const orc_box* box, double* scal,
                     double* coef, int* dm, double* dfb, double* coef_npt, double* dfb_npt) {
  orc_sog s;
  if (sog_setup(level, cut_off, box, &s)) return -1;
  /* scal: mmax, b, sigma, w0, S, S_npt, self_coeff, taylor[6] */
  const double v[13] = {(double)s.mmax, s.b, s.sigma, s.w0, s.S, s.S_npt, s.self_coeff,
                        s.taylor[0], s.taylor[1], s.taylor[2], s.taylor[3], s.taylor[4],
                        s.taylor[5]};
  memcpy(scal, v, sizeof v);
  if (coef) memcpy(coef, s.coef, sizeof(double) * (size_t)s.mmax);
  if (dm) memcpy(dm, s.dm, sizeof s.dm);
  if (dfb) memcpy(dfb, s.dfb, sizeof s.dfb);
  if (coef_npt) memcpy(coef_npt, s.coef_npt, sizeof(double) * (size_t)s.mmax);
  if (dfb_npt) memcpy(dfb_npt, s.dfb_npt, sizeof s.dfb_npt);
  return 0;
}

/* The NPT gather chain of RBSOGSampleKSpace (kspace_calculator.cpp:1242-1301):
 * idx[0] = 0; sample i proposes itself against the sample idx[i - 1] and is
 * accepted when u[i] < min(1, pup qup / (pdown qdown)) with
 * p(m) = Gaussian_modify(m) |k|^4 (coef_npt) and q(m) = Gaussian(m) |k|^2
 * (coef); u[i] are the caller's uniforms on [0, 1). */
int orc_rbsog_idx_npt(int level, double cut_off, const orc_box* box, int p, const double* mx,
                      const double* my, const double* mz, const double* u, int* idx) {
  orc_sog s;
  if (sog_setup(level, cut_off, box, &s)) return -1;
  if (p <= 0) return 0;
  const double L[3] = {box_len(box, 0), box_len(box, 1), box_len(box, 2)};
  idx[0] = 0;
  for (int i = 1; i < p; ++i) {
    const int o = idx[i - 1];
    const double mn[3] = {mx[i], my[i], mz[i]}, mo[3] = {mx[o], my[o], mz[o]};
    double k2n = 0.0, k2o = 0.0, K2n = 0.0, K2o = 0.0;
    for (int d = 0; d < 3; ++d) {
      k2n += pow((mn[d] + 0.00) * 2 * M_PI / L[d], 2);
      k2o += pow((mo[d] + 0.00) * 2 * M_PI / L[d], 2);
      const double kn = (2 * M_PI / L[d]) * mn[d], ko = (2 * M_PI / L[d]) * mo[d];
      K2n += kn * kn;
      K2o += ko * ko;
    }
    const double pup = sog_ghat(&s, s.coef_npt, k2n) * (K2n * K2n);
    const double qup = sog_ghat(&s, s.coef, k2o) * K2o;
    const double pdown = sog_ghat(&s, s.coef_npt, k2o) * (K2o * K2o);
    const double qdown = sog_ghat(&s, s.coef, k2n) * K2n;
    const double r = pup * qup / (pdown * qdown);
    const double acce = r > 1.0 ? 1.0 : r;
    idx[i] = u[i] < acce ? i : o;
  }
  return 0;
}

/* RBSOG k-space virial [6] (xx, yy, zz, xy, xz, yz) at a fixed box (fac =
 * fac_npt = 1): ComputeRBSOGSampleVirialKernel (kspace_calculator_op.hip.cu:
 * 1133-1190) over the P samples with K_npt = K[idx[j]], plus
 * ComputeRBSOGDirectVirialKernel (:1308-1355) over the 6 direct vectors.
 * S, S_npt <= 0 take RBSOGSetup's values. */
int orc_rbsog_virial(int level, double cut_off, const orc_box* box, double qqr2e, double S,
                     double S_npt, int n, int p, const double* q, const double* mx,
                     const double* my, const double* mz, const int* idx, const double* x,
                     const double* y, const double* z, double* virial) {
  orc_sog s;
  if (sog_setup(level, cut_off, box, &s)) return -1;
  const double L[3] = {box_len(box, 0), box_len(box, 1), box_len(box, 2)};
  const double V = L[0] * L[1] * L[2];
  const double Su = S > 0 ? S : s.S, Sn = S_npt > 0 ? S_npt : s.S_npt;
  const int pt = p + 6;
  double* K = (double*)malloc(sizeof(double) * 3 * (size_t)(pt > 0 ? pt : 1));
  double* r2 = (double*)calloc((size_t)(pt > 0 ? pt : 1), sizeof(double));
  for (int k = 0; k < pt; ++k) {
    const double m[3] = {k < p ? mx[k] : s.dm[3 * (k - p)], k < p ? my[k] : s.dm[3 * (k - p) + 1],
                         k < p ? mz[k] : s.dm[3 * (k - p) + 2]};
    for (int d = 0; d < 3; ++d) K[3 * k + d] = m[d] * (2 * M_PI / L[d]);
  }
#pragma omp parallel for schedule(static)
  for (int k = 0; k < pt; ++k) {
    double re = 0.0, im = 0.0;
    for (int i = 0; i < n; ++i) {
      const double ph = K[3 * k] * x[i] + K[3 * k + 1] * y[i] + K[3 * k + 2] * z[i];
      re += q[i] * cos(ph);
      im += q[i] * sin(ph);
    }
    r2[k] = re * re + im * im;
  }
  double v[6] = {0, 0, 0, 0, 0, 0};
  const double mv = (Su / p) * qqr2e / (2.0 * V), mn = -(Sn / p) * qqr2e / (4.0 * V);
  for (int j = 0; j < p; ++j) {
    const double* Kj = K + 3 * j;
    const double* Kn = K + 3 * idx[j];
    const double k2 = Kj[0] * Kj[0] + Kj[1] * Kj[1] + Kj[2] * Kj[2];
    const double kn2 = Kn[0] * Kn[0] + Kn[1] * Kn[1] + Kn[2] * Kn[2];
    const double c1 = r2[j] / k2, c2 = r2[idx[j]] / (kn2 * kn2);
    v[0] += c1 * mv + c2 * mn * Kn[0] * Kn[0];
    v[1] += c1 * mv + c2 * mn * Kn[1] * Kn[1];
    v[2] += c1 * mv + c2 * mn * Kn[2] * Kn[2];
    v[3] += c2 * mn * Kn[0] * Kn[1];
    v[4] += c2 * mn * Kn[0] * Kn[2];
    v[5] += c2 * mn * Kn[1] * Kn[2];
  }
  const double c1v = qqr2e / (2.0 * V), c2v = -qqr2e / (4.0 * V);
  for (int d = 0; d < 6; ++d) {
    const double* Kd = K + 3 * (p + d);
    const double a = c1v * s.dfb[d] * r2[p + d], b2 = c2v * s.dfb_npt[d] * r2[p + d];
    v[0] += a + b2 * Kd[0] * Kd[0];
    v[1] += a + b2 * Kd[1] * Kd[1];
    v[2] += a + b2 * Kd[2] * Kd[2];
    v[3] += b2 * Kd[0] * Kd[1];
    v[4] += b2 * Kd[0] * Kd[2];
    v[5] += b2 * Kd[1] * Kd[2];
  }
  memcpy(virial, v, sizeof v);
  free(K);
  free(r2);
  return 0;
}

/* Exact sampler of p(m) ~ G^(m)|k|^2 on |m|^2 > 1: a mixture over (l, axis d)
 * of separable densities k_d^2 g_l(m_d) prod_(d' != d) g_l(m_d'); one Philox
 * draw per component pick and axis, tables over m = 0, +1, -1, +2, ... */
typedef struct {
  int mmax, ncomp;
  double* comp;   /* cumulative [3 mmax] */
  double* tab;    /* concatenated cumulative tables */
  int off[6 * 128], cnt[6 * 128];
  double tot[6 * 128];
} sog_tables;

static int sog_tables_build(const orc_sog* s, const orc_box* box, sog_tables* t) {
  const double L[3] = {box_len(box, 0), box_len(box, 1), box_len(box, 2)};
  size_t total = 0;
  int M[128][3];
  for (int l = 0; l < s->mmax; ++l)
    for (int d = 0; d < 3; ++d) {
      const double kd = 2 * M_PI / L[d];
      const double a = pow(s->b * s->b, l + 0.0) * (s->sigma * s->sigma) * kd * kd / 2.0;
      M[l][d] = (int)ceil(sqrt(50.0 / a)) + 1;
      if (M[l][d] > (1 << 14)) return -1;
      total += 2 * (size_t)(2 * M[l][d] + 1);
    }
  t->mmax = s->mmax;
  t->ncomp = 3 * s->mmax;
  t->tab = (double*)malloc(sizeof(double) * total);
  t->comp = (double*)malloc(sizeof(double) * (size_t)t->ncomp);
  size_t pos = 0;
  for (int l = 0; l < s->mmax; ++l)
    for (int d = 0; d < 3; ++d) {
      const double kd = 2 * M_PI / L[d];
      const double a = pow(s->b * s->b, l + 0.0) * (s->sigma * s->sigma) * kd * kd / 2.0;
      for (int kind = 0; kind < 2; ++kind) {
        const int ti = (l * 3 + d) * 2 + kind;
        t->off[ti] = (int)pos;
        double acc = 0.0;
        for (int e = 0; e <= 2 * M[l][d]; ++e) {
          const int m = e == 0 ? 0 : ((e & 1) ? (e + 1) / 2 : -(e / 2));
          const double k = kd * m;
          acc += exp(-a * (double)m * (double)m) * (kind ? k * k : 1.0);
          t->tab[pos++] = acc;
        }
        t->cnt[ti] = 2 * M[l][d] + 1;
        t->tot[ti] = acc;
      }
    }
  double acc = 0.0;
  for (int l = 0; l < s->mmax; ++l)
    for (int d = 0; d < 3; ++d) {
      double w = s->coef[l];
      for (int a2 = 0; a2 < 3; ++a2) w *= t->tot[(l * 3 + a2) * 2 + (a2 == d ? 1 : 0)];
      acc += w;
      t->comp[l * 3 + d] = acc;
    }
  return 0;
}

static int sog_first_above(const double* cdf, int cnt, double target) {
  for (int i = 0; i < cnt; ++i)
    if (target < cdf[i]) return i;
  return cnt - 1;
}

static double sog_u53(uint32_t hi, uint32_t lo) {
  return (double)(((((uint64_t)hi) << 32) | lo) >> 11) * (1.0 / 9007199254740992.0);
}

/* Uniforms of the device NPT chain: Philox4x32-10 of counter
 * {i, 0x4e505400, step lo, step hi} under the sampler's key, u = the top 53
 * bits of the first two words. */
void orc_rbsog_npt_uniforms(uint64_t seed, int64_t step, int p, double* u) {
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  for (int i = 0; i < p; ++i) {
    const uint32_t c0[4] = {(uint32_t)i, 0x4e505400u, (uint32_t)step,
                            (uint32_t)((uint64_t)step >> 32)};
    uint32_t c[4];
    orc_philox4x32_10(c0, key, c);
    u[i] = sog_u53(c[0], c[1]);
  }
}

int orc_rbsog_sample_philox(int level, double cut_off, const orc_box* box, int p, uint64_t seed,
                            int64_t step, double* mx, double* my, double* mz) {
  orc_sog s;
  sog_tables t;
  if (sog_setup(level, cut_off, box, &s) || sog_tables_build(&s, box, &t)) return -1;
  int rc = 0;
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  for (int i = 0; i < p && !rc; ++i) {
    int done = 0;
    for (int a = 0; a < 64 && !done; ++a) {
      const uint32_t c0[4] = {(uint32_t)i, (uint32_t)(2 * a), (uint32_t)step,
                              (uint32_t)((uint64_t)step >> 32)};
      const uint32_t d0[4] = {(uint32_t)i, (uint32_t)(2 * a + 1), (uint32_t)step,
                              (uint32_t)((uint64_t)step >> 32)};
      uint32_t c[4], d[4];
      orc_philox4x32_10(c0, key, c);
      orc_philox4x32_10(d0, key, d);
      const int comp = sog_first_above(t.comp, t.ncomp, sog_u53(c[0], c[1]) * t.comp[t.ncomp - 1]);
      const int l = comp / 3, dd = comp - 3 * l;
      const double u[3] = {sog_u53(c[2], c[3]), sog_u53(d[0], d[1]), sog_u53(d[2], d[3])};
      int m[3];
      for (int ax = 0; ax < 3; ++ax) {
        const int ti = (l * 3 + ax) * 2 + (ax == dd ? 1 : 0);
        const int e = sog_first_above(t.tab + t.off[ti], t.cnt[ti], u[ax] * t.tot[ti]);
        m[ax] = e == 0 ? 0 : ((e & 1) ? (e + 1) / 2 : -(e / 2));
      }
      if (m[0] * m[0] + m[1] * m[1] + m[2] * m[2] > 1) {
        mx[i] = m[0];
        my[i] = m[1];
        mz[i] = m[2];
        done = 1;
      }
    }
    if (!done) rc = -2;
  }
  free(t.tab);
  free(t.comp);
  return rc;
}

/* RBSOGSampleKSpace's Metropolis chain (kspace_calculator.cpp:1142-1240):
 * proposals round(N(0, L / (2 pi sigma))) per axis, acceptance
 * min(1, p(new) q(old) / (p(old) q(new))) with p = G^(m)|k|^2 and q the
 * discretised-Gaussian mass MH_D_Modify (:1669-1677); |m|^2 <= 1 redrawn; the
 * odd entries of a chain of 2P are the samples.  Seeded SplitMix64 uniforms
 * stand in for the reference's unseeded std::random_device stream. */
static double sog_q(int m, double f) {
  return m == 0 ? erf(0.5 * f) : 0.5 * (erf((abs(m) + 0.5) * f) - erf((abs(m) - 0.5) * f));
}

int orc_rbsog_sample_mh(int level, double cut_off, const orc_box* box, int p, uint64_t seed,
                        double* mx, double* my, double* mz) {
  orc_sog s;
  if (sog_setup(level, cut_off, box, &s)) return -1;
  const double L[3] = {box_len(box, 0), box_len(box, 1), box_len(box, 2)};
  orc_rng r = {seed};
  double fac[3], mhd[3];
  for (int d = 0; d < 3; ++d) {
    fac[d] = L[d] / (2 * M_PI * s.sigma);
    mhd[d] = sqrt(2 * s.sigma * s.sigma * M_PI * M_PI) / L[d];
  }
  const int n = 2 * p;
  int* cx = (int*)malloc(sizeof(int) * 3 * (size_t)n);
#define PDENS(m)                                                                                \
  (sog_ghat(&s, s.coef,                                                                         \
            pow((m)[0] * 2 * M_PI / L[0], 2) + pow((m)[1] * 2 * M_PI / L[1], 2) +                \
                pow((m)[2] * 2 * M_PI / L[2], 2)) *                                              \
   (pow((m)[0] * 2 * M_PI / L[0], 2) + pow((m)[1] * 2 * M_PI / L[1], 2) +                       \
    pow((m)[2] * 2 * M_PI / L[2], 2)))
  do {
    for (int d = 0; d < 3; ++d) cx[d] = (int)round(mh_gauss(&r, fac[d]));
  } while (cx[0] == 0 && cx[1] == 0 && cx[2] == 0);
  for (int i = 0; i < n - 1; ++i) {
    int mo[3], mn[3];
    for (int d = 0; d < 3; ++d) {
      mn[d] = (int)round(mh_gauss(&r, fac[d]));
      mo[d] = cx[3 * i + d];
    }
    const double pu = PDENS(mn) * sog_q(mo[0], mhd[0]) * sog_q(mo[1], mhd[1]) * sog_q(mo[2], mhd[2]);
    const double pd = PDENS(mo) * sog_q(mn[0], mhd[0]) * sog_q(mn[1], mhd[1]) * sog_q(mn[2], mhd[2]);
    const double acc = pu / pd > 1.0 ? 1.0 : pu / pd;
    const int* pick = rng_uniform(&r) < acc ? mn : mo;
    for (int d = 0; d < 3; ++d) cx[3 * (i + 1) + d] = pick[d];
    const int* q = cx + 3 * (i + 1);
    if (q[0] * q[0] + q[1] * q[1] + q[2] * q[2] <= 1) i = i - 1;
  }
#undef PDENS
  for (int i = 0; i < p; ++i) {
    mx[i] = cx[3 * (2 * i + 1)];
    my[i] = cx[3 * (2 * i + 1) + 1];
    mz[i] = cx[3 * (2 * i + 1) + 2];
  }
  free(cx);
  return 0;
}

/* ComputeRBSOG's force and energy for given samples: the sampled vectors
 * (c_k = -(S/P) qqr2e / (V k^2)) and the six direct ones (c_k = -qqr2e G^/V),
 * rho by ComputePnumberChargeStructureFactorSOG, energies of
 * ComputeRBSOGSample/DirectEnergyKernel and the self term (:1525-1535).
 * S <= 0: RBSOGSetup's S. */
int orc_rbsog_force(int level, double cut_off, const orc_box* box, double qqr2e, double S, int n,
                    int p, const double* q, const double* mx, const double* my,
                    const double* mz, const double* x, const double* y, const double* z,
                    double* fx, double* fy, double* fz, double* energy) {
  orc_sog s;
  if (sog_setup(level, cut_off, box, &s)) return -1;
  const double L[3] = {box_len(box, 0), box_len(box, 1), box_len(box, 2)};
  const double V = L[0] * L[1] * L[2], Su = S > 0 ? S : s.S;
  const int pt = p + 6;
  double* K = (double*)malloc(sizeof(double) * 3 * (size_t)pt);
  double* c = (double*)malloc(sizeof(double) * (size_t)pt);
  double* re = (double*)calloc((size_t)pt, sizeof(double));
  double* im = (double*)calloc((size_t)pt, sizeof(double));
  double e = 0.0;
  for (int k = 0; k < pt; ++k) {
    const double m[3] = {k < p ? mx[k] : s.dm[3 * (k - p)], k < p ? my[k] : s.dm[3 * (k - p) + 1],
                         k < p ? mz[k] : s.dm[3 * (k - p) + 2]};
    for (int d = 0; d < 3; ++d) K[3 * k + d] = 2 * M_PI * m[d] / L[d];
  }
#pragma omp parallel for schedule(static)
  for (int k = 0; k < pt; ++k) {
    double r = 0.0, ii = 0.0;
    for (int i = 0; i < n; ++i) {
      const double ph = K[3 * k] * x[i] + K[3 * k + 1] * y[i] + K[3 * k + 2] * z[i];
      r += q[i] * cos(ph);
      ii += q[i] * sin(ph);
    }
    re[k] = r;
    im[k] = ii;
  }
  for (int k = 0; k < pt; ++k) {
    const double k2 = K[3 * k] * K[3 * k] + K[3 * k + 1] * K[3 * k + 1] + K[3 * k + 2] * K[3 * k + 2];
    const double r2 = re[k] * re[k] + im[k] * im[k];
    if (k < p) {
      c[k] = -(Su / p) * qqr2e / V / k2;
      e += (Su / (2.0 * p * V)) * qqr2e * r2 / k2;
    } else {
      c[k] = -qqr2e / V * s.dfb[k - p];
      e += qqr2e / (2.0 * V) * s.dfb[k - p] * r2;
    }
  }
  double qsq = 0.0;
  for (int i = 0; i < n; ++i) qsq += q[i] * q[i];
  e += -s.self_coeff * qsq * qqr2e;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    double f[3] = {0, 0, 0};
    for (int k = 0; k < pt; ++k) {
      const double ph = K[3 * k] * x[i] + K[3 * k + 1] * y[i] + K[3 * k + 2] * z[i];
      const double t = (cos(ph) * im[k] - sin(ph) * re[k]) * c[k];
      for (int d = 0; d < 3; ++d) f[d] += q[i] * t * K[3 * k + d];
    }
    fx[i] = f[0];
    fy[i] = f[1];
    fz[i] = f[2];
  }
  if (energy) *energy = e;
  free(K);
  free(c);
  free(re);
  free(im);
  return 0;
}

/* The far field the sampled sum estimates, summed exactly: all m with
 * |m_d| <= mcut and |m|^2 > 1, weight G^(m) (the sampled estimator's
 * expectation is S / S_full times this, S_full = sum G^(m) |k|^2 over the
 * same m, written to *S_full). */
int orc_rbsog_far_exact(int level, double cut_off, const orc_box* box, double qqr2e, int n,
                        const double* q, const double* x, const double* y, const double* z,
                        int mcut, double* fx, double* fy, double* fz, double* S_full) {
  orc_sog s;
  if (sog_setup(level, cut_off, box, &s)) return -1;
  const double L[3] = {box_len(box, 0), box_len(box, 1), box_len(box, 2)};
  const double V = L[0] * L[1] * L[2];
  const int side = 2 * mcut + 1;
  const int nk = side * side * side;
  double* K = (double*)malloc(sizeof(double) * 4 * (size_t)nk);
  int cntk = 0;
  double Sf = 0.0;
  for (int a = -mcut; a <= mcut; ++a)
    for (int b = -mcut; b <= mcut; ++b)
      for (int c = -mcut; c <= mcut; ++c) {
        if (a * a + b * b + c * c <= 1) continue;
        double* k = K + 4 * (size_t)cntk++;
        k[0] = 2 * M_PI * a / L[0];
        k[1] = 2 * M_PI * b / L[1];
        k[2] = 2 * M_PI * c / L[2];
        const double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
        k[3] = sog_ghat(&s, s.coef, k2);
        Sf += k[3] * k2;
      }
  double* re = (double*)calloc((size_t)cntk, sizeof(double));
  double* im = (double*)calloc((size_t)cntk, sizeof(double));
#pragma omp parallel for schedule(static)
  for (int k = 0; k < cntk; ++k) {
    double r = 0.0, ii = 0.0;
    for (int i = 0; i < n; ++i) {
      const double ph = K[4 * k] * x[i] + K[4 * k + 1] * y[i] + K[4 * k + 2] * z[i];
      r += q[i] * cos(ph);
      ii += q[i] * sin(ph);
    }
    re[k] = r;
    im[k] = ii;
  }
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    double f[3] = {0, 0, 0};
    for (int k = 0; k < cntk; ++k) {
      const double ph = K[4 * k] * x[i] + K[4 * k + 1] * y[i] + K[4 * k + 2] * z[i];
      const double t = (cos(ph) * im[k] - sin(ph) * re[k]) * (-qqr2e / V * K[4 * k + 3]);
      for (int d = 0; d < 3; ++d) f[d] += q[i] * t * K[4 * k + d];
    }
    fx[i] = f[0];
    fy[i] = f[1];
    fz[i] = f[2];
  }
  if (S_full) *S_full = Sf;
  free(K);
  free(re);
  free(im);
  return 0;
}

/* VERLET-SOG pair force (ComputeLJCutCoulForceUserKernel with lj126 and
 * CoulCutForceUser, lj_cut_coul_kspace_op.hip.cu:196-254, 357-470, lj_op.hip.cu:18-37). */
void orc_pair_force_verlet_sog(int level, double cut_off, const orc_box* box, double qqr2e,
                               int n, const int* type, const double* sigma, const double* eps,
                               const double* q, const double* x, const double* y,
                               const double* z, int cap, const int* count, const int* cand,
                               double* fx, double* fy, double* fz, double* energy,
                               double* flat_virial) {
  orc_sog s;
  if (sog_setup(level, cut_off, box, &s)) return;
  const double cut2 = cut_off * cut_off;
  double elj = 0.0, ecl = 0.0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : elj, ecl)
  for (int i = 0; i < n; ++i) {
    double f[3] = {0, 0, 0}, v[6] = {0, 0, 0, 0, 0, 0};
    for (int t = 0; t < count[i]; ++t) {
      const int j = cand[(size_t)i * cap + t];
      double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
      min_image_while(box, &dx, &dy, &dz);
      const double d2 = dx * dx + dy * dy + dz * dz;
      if (!(d2 < cut2)) continue;
      const double eij = sqrt(eps[type[i]] * eps[type[j]]);
      const double sij = (sigma[type[i]] + sigma[type[j]]) / 2;
      const double s6 = pow(sij, 6.0), d6 = pow(d2, 3.0), sd6 = s6 / d6;
      const double flj = -24 * eij * ((2 * sd6 - 1) * sd6) / d2;
      const double r2inv = 1.0 / d2, rinv = sqrt(r2inv), r3inv = rinv * r2inv;
      const double pre = qqr2e * q[i] * q[j];
      const double poly = s.taylor[0] + s.taylor[1] * d2 + s.taylor[2] * pow(d2, 2.0) +
                          s.taylor[3] * pow(d2, 3.0) + s.taylor[4] * pow(d2, 4.0) +
                          s.taylor[5] * pow(d2, 5.0);
      const double fp = flj + (-pre * (r3inv + poly));
      f[0] += dx * fp;
      f[1] += dy * fp;
      f[2] += dz * fp;
      /* ComputeVirial (lj_op.hip.cu:76-88) of the pair force */
      v[0] += -0.5 * dx * dx * fp;
      v[1] += -0.5 * dy * dy * fp;
      v[2] += -0.5 * dz * dz * fp;
      v[3] += -0.5 * dx * dy * fp;
      v[4] += -0.5 * dx * dz * fp;
      v[5] += -0.5 * dy * dz * fp;
      elj += 0.5 * (4 * eij * (s6 / d6 - 1) * sd6);
      const double norm = 2.0 * log(s.b) / sqrt(2.0 * M_PI * s.sigma * s.sigma);
      double sume = norm * s.w0 * exp(-d2 / (2.0 * s.sigma * s.sigma));
      for (int l = 1; l < s.mmax; ++l)
        sume += norm * (1.0 / pow(s.b, l + 0.00)) *
                exp(-d2 / (2 * s.sigma * s.sigma * pow(s.b, l + 0.00) * pow(s.b, l + 0.00)));
      ecl += 0.5 * pre * (rinv - sume);
    }
    fx[i] = f[0];
    fy[i] = f[1];
    fz[i] = f[2];
    if (flat_virial)
      for (int c = 0; c < 6; ++c) flat_virial[(size_t)c * n + i] = v[c];
  }
  if (energy) {
    energy[0] = elj;
    energy[1] = ecl;
  }
}
