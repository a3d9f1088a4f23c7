// rbsog.cpp -- see rbsog.h.
//
// Follows KSpaceCalculator::Init's RBSOG branch (src/force/src/
// kspace_calculator.cpp:253-330), RBSOGInit (:988-1042), RBSOGSetup
// (:1044-1140), the direct-sum vectors and self energy of ComputeRBSOG
// (:1423-1535), Compute_W01 (src/common/RBEPSample.h:19-34) and
// LJCutCoulKspace::LJCoulSOGInit (src/force/src/lj_cut_coul_kspace.cpp:651-711).
// Two properties of the reference are kept as they are, so that forces match:
// every Gaussian's Fourier weight carries w0 (coef[l] = coef[0] b^(2l); the
// l = 1 assignment in RBSOGInit is overwritten by the recurrence), and S's
// high-k sum holds only the l = 0 Gaussian (the loop's stop value is not reset
// between Gaussians, so the loop body runs for l = 0 only).
#include "rbsog.h"

#include <cmath>
#include <stdexcept>
#include <string>

namespace rbx_host {
namespace {

struct Preset {
  double b, sigma_at_rc10, target_accuracy;
  int mmax;
};
// rbsog_level presets (src/force/include/rbsog_level_preset.h:14-38)
const Preset kPresets[5] = {
    {2.0, 5.027010924194599, 2.289e-3, 6},
    {1.62976708826776469, 3.633717409009413, 1.158e-4, 16},
    {1.48783512395703226, 2.662784519725113, 1.142e-5, 30},
    {1.32070036405934420, 2.277149356440992, 5.583e-8, 64},
    {1.21812525709410644, 1.774456369233284, 3.389e-11, 102},
};

double g_sigma(double s, double r) { return std::exp(-r * r / (2 * s * s)) / std::sqrt(2 * M_PI * s * s); }

double w0_of(double r0, double b) {
  double sum = 0.0;
  for (int i = 1; i < 200; ++i) sum += std::pow(b, -i + 0.0) * g_sigma(1.0, std::pow(b, -i + 0.0) * r0);
  return (1.0 / g_sigma(1.0, r0)) * ((1.0 / (2 * std::log(b) * r0)) - sum);
}

// KSpaceCalculator::Gaussian (:1559-1573): sum_l coef_l exp(-b^(2l) sigma^2 k^2 / 2)
double gaussian_k(double k2, const RbsogSetup& s, const std::vector<double>& coef) {
  double sum = 0.0;
  const double b2 = s.b * s.b;
  for (int i = 0; i < s.mmax; ++i)
    sum += coef[i] * std::exp(-(std::pow(b2, i + 0.0) * s.sigma * s.sigma) * k2 / 2.0);
  return sum;
}

double k2_of(int i, int j, int k, const double L[3]) {
  return std::pow((i + 0.00) * 2 * M_PI / L[0], 2) + std::pow((j + 0.00) * 2 * M_PI / L[1], 2) +
         std::pow((k + 0.00) * 2 * M_PI / L[2], 2);
}

}  // namespace

RbsogSetup rbsog_setup(int level, double cut_off, const rbx_box& box) {
  if (level < 0 || level > 4)
    throw std::runtime_error("RBSOG rbsog_level must be in [0, 4]. Current value: " +
                             std::to_string(level));
  if (!(cut_off > 0)) throw std::runtime_error("RBSOG needs cut_off > 0");
  RbsogSetup s;
  const Preset& p = kPresets[level];
  s.level = level;
  s.b = p.b;
  s.sigma = p.sigma_at_rc10 * cut_off / 10.0;
  s.mmax = p.mmax;
  const double L[3] = {box.hi[0] - box.lo[0], box.hi[1] - box.lo[1], box.hi[2] - box.lo[2]};
  for (double l : L)
    if (!(l > 0)) throw std::runtime_error("RBSOG needs a box of positive size");
  // RBSOGInit
  s.w0 = w0_of(cut_off / s.sigma, s.b);
  const double sigma2 = s.sigma * s.sigma, sigma4 = sigma2 * sigma2;
  const double b2 = s.b * s.b, b4 = b2 * b2, logb = std::log(s.b);
  s.coef.resize(s.mmax);
  s.coef_npt.resize(s.mmax);
  s.coef[0] = 4 * M_PI * logb * s.w0 * sigma2;
  s.coef_npt[0] = 8 * M_PI * logb * s.w0 * sigma4;
  for (int i = 1; i < s.mmax; ++i) {
    s.coef[i] = s.coef[i - 1] * b2;
    s.coef_npt[i] = s.coef_npt[i - 1] * b4;
  }
  // RBSOGSetup: low-k part (i, j, k in [0, Kcut], i^2 + j^2 + k^2 <= Kcut = 1)
  const int kcut = 1;
  double sum_1 = 0, sum_npt_1 = 0;
  for (int i = 0; i < kcut + 1; ++i)
    for (int j = 0; j < kcut + 1; ++j)
      for (int k = 0; k < kcut + 1; ++k)
        if (i * i + j * j + k * k <= kcut) {
          const double Kx = (2 * M_PI / L[0]) * (i + 0.00), Ky = (2 * M_PI / L[1]) * (j + 0.00),
                       Kz = (2 * M_PI / L[2]) * (k + 0.00);
          const double K2 = Kx * Kx + Ky * Ky + Kz * Kz, K4 = K2 * K2;
          const double k2 = k2_of(i, j, k, L);
          sum_1 += 2 * gaussian_k(k2, s, s.coef) * K2;
          sum_npt_1 += 2 * gaussian_k(k2, s, s.coef_npt) * K4;
        }
  // high-k part, analytic in each axis; the stop value carries over (see top)
  const double prd = std::max(L[0], std::max(L[1], L[2]));
  std::vector<double> sl(s.mmax);  // widths s_l: sqrt(2) sigma b^l by recurrence
  sl[0] = std::sqrt(2.0) * s.sigma;
  for (int i = 1; i < s.mmax; ++i) sl[i] = sl[i - 1] * s.b;
  double sum = 0, sum_npt = 0, bound = 1.0;
  for (int i = 0; i < s.mmax; ++i) {
    double H[3] = {0, 0, 0}, Y[3] = {0, 0, 0}, YY[3] = {0, 0, 0};
    const double sl_i = sl[i], sl_sq = sl_i * sl_i;
    int j = 1;
    while (bound > 1e-12) {
      for (int d = 0; d < 3; ++d) {
        const double kd = M_PI * j / L[d];
        const double e = std::exp(-(kd * sl_i * kd * sl_i));
        H[d] += 2 * e;
        Y[d] += 2 * e * (4 * kd * kd);
        YY[d] += 2 * e * (16 * kd * kd * kd * kd);
      }
      const double kmin = M_PI * j / prd, kmin2 = kmin * kmin;
      ++j;
      bound = std::exp(4 * i * logb - kmin2 * sl_sq) * (kmin2 * kmin2) * sigma4;
    }
    for (double& h : H) h += 1;
    sum += s.coef[i] * (Y[0] * H[1] * H[2] + H[0] * Y[1] * H[2] + H[0] * H[1] * Y[2]);
    sum_npt += s.coef_npt[i] * (YY[0] * H[1] * H[2] + H[0] * YY[1] * H[2] + H[0] * H[1] * YY[2] +
                                2 * Y[0] * Y[1] * H[2] + 2 * Y[0] * H[1] * Y[2] +
                                2 * H[0] * Y[1] * Y[2]);
  }
  s.S = sum - sum_1;
  s.S_npt = sum_npt - sum_npt_1;
  // direct-sum vectors (ComputeRBSOG :1425-1451): loops -1..1, |m|^2 <= Kcut, m != 0
  for (int i = -1; i <= 1; ++i)
    for (int j = -1; j <= 1; ++j)
      for (int k = -1; k <= 1; ++k)
        if (!(i == 0 && j == 0 && k == 0) && i * i + j * j + k * k <= kcut) {
          const double Kx = (2 * M_PI / L[0]) * (i + 0.00), Ky = (2 * M_PI / L[1]) * (j + 0.00),
                       Kz = (2 * M_PI / L[2]) * (k + 0.00);
          s.direct_m.insert(s.direct_m.end(), {i, j, k});
          s.direct_fb.push_back(gaussian_k(Kx * Kx + Ky * Ky + Kz * Kz, s, s.coef));
          s.direct_fb_npt.push_back(gaussian_k(Kx * Kx + Ky * Ky + Kz * Kz, s, s.coef_npt));
        }
  s.self_coeff = (logb / (std::sqrt(2 * M_PI) * s.sigma)) *
                 (s.w0 + (1 - std::pow(s.b, -s.mmax + 0.0)) / (s.b - 1));
  // LJCoulSOGInit: Taylor coefficients of the short-range force
  {
    std::vector<double> bl3_inv(s.mmax), inv2(s.mmax);
    for (int i = 0; i < s.mmax; ++i) {
      const double bl = std::pow(s.b, i + 0.0), bl_inv = 1.0 / bl;
      bl3_inv[i] = bl_inv * bl_inv * bl_inv;
      inv2[i] = 1.0 / (2.0 * s.sigma * s.sigma * bl * bl);
    }
    bl3_inv[0] = s.w0;
    const double c = logb / (s.sigma * s.sigma * std::sqrt(2 * M_PI * s.sigma * s.sigma));
    const double fact[6] = {1, 1, 2, 6, 24, 120};
    for (int i = 0; i < 6; ++i) {
      double ss = 0.0;
      for (int j = 0; j < s.mmax; ++j) ss += bl3_inv[j] * (1.0 / fact[i]) * std::pow(inv2[j], i + 0.0);
      s.taylor[i] = std::pow(-1.0, i + 1.0) * 2.0 * c * ss;
    }
  }
  // sampler tables: per (l, axis) the 1-D factors exp(-a m^2) and k^2 exp(-a m^2)
  s.tab_off.assign(s.mmax * 6, 0);
  s.tab_cnt.assign(s.mmax * 6, 0);
  s.tab_tot.assign(s.mmax * 6, 0.0);
  for (int l = 0; l < s.mmax; ++l)
    for (int d = 0; d < 3; ++d) {
      const double kd = 2 * M_PI / L[d];
      const double a = std::pow(b2, l + 0.0) * sigma2 * kd * kd / 2.0;
      int M = (int)std::ceil(std::sqrt(50.0 / a)) + 1;
      if (M > (1 << 14))
        throw std::runtime_error("RBSOG: box too large for the sampler tables (" +
                                 std::to_string(M) + " entries per axis)");
      for (int kind = 0; kind < 2; ++kind) {
        const int t = (l * 3 + d) * 2 + kind;
        s.tab_off[t] = (int)s.tables.size();
        double acc = 0.0;
        for (int e = 0; e <= 2 * M; ++e) {
          const int m = e == 0 ? 0 : ((e & 1) ? (e + 1) / 2 : -(e / 2));
          const double k = kd * m;
          const double w = std::exp(-a * (double)m * (double)m) * (kind ? k * k : 1.0);
          acc += w;
          s.tables.push_back(acc);
        }
        s.tab_cnt[t] = 2 * M + 1;
        s.tab_tot[t] = acc;
      }
    }
  double acc = 0.0;
  for (int l = 0; l < s.mmax; ++l)
    for (int d = 0; d < 3; ++d) {
      double w = s.coef[l];
      for (int a = 0; a < 3; ++a) w *= s.tab_tot[(l * 3 + a) * 2 + (a == d ? 1 : 0)];
      acc += w;
      s.comp_cdf.push_back(acc);
    }
  // the mixture total is sum over all m of G^(m)|k|^2; less the |m| = 1 terms
  double unit = 0.0;
  for (size_t k = 0; k < s.direct_fb.size(); ++k) {
    double k2 = 0.0;
    for (int d = 0; d < 3; ++d) {
      const double kd = 2 * M_PI * s.direct_m[3 * k + d] / L[d];
      k2 += kd * kd;
    }
    unit += s.direct_fb[k] * k2;
  }
  s.S_full = acc - unit;
  return s;
}

}  // namespace rbx_host
