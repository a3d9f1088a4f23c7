// rbsog.h -- parameters of RBMD's RBSOG k-space and VERLET-SOG real space
// (random-batch sum-of-Gaussians), computed on the host once per box.
#pragma once
#include <vector>

#include "rbx.h"

namespace rbx_host {

struct RbsogSetup {
  int level = 0, mmax = 0;
  double b = 0, sigma = 0, w0 = 0;
  std::vector<double> coef, coef_npt;  // Fourier weights of the Gaussians, [mmax]
  double S = 0, S_npt = 0;             // sampling normalisations (RBSOGSetup)
  double S_full = 0;                   // sum of G^(m)|k|^2 over |m|^2 > 1 (exact)
  double taylor[6] = {0, 0, 0, 0, 0, 0};
  double self_coeff = 0;               // E_self = -self_coeff * sum q^2 * qqr2e
  // the |m|^2 <= Kcut = 1 vectors summed directly, and their weights G^(k)
  std::vector<int> direct_m;           // [6][3]
  std::vector<double> direct_fb;       // [6]
  std::vector<double> direct_fb_npt;   // [6], with coef_npt (virial)
  // exact sampler of p(m) ~ G^(m) |k|^2: a mixture over (Gaussian l, axis d)
  // of separable densities; per (l, axis, kind) a cumulative table over the
  // order m = 0, +1, -1, +2, -2, ... (kind 0: g_l(m), kind 1: k^2 g_l(m))
  std::vector<double> comp_cdf;        // [3 mmax] cumulative component weights
  std::vector<double> tables;          // concatenated cumulative tables
  std::vector<int> tab_off, tab_cnt;   // [mmax][3][2]
  std::vector<double> tab_tot;         // [mmax][3][2]
};

// Throws std::runtime_error on a level outside [0, 4] or a bad box.
RbsogSetup rbsog_setup(int level, double cut_off, const rbx_box& box);

}  // namespace rbx_host
