// rbx_special.cu -- CVFF special-bond weights on the RBL pair force.
//
// RBMD's CVFF runs ComputeSpecialLJCutCoulRBLForce (src/force/src/cvff_op/
// rocm/cvff_op.hip.cu:401-533): the LJCutCoulKspace RBL pair force with, for
// a pair listed in atom i's special row at position k (1-2 / 1-3 / 1-4 by the
// cumulative counts, weight w), the LJ term times w and the erfc Coulomb
// minus (1 - w) times the bare Coulomb -qqr2e qi qj / r^3 -- so a pair
// excluded from real space (w = 0) also cancels its k-space interaction.
// Special pairs are a handful per atom (bonded neighbours), so instead of a
// weight lookup for each of the ~500 candidates per atom inside the fused
// pair kernel, this kernel adds, after it, the difference for each special
// pair the RBL lists hold this step:
//     F_i += (w - 1) (m * f_lj + f_bare) (r_j - r_i),
// m = 1 in the core, pice_num in a selected shell pair (f_bare is not
// multiplied by pice_num, as in the reference).  List membership uses the
// same exact FP64 predicates and batch hash as the fused kernel, and the
// per-block sums of the added forces join the fused kernel's partial sums,
// so the mean-force removal covers them.  One thread per atom with specials
// (each updates only its own atom: the rows are symmetric).
#include <math.h>

#include "rbx_common.cuh"
#include "rbx_kernels.h"
#include "rbx_pair_device.cuh"

namespace rbx {

namespace {
constexpr int SPEC_BLOCK = 128;

__global__ void __launch_bounds__(SPEC_BLOCK) k_special_rbl(
    PairParams pp, int natoms, const int* __restrict__ atoms_h, const int* __restrict__ cnt,
    const int* __restrict__ part, int maxs, double w12, double w13, double w14,
    const int* __restrict__ where, const double* __restrict__ x, const double* __restrict__ y,
    const double* __restrict__ z, const double* __restrict__ q, const int* __restrict__ type,
    const unsigned long long* __restrict__ key_a, const unsigned long long* __restrict__ key_b,
    int epoch_arg, const int* epoch_dev, double* fx, double* fy, double* fz, double* fpart) {
  __shared__ double sh[3][SPEC_BLOCK / 32];
  const int epoch = epoch_dev ? *epoch_dev : epoch_arg;
  double s[3] = {0, 0, 0};
  for (int a = blockIdx.x * SPEC_BLOCK + threadIdx.x; a < natoms; a += gridDim.x * SPEC_BLOCK) {
    const int h = atoms_h[a];
    const int i = where[h];
    // LoadSpecialCounts (cvff_op.hip.cu:51-77)
    int n12 = max(cnt[3 * h], 0), n13 = max(cnt[3 * h + 1], 0), n14 = max(cnt[3 * h + 2], 0);
    if (n12 > n13) n13 = n12;
    if (n13 > n14) n14 = n13;
    if (n14 > maxs) n14 = maxs;
    if (n13 > n14) n13 = n14;
    if (n12 > n13) n12 = n13;
    const unsigned long long ea = key_a[i] ^ (unsigned long long)(long long)epoch;
    const double xi = x[i], yi = y[i], zi = z[i], qi = q[i];
    const int ti = type[i];
    double f3[3] = {0, 0, 0};
    for (int k = 0; k < n14; ++k) {
      const int j = where[part[(size_t)h * maxs + k]];
      if (j == i) continue;
      const double w = k < n12 ? w12 : (k < n13 ? w13 : w14);
      if (w == 1.0) continue;
      const double d2 = exact_d2(pp, x, y, z, i, j);
      const Classified c = classify_exact(d2, pp);
      double m;
      if (c.core_active)
        m = 1.0;
      else if (c.shell_window && rbl_selected(ea, key_b[j], pp.div))
        m = (double)pp.freq;
      else
        continue;
      const double dx = min_image1(x[j] - xi, pp.box.len[0], pp.box.half[0]);
      const double dy = min_image1(y[j] - yi, pp.box.len[1], pp.box.half[1]);
      const double dz = min_image1(z[j] - zi, pp.box.len[2], pp.box.half[2]);
      const double r2 = dx * dx + dy * dy + dz * dz;
      const int pt = ti * pp.ntypes + type[j];
      const double eps = pp.lj_eps[pt], s6 = pp.lj_s6[pt];
      const double r2inv = 1.0 / r2, r6inv = r2inv * r2inv * r2inv;
      const double flj = -m * r2inv * r6inv * (48.0 * eps * s6 * s6 * r6inv - 24.0 * eps * s6);
      const double dis = sqrt(r2);
      const double bare = -pp.qqr2e * qi * q[j] / (r2 * dis);
      const double f = (w - 1.0) * (flj + bare);
      f3[0] += f * dx;
      f3[1] += f * dy;
      f3[2] += f * dz;
    }
    fx[i] += f3[0];
    fy[i] += f3[1];
    fz[i] += f3[2];
    s[0] += f3[0];
    s[1] += f3[1];
    s[2] += f3[2];
  }
  // fixed-order block sums for the mean removal
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  for (int d = 0; d < 3; ++d) {
    const double v = warp_sum(s[d]);
    if (l == 0) sh[d][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0;
    for (int k = 0; k < SPEC_BLOCK / 32; ++k) t += sh[threadIdx.x][k];
    fpart[(size_t)blockIdx.x * 3 + threadIdx.x] = t;
  }
}
}  // namespace

int launch_special_rbl(const PairParams& pp, int natoms, const int* atoms_h, const int* cnt,
                       const int* part, int maxs, double w12, double w13, double w14,
                       const int* where, const double* x, const double* y, const double* z,
                       const double* q, const int* type, const unsigned long long* key_a,
                       const unsigned long long* key_b, int epoch, const int* epoch_dev,
                       double* fx, double* fy, double* fz, double* fpart, cudaStream_t st) {
  k_special_rbl<<<SPEC_PARTS, SPEC_BLOCK, 0, st>>>(pp, natoms, atoms_h, cnt, part, maxs, w12, w13,
                                                   w14, where, x, y, z, q, type, key_a, key_b,
                                                   epoch, epoch_dev, fx, fy, fz, fpart);
  count_launch();
  return check_launch("special_rbl");
}

}  // namespace rbx
