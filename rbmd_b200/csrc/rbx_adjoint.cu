// rbx_adjoint.cu -- adjoint (vector-Jacobian product) of the RBL + RBE force
// for force-field fitting: plain FP64 for FP64 engines; FP32 pair terms and
// FP32 k-space terms on exact fixed-point phases with FP64 sums for engines
// in the mixed form.
//
// For an upstream g = dL/dF it gives dL/d(eps_t, sigma_t) per type, dL/dq_i,
// dL/dalpha and dL/dr_i (the Hessian-vector product), for the lists, batch
// selection and k-samples of the engine's last force evaluation.  Nothing is
// stored per pair: the pair terms and the k-space phases are recomputed.
//
// Force (ComputeLJCutCoulRBLForce, lj_cut_coul_kspace_op.hip.cu:569-683; mean
// removal lj_cut_coul_kspace.cpp:537-563; ComputeRBEForce,
// kspace_calculator_op.hip.cu:98-125, 678-738):
//   F_i = P_i - mean(P) + K_i,  P_i = sum_{j in L(i)} s_ij f(r^2) (r_j - r_i)
// With g' = g - mean(g), pair (i, j) adds s (df/dtheta)(g'_i . d) to the
// parameter gradient and c = s (f g'_i + 2 f'(g'_i . d) d) to dL/dr_j, -c to
// dL/dr_i.  The pair kernel runs a warp per atom m over its candidate row,
// which is symmetric, and tests both m in L(j) and j in L(m) (the same
// distance windows; the shell batch hash evaluated from either side), so each
// atom gathers its own gradient without atomics.  The k-space part uses
// a_k = sum_i q_i (g_i.k) cos(k.r_i), b_k = sum_i q_i (g_i.k) sin(k.r_i).
#include <math.h>

#include "rbx_common.cuh"
#include "rbx_kernels.h"
#include "rbx_pair_device.cuh"

namespace rbx {

constexpr int ADJ_WARPS = 8;
constexpr int ADJ_BLOCK = 32 * ADJ_WARPS;
constexpr int ADJ_MAX_TYPES = 16;

// Pair terms of one (i, j) at squared distance r2 (windows already applied):
// f, f' = df/d(r^2), df/deps_ij, df/dsigma_ij, the Coulomb shape h (f_C = q q h)
// and dh/dalpha.
struct PairTerms {
  double f, fp, df_de, df_ds, h, dh_da;
};

__device__ __forceinline__ PairTerms pair_terms(double e, double sg, double qq, double r2,
                                                double alpha, double qqr2e) {
  PairTerms t;
  const double ui = 1.0 / r2;
  const double s6 = sg * sg * sg * sg * sg * sg;
  const double u = s6 * ui * ui * ui;  // sigma^6 / r^6
  const double f_lj = -24.0 * e * (2.0 * u * u - u) * ui;
  const double ui2 = ui * ui, ui4 = ui2 * ui2;
  const double fp_lj = 24.0 * e * (14.0 * s6 * s6 * ui4 * ui4 - 4.0 * s6 * ui4 * ui);
  const double r = sqrt(r2);
  const double b = sqrt(alpha);
  const double ex = exp(-alpha * r2);
  const double ec = erfc(b * r);
  const double two_b_pi = 2.0 * b / 1.77245385090551602729;  // 2 b / sqrt(pi)
  t.h = -qqr2e * (ec * ui + two_b_pi * ex / r) / r;
  const double dh_dr = qqr2e * (3.0 * ec * ui2 + two_b_pi * ex * (3.0 * ui + 2.0 * alpha) / r);
  t.dh_da = qqr2e * two_b_pi * ex;
  t.f = f_lj + qq * t.h;
  t.fp = fp_lj + qq * dh_dr / (2.0 * r);
  t.df_de = f_lj / e;
  t.df_ds = -144.0 * e * (4.0 * u * u - u) * ui / sg;
  return t;
}

// The same pair terms in FP32 (mixed form), returned widened to FP64 for the
// FP64 sums of the adjoint.
__device__ __forceinline__ PairTerms pair_terms_f32(float e, float sg, float qq, float r2,
                                                    float alpha, float qqr2e) {
  const float ui = 1.0f / r2;
  const float s2 = sg * sg, s6 = s2 * s2 * s2;
  const float u = s6 * ui * ui * ui;
  const float f_lj = -24.0f * e * (2.0f * u * u - u) * ui;
  const float ui2 = ui * ui, ui4 = ui2 * ui2;
  const float fp_lj = 24.0f * e * (14.0f * s6 * s6 * ui4 * ui4 - 4.0f * s6 * ui4 * ui);
  const float r = sqrtf(r2);
  const float b = sqrtf(alpha);
  const float ex = expf(-alpha * r2);
  const float ec = erfcf(b * r);
  const float two_b_pi = 2.0f * b / 1.77245385090551602729f;
  const float h = -qqr2e * (ec * ui + two_b_pi * ex / r) / r;
  const float dh_dr = qqr2e * (3.0f * ec * ui2 + two_b_pi * ex * (3.0f * ui + 2.0f * alpha) / r);
  PairTerms t;
  t.h = h;
  t.dh_da = qqr2e * two_b_pi * ex;
  t.f = f_lj + qq * h;
  t.fp = fp_lj + qq * dh_dr / (2.0f * r);
  t.df_de = f_lj / e;
  t.df_ds = -144.0f * e * (4.0f * u * u - u) * ui / sg;
  return t;
}

// Block partials: [block][2 * ntypes + 1] = d_eps[0..nt), d_sigma[0..nt), d_alpha.
// F32: pair terms in FP32 (mixed form), sums in FP64 either way.
template <bool F32>
__global__ void __launch_bounds__(ADJ_BLOCK)
k_adj_pair(PairParams pp, int n, const double* __restrict__ x, const double* __restrict__ y,
           const double* __restrict__ z, const double* __restrict__ q,
           const int* __restrict__ type, const double* __restrict__ sigma_t,
           const double* __restrict__ eps_t, const unsigned long long* __restrict__ key_a,
           const unsigned long long* __restrict__ key_b, int epoch, Rows rows,
           const double* __restrict__ gx, const double* __restrict__ gy,
           const double* __restrict__ gz, double mgx, double mgy, double mgz,
           double* __restrict__ d_rx, double* __restrict__ d_ry, double* __restrict__ d_rz,
           double* __restrict__ d_q, double* __restrict__ part) {
  __shared__ double s_part[ADJ_WARPS][2 * ADJ_MAX_TYPES + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nt = pp.ntypes, npar = 2 * nt + 1;
  for (int t = threadIdx.x; t < ADJ_WARPS * (2 * ADJ_MAX_TYPES + 1); t += ADJ_BLOCK)
    (&s_part[0][0])[t] = 0.0;
  __syncthreads();
  double acc[2 * ADJ_MAX_TYPES + 1];
  for (int t = 0; t < npar; ++t) acc[t] = 0.0;
  const double freq = (double)pp.freq;
  for (int m = blockIdx.x * ADJ_WARPS + warp; m < n; m += gridDim.x * ADJ_WARPS) {
    const double xm = x[m], ym = y[m], zm = z[m], qm = q[m];
    const int tm = type[m];
    const double gpx = gx[m] - mgx, gpy = gy[m] - mgy, gpz = gz[m] - mgz;
    const unsigned long long ea_m = key_a[m] ^ (unsigned long long)(long long)epoch;
    const unsigned long long kb_m = key_b[m];
    double rx = 0.0, ry = 0.0, rz = 0.0, dq = 0.0;
    int nf, nb;
    row_extent(rows, m, nf, nb);
    const int* row = rows.idx + (size_t)m * rows.cap;
    for (int k = lane; k < nf + nb; k += 32) {
      const int j = row_at(row, rows.cap, nf, nb, k);
      if (j == m) continue;
      const Classified c = classify_exact(exact_d2(pp, x, y, z, m, j), pp);
      if (!c.core_active && !c.shell_window) continue;
      const bool in_m = c.core_active || rbl_selected(ea_m, key_b[j], pp.div);
      const unsigned long long ea_j = key_a[j] ^ (unsigned long long)(long long)epoch;
      const bool in_j = c.core_active || rbl_selected(ea_j, kb_m, pp.div);
      if (!in_m && !in_j) continue;
      const double s = c.core_active ? 1.0 : freq;
      // r_j - r_m, MinImageDistance (box.h:51-73), as in the force kernel
      const double dx = min_image1(x[j] - xm, pp.box.len[0], pp.box.half[0]);
      const double dy = min_image1(y[j] - ym, pp.box.len[1], pp.box.half[1]);
      const double dz = min_image1(z[j] - zm, pp.box.len[2], pp.box.half[2]);
      const double r2 = dx * dx + dy * dy + dz * dz;
      const int tj = type[j];
      const double e = sqrt(eps_t[tm] * eps_t[tj]);
      const double sg = 0.5 * (sigma_t[tm] + sigma_t[tj]);
      const double qj = q[j];
      const PairTerms pt =
          F32 ? pair_terms_f32((float)e, (float)sg, (float)(qm * qj), (float)r2, (float)pp.alpha,
                               (float)pp.qqr2e)
              : pair_terms(e, sg, qm * qj, r2, pp.alpha, pp.qqr2e);
      if (in_m) {  // pair (m, j) of m's force: parameters and -c on r_m
        const double gd = gpx * dx + gpy * dy + gpz * dz;
        const double w = s * gd;
        const double cf = s * pt.f, cd = 2.0 * s * pt.fp * gd;
        rx -= cf * gpx + cd * dx;
        ry -= cf * gpy + cd * dy;
        rz -= cf * gpz + cd * dz;
        dq += w * pt.h * qj;
        acc[tm] += w * pt.df_de * e / (2.0 * eps_t[tm]);
        acc[tj] += w * pt.df_de * e / (2.0 * eps_t[tj]);
        acc[nt + tm] += 0.5 * w * pt.df_ds;
        acc[nt + tj] += 0.5 * w * pt.df_ds;
        acc[2 * nt] += w * qm * qj * pt.dh_da;
      }
      if (in_j) {  // pair (j, m) of j's force: +c on r_m, and its q_m factor
        const double gjx = gx[j] - mgx, gjy = gy[j] - mgy, gjz = gz[j] - mgz;
        const double gd = gjx * dx + gjy * dy + gjz * dz;  // d = r_j - r_m: g'_j . (-(r_m - r_j))
        const double cf = s * pt.f, cd = 2.0 * s * pt.fp * gd;
        rx += cf * gjx + cd * dx;
        ry += cf * gjy + cd * dy;
        rz += cf * gjz + cd * dz;
        dq -= s * gd * pt.h * qj;  // w_j = s g'_j . (r_m - r_j) = -s gd
      }
    }
    rx = warp_sum(rx);
    ry = warp_sum(ry);
    rz = warp_sum(rz);
    dq = warp_sum(dq);
    if (lane == 0) {
      d_rx[m] = rx;
      d_ry[m] = ry;
      d_rz[m] = rz;
      d_q[m] = dq;
    }
  }
  for (int t = 0; t < npar; ++t) {
    const double v = warp_sum(acc[t]);
    if (lane == 0) s_part[warp][t] = v;
  }
  __syncthreads();
  if (threadIdx.x < npar) {
    double v = 0.0;
    for (int w = 0; w < ADJ_WARPS; ++w) v += s_part[w][threadIdx.x];
    part[(size_t)blockIdx.x * npar + threadIdx.x] = v;
  }
}

// k-space, pass 1: per-block partial sums of a_k and b_k, part[k][block].
constexpr int ADJK_BLOCK = 128;
__global__ void __launch_bounds__(ADJK_BLOCK)
k_adj_k_ab(int n, int p, int chunk, const KTab* __restrict__ tab, const double* __restrict__ q,
           const double* __restrict__ x, const double* __restrict__ y,
           const double* __restrict__ z, const double* __restrict__ gx,
           const double* __restrict__ gy, const double* __restrict__ gz,
           double* __restrict__ part_a, double* __restrict__ part_b) {
  const int k = blockIdx.y * ADJK_BLOCK + threadIdx.x;
  if (k >= p) return;
  const double kx = tab[k].kx, ky = tab[k].ky, kz = tab[k].kz;
  const int a0 = blockIdx.x * chunk, a1 = min(n, a0 + chunk);
  double sa = 0.0, sb = 0.0;
  for (int i = a0; i < a1; ++i) {
    double s, c;
    sincos(kx * x[i] + ky * y[i] + kz * z[i], &s, &c);
    const double w = q[i] * (gx[i] * kx + gy[i] * ky + gz[i] * kz);
    sa += w * c;
    sb += w * s;
  }
  part_a[(size_t)k * gridDim.x + blockIdx.x] = sa;
  part_b[(size_t)k * gridDim.x + blockIdx.x] = sb;
}

// k-space, pass 2: per-atom dL/dq and dL/dr, and per-block sums of g . K
// (for dL/dalpha).  ab[k] = {a_k, b_k} reduced in fixed order beforehand.
__global__ void __launch_bounds__(ADJK_BLOCK)
k_adj_k_scatter(int n, int p, double cscale, const KTab* __restrict__ tab,
                const double* __restrict__ ab, const double* __restrict__ q,
                const double* __restrict__ x, const double* __restrict__ y,
                const double* __restrict__ z, const double* __restrict__ gx,
                const double* __restrict__ gy, const double* __restrict__ gz,
                double* __restrict__ d_rx, double* __restrict__ d_ry, double* __restrict__ d_rz,
                double* __restrict__ d_q, double* __restrict__ part_gk) {
  __shared__ double s_sum[ADJK_BLOCK / 32];
  const int i = blockIdx.x * ADJK_BLOCK + threadIdx.x;
  double gk_sum = 0.0;
  if (i < n) {
    const double xi = x[i], yi = y[i], zi = z[i], qi = q[i];
    const double gix = gx[i], giy = gy[i], giz = gz[i];
    double rx = 0.0, ry = 0.0, rz = 0.0, dq = 0.0;
    for (int k = 0; k < p; ++k) {
      const KTab t = tab[k];
      const double k2 = t.kx * t.kx + t.ky * t.ky + t.kz * t.kz;
      const double ck = cscale / k2;  // -4 pi qqr2e S / (P V k^2)
      double s, c;
      sincos(t.kx * xi + t.ky * yi + t.kz * zi, &s, &c);
      const double gk = gix * t.kx + giy * t.ky + giz * t.kz;
      // t.a = c_k Re rho_k, t.b = c_k Im rho_k
      const double ak = ab[2 * k], bk = ab[2 * k + 1];
      dq += gk * (c * t.b - s * t.a) + ck * (ak * s - bk * c);
      const double coef = -gk * (s * t.b + c * t.a) + ck * (ak * c + bk * s);
      rx += coef * t.kx;
      ry += coef * t.ky;
      rz += coef * t.kz;
      gk_sum += gk * (c * t.b - s * t.a);
    }
    d_rx[i] += qi * rx;
    d_ry[i] += qi * ry;
    d_rz[i] += qi * rz;
    d_q[i] += dq;
    gk_sum *= qi;
  }
  gk_sum = block_sum_det<ADJK_BLOCK>(gk_sum, s_sum);
  if (threadIdx.x == 0) part_gk[blockIdx.x] = gk_sum;
}

// Mixed form of the k-space passes: the phase k.r_i = 2 pi (m . u_i) / 2^32 from
// the 32-bit fixed-point record u_i exactly in integer arithmetic, sin and
// cos on the SFU, every term in FP32 and every sum in FP64.
__global__ void __launch_bounds__(ADJK_BLOCK)
k_adj_k_ab_mixed(int n, int p, int chunk, const KTab* __restrict__ tab,
                 const uint4* __restrict__ atoms, const double* __restrict__ gx,
                 const double* __restrict__ gy, const double* __restrict__ gz,
                 double* __restrict__ part_a, double* __restrict__ part_b) {
  const int k = blockIdx.y * ADJK_BLOCK + threadIdx.x;
  if (k >= p) return;
  const KTab t = tab[k];
  const unsigned m0 = (unsigned)t.m[0], m1 = (unsigned)t.m[1], m2 = (unsigned)t.m[2];
  const float kx = (float)t.kx, ky = (float)t.ky, kz = (float)t.kz;
  const float ang = (float)(2.0 * RBX_PI / 4294967296.0);
  const int a0 = blockIdx.x * chunk, a1 = min(n, a0 + chunk);
  double sa = 0.0, sb = 0.0;
  for (int i = a0; i < a1; ++i) {
    const uint4 a = atoms[i];
    const unsigned ph = m0 * a.x + m1 * a.y + m2 * a.z;
    float sn, cs;
    __sincosf((float)(int)ph * ang, &sn, &cs);
    const float w = __uint_as_float(a.w) *
                    ((float)gx[i] * kx + (float)gy[i] * ky + (float)gz[i] * kz);
    sa += (double)(w * cs);
    sb += (double)(w * sn);
  }
  part_a[(size_t)k * gridDim.x + blockIdx.x] = sa;
  part_b[(size_t)k * gridDim.x + blockIdx.x] = sb;
}

__global__ void __launch_bounds__(ADJK_BLOCK)
k_adj_k_scatter_mixed(int n, int p, double cscale, const KTab* __restrict__ tab,
                      const double* __restrict__ ab, const uint4* __restrict__ atoms,
                      const double* __restrict__ gx, const double* __restrict__ gy,
                      const double* __restrict__ gz, double* __restrict__ d_rx,
                      double* __restrict__ d_ry, double* __restrict__ d_rz,
                      double* __restrict__ d_q, double* __restrict__ part_gk) {
  __shared__ double s_sum[ADJK_BLOCK / 32];
  const int i = blockIdx.x * ADJK_BLOCK + threadIdx.x;
  double gk_sum = 0.0;
  if (i < n) {
    const uint4 a = atoms[i];
    const float qi = __uint_as_float(a.w);
    const float gix = (float)gx[i], giy = (float)gy[i], giz = (float)gz[i];
    const float ang = (float)(2.0 * RBX_PI / 4294967296.0);
    double rx = 0.0, ry = 0.0, rz = 0.0, dq = 0.0;
    for (int k = 0; k < p; ++k) {
      const KTab t = tab[k];
      const float kx = (float)t.kx, ky = (float)t.ky, kz = (float)t.kz;
      const float ck = (float)(cscale / (t.kx * t.kx + t.ky * t.ky + t.kz * t.kz));
      const unsigned ph =
          (unsigned)t.m[0] * a.x + (unsigned)t.m[1] * a.y + (unsigned)t.m[2] * a.z;
      float sn, cs;
      __sincosf((float)(int)ph * ang, &sn, &cs);
      const float gk = gix * kx + giy * ky + giz * kz;
      const float ta = (float)t.a, tb = (float)t.b;
      const float ak = (float)ab[2 * k], bk = (float)ab[2 * k + 1];
      const float g1 = gk * (cs * tb - sn * ta);
      dq += (double)(g1 + ck * (ak * sn - bk * cs));
      const float coef = -gk * (sn * tb + cs * ta) + ck * (ak * cs + bk * sn);
      rx += (double)(coef * kx);
      ry += (double)(coef * ky);
      rz += (double)(coef * kz);
      gk_sum += (double)g1;
    }
    d_rx[i] += (double)qi * rx;
    d_ry[i] += (double)qi * ry;
    d_rz[i] += (double)qi * rz;
    d_q[i] += dq;
    gk_sum *= (double)qi;
  }
  gk_sum = block_sum_det<ADJK_BLOCK>(gk_sum, s_sum);
  if (threadIdx.x == 0) part_gk[blockIdx.x] = gk_sum;
}

// Fixed-order reduction of part[k][nb] into out[2 * k + which].
__global__ void k_adj_reduce_k(int p, int nb, const double* __restrict__ part_a,
                               const double* __restrict__ part_b, double* __restrict__ ab) {
  __shared__ double sh[32];
  const int k = blockIdx.x;
  double a = 0.0, b = 0.0;
  for (int t = threadIdx.x; t < nb; t += blockDim.x) {
    a += part_a[(size_t)k * nb + t];
    b += part_b[(size_t)k * nb + t];
  }
  a = block_sum_det<128>(a, sh);
  b = block_sum_det<128>(b, sh);
  if (threadIdx.x == 0) {
    ab[2 * k] = a;
    ab[2 * k + 1] = b;
  }
}

__global__ void k_gather_vec3(int n, const int* __restrict__ orig, const double* __restrict__ src,
                              double* __restrict__ x, double* __restrict__ y,
                              double* __restrict__ z) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t o = (size_t)orig[i] * 3;
  x[i] = src[o];
  y[i] = src[o + 1];
  z[i] = src[o + 2];
}

int launch_gather_vec3(int n, const int* orig, const double* src, double* x, double* y, double* z,
                       cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_gather_vec3<<<(n + 255) / 256, 256, 0, st>>>(n, orig, src, x, y, z);
  count_launch();
  return check_launch("gather_vec3");
}

int adj_pair_blocks(int n) {
  const int b = (n + ADJ_WARPS - 1) / ADJ_WARPS;
  return b < 4 * sm_count() ? (b < 1 ? 1 : b) : 4 * sm_count();
}

int launch_adj_pair(const PairParams& pp, int n, const double* x, const double* y,
                    const double* z, const double* q, const int* type, const double* sigma_t,
                    const double* eps_t, const unsigned long long* key_a,
                    const unsigned long long* key_b, int epoch, const Rows& rows,
                    const double* gx, const double* gy,
                    const double* gz, const double mean_g[3], double* d_rx, double* d_ry,
                    double* d_rz, double* d_q, double* part, int nblocks, cudaStream_t st,
                    bool f32) {
  if (pp.ntypes > ADJ_MAX_TYPES) {
    set_error("adjoint: at most %d atom types", ADJ_MAX_TYPES);
    return RBX_ERR_INVALID;
  }
  auto kern = f32 ? k_adj_pair<true> : k_adj_pair<false>;
  kern<<<nblocks, ADJ_BLOCK, 0, st>>>(pp, n, x, y, z, q, type, sigma_t, eps_t, key_a, key_b,
                                            epoch, rows, gx, gy, gz, mean_g[0],
                                            mean_g[1], mean_g[2], d_rx, d_ry, d_rz, d_q, part);
  count_launch();
  return check_launch("adj_pair");
}

int adj_k_blocks(int n) { return (n + ADJK_BLOCK - 1) / ADJK_BLOCK; }

int launch_adj_kspace(int n, int p, double cscale, const KTab* tab, const double* q,
                      const double* x, const double* y, const double* z, const double* gx,
                      const double* gy, const double* gz, double* part_a, double* part_b,
                      int nparts, double* ab, double* d_rx, double* d_ry, double* d_rz,
                      double* d_q, double* part_gk, cudaStream_t st) {
  if (p <= 0 || n <= 0) return RBX_OK;
  const int chunk = (n + nparts - 1) / nparts;
  const int nb = (n + chunk - 1) / chunk;
  k_adj_k_ab<<<dim3(nb, (p + ADJK_BLOCK - 1) / ADJK_BLOCK), ADJK_BLOCK, 0, st>>>(
      n, p, chunk, tab, q, x, y, z, gx, gy, gz, part_a, part_b);
  count_launch();
  int rc = check_launch("adj_k_ab");
  if (rc) return rc;
  k_adj_reduce_k<<<p, 128, 0, st>>>(p, nb, part_a, part_b, ab);
  count_launch();
  rc = check_launch("adj_reduce_k");
  if (rc) return rc;
  k_adj_k_scatter<<<adj_k_blocks(n), ADJK_BLOCK, 0, st>>>(n, p, cscale, tab, ab, q, x, y, z, gx,
                                                          gy, gz, d_rx, d_ry, d_rz, d_q, part_gk);
  count_launch();
  return check_launch("adj_k_scatter");
}

int launch_adj_kspace_mixed(int n, int p, double cscale, const KTab* tab, const uint4* atoms,
                            const double* gx, const double* gy, const double* gz, double* part_a,
                            double* part_b, int nparts, double* ab, double* d_rx, double* d_ry,
                            double* d_rz, double* d_q, double* part_gk, cudaStream_t st) {
  if (p <= 0 || n <= 0) return RBX_OK;
  const int chunk = (n + nparts - 1) / nparts;
  const int nb = (n + chunk - 1) / chunk;
  k_adj_k_ab_mixed<<<dim3(nb, (p + ADJK_BLOCK - 1) / ADJK_BLOCK), ADJK_BLOCK, 0, st>>>(
      n, p, chunk, tab, atoms, gx, gy, gz, part_a, part_b);
  count_launch();
  int rc = check_launch("adj_k_ab_mixed");
  if (rc) return rc;
  k_adj_reduce_k<<<p, 128, 0, st>>>(p, nb, part_a, part_b, ab);
  count_launch();
  rc = check_launch("adj_reduce_k");
  if (rc) return rc;
  k_adj_k_scatter_mixed<<<adj_k_blocks(n), ADJK_BLOCK, 0, st>>>(
      n, p, cscale, tab, ab, atoms, gx, gy, gz, d_rx, d_ry, d_rz, d_q, part_gk);
  count_launch();
  return check_launch("adj_k_scatter_mixed");
}

}  // namespace rbx
