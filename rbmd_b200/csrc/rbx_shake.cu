// rbx_shake.cu -- SHAKE / RATTLE for rigid three-atom clusters (water).
//
// Follows the serial path of RBMD's ShakeController (shake_controller.cpp:
// 2130-2220) and its kernels ShakeA / ShakeB (shake_controller_op.hip.cu:
// 19-389, 391-660): every cluster (i0, i1, i2) with i1 the centre holds
// |r01| = |r12| = bond and |r02| = bond12 = sqrt(2 bond^2 (1 - cos angle)).
// ShakeA, after the drift, solves the three position multipliers by the
// fixed-point iteration of the quadratic constraint equations (tolerance
// 1e-5 on the multipliers, at most 5000 rounds) with the bond vectors of
// the step's start, moves the atoms and adds the same change / dt to their
// velocities; ShakeB, after the second half kick, removes the velocity
// components along the bonds of the new positions (a 3 x 3 linear solve).
// One thread per cluster; clusters are disjoint, so no atomics on atoms.
// ShakeA also refreshes the moved atoms' fixed-point records, which the list
// screens of both precision forms read, and their skin-check displacement.
// The reference recomputes the unconstrained update from copies of x and v
// taken before the drift and the kick and copies its result over every atom;
// here the unconstrained positions and half-step velocities are the ones the
// drift and kick kernels already wrote, and atoms outside clusters are left
// as they are.
#include <math.h>

#include "rbx_common.cuh"
#include "rbx_kernels.h"

namespace rbx {

namespace {
constexpr int SHAKE_BLOCK = 128;

// MinImageDistance_fix (box.h:99-112): d -= L rint(d / L).
__device__ __forceinline__ void min_image_rint(const DBox& b, double* d) {
#pragma unroll
  for (int k = 0; k < 3; ++k) d[k] -= b.len[k] * rint(d[k] * (1.0 / b.len[k]));
}

__device__ __forceinline__ double dot3(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// a - b, min image (MinImageDistanceVec, box.h:115-131)
__device__ __forceinline__ void sub_mi(const DBox& b, const double* a, const double* c,
                                       double* out) {
  out[0] = a[0] - c[0];
  out[1] = a[1] - c[1];
  out[2] = a[2] - c[2];
  min_image_rint(b, out);
}

// Cofactor inverse of a 3 x 3 matrix, the reference's order of terms.
__device__ __forceinline__ void inverse3(const double a[3][3], double ai[3][3], double* det) {
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
  *det = d;
}

__device__ __forceinline__ void load3(const double* x, const double* y, const double* z, int i,
                                      double* p) {
  p[0] = x[i];
  p[1] = y[i];
  p[2] = z[i];
}

__global__ void __launch_bounds__(SHAKE_BLOCK) k_shake_a(
    DBox b, ShakeParams sp, int nc, const int* __restrict__ cl, const int* __restrict__ where,
    const int* __restrict__ type, const double* __restrict__ mass, const double* __restrict__ xs,
    const double* __restrict__ ys, const double* __restrict__ zs, double* x, double* y, double* z,
    double* vx, double* vy, double* vz, ImageRefs img, const double* __restrict__ x0,
    const double* __restrict__ y0, const double* __restrict__ z0, unsigned long long* max_d2,
    uint4* atoms, const double* __restrict__ q, int* status) {
  const int c = blockIdx.x * SHAKE_BLOCK + threadIdx.x;
  double dmax = 0.0;
  if (c < nc) {
    int id[3];
    double po[3][3], pu[3][3], im[3];
    for (int k = 0; k < 3; ++k) {
      id[k] = where[cl[3 * c + k]];
      load3(xs, ys, zs, id[k], po[k]);
      load3(x, y, z, id[k], pu[k]);
      im[k] = 1 / mass[type[id[k]]];
    }
    // bond vectors at the step's start and after the unconstrained update
    double r01[3], r12[3], r20[3], s10[3], s21[3], s02[3];
    sub_mi(b, po[1], po[0], r01);
    sub_mi(b, po[2], po[1], r12);
    sub_mi(b, po[0], po[2], r20);
    sub_mi(b, pu[0], pu[1], s10);
    sub_mi(b, pu[1], pu[2], s21);
    sub_mi(b, pu[2], pu[0], s02);
    const double r01sq = dot3(r01, r01), r02sq = dot3(r20, r20), r12sq = dot3(r12, r12);
    const double s01sq = dot3(s10, s10), s02sq = dot3(s02, s02), s12sq = dot3(s21, s21);
    double a[3][3], ai[3][3], det;
    a[0][0] = 2 * (im[0] + im[1]) * dot3(s10, r01);
    a[0][1] = -2 * im[1] * dot3(s10, r12);
    a[0][2] = -2 * im[0] * dot3(s10, r20);
    a[1][0] = -2 * im[1] * dot3(s21, r01);
    a[1][1] = 2 * (im[1] + im[2]) * dot3(s21, r12);
    a[1][2] = -2 * im[2] * dot3(s21, r20);
    a[2][0] = -2 * im[0] * dot3(s02, r01);
    a[2][1] = -2 * im[2] * dot3(s02, r12);
    a[2][2] = 2 * (im[0] + im[2]) * dot3(s02, r20);
    inverse3(a, ai, &det);
    const double r0120 = dot3(r01, r20), r0112 = dot3(r01, r12), r2012 = dot3(r20, r12);
    // quadratic terms of each constraint in (l01, l20, l12):
    // [l01^2, l12^2, l20^2, l01 l20, l01 l12, l20 l12]
    const double q1[6] = {(im[0] + im[1]) * (im[0] + im[1]) * r01sq, im[1] * im[1] * r12sq,
                          im[0] * im[0] * r02sq, -2 * (im[0] + im[1]) * im[0] * r0120,
                          -2 * (im[0] + im[1]) * im[1] * r0112, 2 * im[0] * im[1] * r2012};
    const double q2[6] = {im[1] * im[1] * r01sq, (im[1] + im[2]) * (im[1] + im[2]) * r12sq,
                          im[2] * im[2] * r02sq, 2 * im[1] * im[2] * r0120,
                          -2 * (im[1] + im[2]) * im[1] * r0112,
                          -2 * (im[1] + im[2]) * im[2] * r2012};
    const double q3[6] = {im[0] * im[0] * r01sq, im[2] * im[2] * r12sq,
                          (im[0] + im[2]) * (im[0] + im[2]) * r02sq,
                          -2 * (im[0] + im[2]) * im[0] * r0120, 2 * im[0] * im[2] * r0112,
                          -2 * (im[0] + im[2]) * im[2] * r2012};
    double l01 = 0, l20 = 0, l12 = 0;
    bool done = false, overflow = false;
    int it = 0;
    while (!done && it < sp.max_iter) {
      const double t[6] = {l01 * l01, l12 * l12, l20 * l20, l01 * l20, l01 * l12, l20 * l12};
      const double quad1 = q1[0] * t[0] + q1[2] * t[2] + q1[1] * t[1] + q1[3] * t[3] +
                           q1[4] * t[4] + q1[5] * t[5];
      const double quad2 = q2[0] * t[0] + q2[2] * t[2] + q2[1] * t[1] + q2[3] * t[3] +
                           q2[4] * t[4] + q2[5] * t[5];
      const double quad3 = q3[0] * t[0] + q3[2] * t[2] + q3[1] * t[1] + q3[3] * t[3] +
                           q3[4] * t[4] + q3[5] * t[5];
      const double b1 = sp.b1sq - s01sq - quad1;
      const double b2 = sp.b2sq - s12sq - quad2;
      const double b3 = sp.b12sq - s02sq - quad3;
      const double n01 = ai[0][0] * b1 + ai[0][1] * b2 + ai[0][2] * b3;
      const double n12 = ai[1][0] * b1 + ai[1][1] * b2 + ai[1][2] * b3;
      const double n20 = ai[2][0] * b1 + ai[2][1] * b2 + ai[2][2] * b3;
      done = fabs(n01 - l01) <= sp.tol && fabs(n20 - l20) <= sp.tol && fabs(n12 - l12) <= sp.tol;
      l01 = n01;
      l20 = n20;
      l12 = n12;
      if (isnan(l01) || isnan(l20) || isnan(l12) || fabs(l01) > 1e20 || fabs(l20) > 1e20 ||
          fabs(l12) > 1e20) {
        done = true;
        overflow = true;
      }
      ++it;
    }
    if (!done || overflow || fabs(det) < 1e-4) atomicAdd(status, 1);
    double dp[3][3];
    for (int k = 0; k < 3; ++k) {
      dp[0][k] = l01 * r01[k] * im[0] - l20 * r20[k] * im[0];
      dp[1][k] = l12 * r12[k] * im[1] - l01 * r01[k] * im[1];
      dp[2][k] = l20 * r20[k] * im[2] - l12 * r12[k] * im[2];
    }
    double* vel[3] = {vx, vy, vz};
    double* pos[3] = {x, y, z};
    for (int a2 = 0; a2 < 3; ++a2) {
      const int i = id[a2];
      double p[3];
      for (int k = 0; k < 3; ++k) {
        vel[k][i] = vel[k][i] + dp[a2][k] / sp.dt;
        p[k] = pu[a2][k] + dp[a2][k];
        // ApplyPBC (box.h:133-169) with the image count
        int w = 0;
        if (p[k] >= b.lo[k] + b.len[k]) {
          p[k] -= b.len[k];
          w = 1;
        }
        if (p[k] < b.lo[k]) {
          p[k] += b.len[k];
          w = -1;
        }
        if (w && img.c[k]) img.c[k][i] += w;
        pos[k][i] = p[k];
      }
      if (max_d2) {
        const double ddx = min_image1(p[0] - x0[i], b.len[0], b.half[0]);
        const double ddy = min_image1(p[1] - y0[i], b.len[1], b.half[1]);
        const double ddz = min_image1(p[2] - z0[i], b.len[2], b.half[2]);
        dmax = fmax(dmax, ddx * ddx + ddy * ddy + ddz * ddz);
      }
      if (atoms) {
        uint4 r;
        r.x = to_fixed(p[0], b.lo[0], 4294967296.0 / b.len[0]);
        r.y = to_fixed(p[1], b.lo[1], 4294967296.0 / b.len[1]);
        r.z = to_fixed(p[2], b.lo[2], 4294967296.0 / b.len[2]);
        r.w = __float_as_uint((float)q[i]);
        atoms[i] = r;
      }
    }
  }
  if (max_d2) warp_max_atomic(dmax, max_d2);
}

__global__ void __launch_bounds__(SHAKE_BLOCK) k_shake_b(
    DBox b, int nc, const int* __restrict__ cl, const int* __restrict__ where,
    const int* __restrict__ type, const double* __restrict__ mass, const double* __restrict__ x,
    const double* __restrict__ y, const double* __restrict__ z, double* vx, double* vy, double* vz,
    int* status) {
  const int c = blockIdx.x * SHAKE_BLOCK + threadIdx.x;
  if (c >= nc) return;
  int id[3];
  double p[3][3], v[3][3], im[3];
  for (int k = 0; k < 3; ++k) {
    id[k] = where[cl[3 * c + k]];
    load3(x, y, z, id[k], p[k]);
    load3(vx, vy, vz, id[k], v[k]);
    im[k] = 1 / mass[type[id[k]]];
  }
  double r01[3], r12[3], r20[3], sv10[3], sv21[3], sv02[3];
  sub_mi(b, p[1], p[0], r01);
  sub_mi(b, p[2], p[1], r12);
  sub_mi(b, p[0], p[2], r20);
  for (int k = 0; k < 3; ++k) {
    sv10[k] = v[0][k] - v[1][k];
    sv21[k] = v[1][k] - v[2][k];
    sv02[k] = v[2][k] - v[0][k];
  }
  double a[3][3], ai[3][3], det;
  a[0][0] = (im[1] + im[0]) * dot3(r01, r01);
  a[0][1] = -im[1] * dot3(r01, r12);
  a[0][2] = (-im[0]) * dot3(r01, r20);
  a[1][0] = a[0][1];
  a[1][1] = (im[1] + im[2]) * dot3(r12, r12);
  a[1][2] = -(im[2]) * dot3(r20, r12);
  a[2][0] = a[0][2];
  a[2][1] = a[1][2];
  a[2][2] = (im[0] + im[2]) * dot3(r20, r20);
  const double cc[3] = {-dot3(sv10, r01), -dot3(sv21, r12), -dot3(sv02, r20)};
  inverse3(a, ai, &det);
  if (fabs(det) < 1e-4) atomicAdd(status, 1);
  double l[3];
  for (int r = 0; r < 3; ++r) {
    l[r] = 0;
    l[r] += ai[r][0] * cc[0];
    l[r] += ai[r][1] * cc[1];
    l[r] += ai[r][2] * cc[2];
  }
  double* vel[3] = {vx, vy, vz};
  for (int k = 0; k < 3; ++k) {
    vel[k][id[0]] = v[0][k] + (l[0] * r01[k] * im[0] - l[2] * r20[k] * im[0]);
    vel[k][id[1]] = v[1][k] + (l[1] * r12[k] * im[1] - l[0] * r01[k] * im[1]);
    vel[k][id[2]] = v[2][k] + (l[2] * r20[k] * im[2] - l[1] * r12[k] * im[2]);
  }
}

__global__ void k_inverse_perm(int n, const int* __restrict__ orig, int* __restrict__ where) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) where[orig[i]] = i;
}
}  // namespace

int launch_inverse_perm(int n, const int* orig, int* where, cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_inverse_perm<<<(n + 255) / 256, 256, 0, st>>>(n, orig, where);
  count_launch();
  return check_launch("inverse_perm");
}

int launch_shake_a(const DBox& b, const ShakeParams& sp, int nc, const int* cl, const int* where,
                   const int* type, const double* mass, Pos3 old, Pos3 pos, Pos3 vel,
                   ImageRefs img, const double* x0, const double* y0, const double* z0,
                   unsigned long long* max_d2, uint4* atoms, const double* q, int* status,
                   cudaStream_t st) {
  if (nc <= 0) return RBX_OK;
  k_shake_a<<<(nc + SHAKE_BLOCK - 1) / SHAKE_BLOCK, SHAKE_BLOCK, 0, st>>>(
      b, sp, nc, cl, where, type, mass, old.x, old.y, old.z, pos.x, pos.y, pos.z, vel.x, vel.y,
      vel.z, img, x0, y0, z0, max_d2, atoms, q, status);
  count_launch();
  return check_launch("shake_a");
}

int launch_shake_b(const DBox& b, int nc, const int* cl, const int* where, const int* type,
                   const double* mass, Pos3 pos, Pos3 vel, int* status, cudaStream_t st) {
  if (nc <= 0) return RBX_OK;
  k_shake_b<<<(nc + SHAKE_BLOCK - 1) / SHAKE_BLOCK, SHAKE_BLOCK, 0, st>>>(
      b, nc, cl, where, type, mass, pos.x, pos.y, pos.z, vel.x, vel.y, vel.z, status);
  count_launch();
  return check_launch("shake_b");
}

}  // namespace rbx
