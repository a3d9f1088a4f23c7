/* Reference-kernel harness, k-space: RBMD's own op functors from
 * src/force/src/kspace_calculator_op/rocm/kspace_calculator_op.hip.cu, compiled
 * in place and exposed through extern "C" entry points taking device pointers
 * of rbmd::Real (float or double per build).  Test infrastructure only. */
#include "force/src/kspace_calculator_op/rocm/kspace_calculator_op.hip.cu"
#include "ref_common.h"

extern "C" {

int ref_real_size(void) { return (int)sizeof(rbmd::Real); }

int ref_rbe_rho(const double* lo, const double* hi, int n, int p, const rbmd::Real* q,
                const rbmd::Real* mx, const rbmd::Real* my, const rbmd::Real* mz,
                const rbmd::Real* x, const rbmd::Real* y, const rbmd::Real* z, rbmd::Real* re,
                rbmd::Real* im) {
  op::ComputePnumberChargeStructureFactorOp<device::DEVICE_GPU>()(ref_make_box(lo, hi), n, p, q,
                                                                  mx, my, mz, x, y, z, re, im);
  return ref_sync();
}

int ref_rbe_force(const double* lo, const double* hi, int n, int p, double alpha, double S,
                  double qqr2e, const rbmd::Real* re, const rbmd::Real* im, const rbmd::Real* q,
                  const rbmd::Real* mx, const rbmd::Real* my, const rbmd::Real* mz,
                  const rbmd::Real* x, const rbmd::Real* y, const rbmd::Real* z, rbmd::Real* fx,
                  rbmd::Real* fy, rbmd::Real* fz) {
  op::ComputeRBEForceOp<device::DEVICE_GPU>()(ref_make_box(lo, hi), n, p, (rbmd::Real)alpha,
                                              (rbmd::Real)S, (rbmd::Real)qqr2e, re, im, q, mx, my,
                                              mz, x, y, z, fx, fy, fz);
  return ref_sync();
}

int ref_rbe_virial(const double* lo, const double* hi, int p, double alpha, double S,
                   double qqr2e, double qsq, double qsum, const rbmd::Real* re,
                   const rbmd::Real* im, const rbmd::Real* mx, const rbmd::Real* my,
                   const rbmd::Real* mz, rbmd::Real* virial, rbmd::Real* energy) {
  op::ComputeRBEForceVirialOp<device::DEVICE_GPU>()(
      ref_make_box(lo, hi), p, (rbmd::Real)alpha, (rbmd::Real)S, (rbmd::Real)qqr2e,
      (rbmd::Real)qsq, (rbmd::Real)qsum, re, im, mx, my, mz, virial, energy);
  return ref_sync();
}

int ref_ewald_rho(int n, int nk, const rbmd::Real* q, const rbmd::Real* x, const rbmd::Real* y,
                  const rbmd::Real* z, const rbmd::Real* kx, const rbmd::Real* ky,
                  const rbmd::Real* kz, rbmd::Real* re, rbmd::Real* im) {
  op::ComputeKspaceChargeStructureFactorOp<device::DEVICE_GPU>()(n, nk, q, x, y, z, kx, ky, kz, re,
                                                                 im);
  return ref_sync();
}

int ref_ewald_force(const double* lo, const double* hi, int n, const int* kmax, double alpha,
                    double qqr2e, const rbmd::Real* re, const rbmd::Real* im, const rbmd::Real* q,
                    const rbmd::Real* x, const rbmd::Real* y, const rbmd::Real* z, rbmd::Real* fx,
                    rbmd::Real* fy, rbmd::Real* fz, rbmd::Real* flat_virial) {
  Int3 km;
  km.x = kmax[0];
  km.y = kmax[1];
  km.z = kmax[2];
  op::ComputeEwaldForceOp<device::DEVICE_GPU>()(ref_make_box(lo, hi), n, km, (rbmd::Real)alpha,
                                                (rbmd::Real)qqr2e, re, im, q, x, y, z, fx, fy, fz,
                                                flat_virial);
  return ref_sync();
}

/* RBSOG far field as ComputeRBSOG runs it (kspace_calculator.cpp:1331-1530):
 * ρ(k) of the P sampled vectors (ComputePnumberChargeStructureFactorSOGOp),
 * ComputeRBSOGSampleForceOp (force, energy_parts[0], virial with the NPT
 * terms over K_npt = K[idx_npt]), then ρ(k) of the direct vectors and
 * ComputeRBSOGDirectForceOp (force, energy, virial), both accumulating into the
 * same energy and virial buffers as the host code passes them.  K, K_npt and
 * the direct vectors are Cartesian (2π m / L); fac / fac_npt as
 * ComputeRBSOGFactorOp leaves them at a fixed box (all ones).  Outputs go to
 * separate force arrays per part. */
int ref_rbsog(const double* lo, const double* hi, int n, int p, double qqr2e, double S0,
              double S_npt, const rbmd::Real* kx, const rbmd::Real* ky, const rbmd::Real* kz,
              const rbmd::Real* knx, const rbmd::Real* kny, const rbmd::Real* knz,
              const int* idx_npt, const rbmd::Real* fac, const rbmd::Real* fac_npt, int nd,
              const rbmd::Real* dx, const rbmd::Real* dy, const rbmd::Real* dz,
              const rbmd::Real* fb, const rbmd::Real* fb_npt, const rbmd::Real* q,
              const rbmd::Real* x, const rbmd::Real* y, const rbmd::Real* z, rbmd::Real* rho_re,
              rbmd::Real* rho_im, rbmd::Real* drho_re, rbmd::Real* drho_im, rbmd::Real* fsx,
              rbmd::Real* fsy, rbmd::Real* fsz, rbmd::Real* fdx, rbmd::Real* fdy,
              rbmd::Real* fdz, rbmd::Real* virial_sample, rbmd::Real* virial_direct,
              rbmd::Real* energy_parts) {
  const Box box = ref_make_box(lo, hi);
  op::ComputePnumberChargeStructureFactorSOGOp<device::DEVICE_GPU>()(box, n, p, q, kx, ky, kz, x,
                                                                     y, z, rho_re, rho_im);
  op::ComputeRBSOGSampleForceOp<device::DEVICE_GPU>()(
      box, n, p, (rbmd::Real)qqr2e, (rbmd::Real)S0, (rbmd::Real)S_npt, kx, ky, kz, knx, kny, knz,
      idx_npt, fac, fac_npt, rho_re, rho_im, q, x, y, z, fsx, fsy, fsz, virial_sample,
      energy_parts);
  op::ComputeDirectChargeStructureFactorOp<device::DEVICE_GPU>()(n, nd, dx, dy, dz, q, x, y, z,
                                                                 drho_re, drho_im);
  op::ComputeRBSOGDirectForceOp<device::DEVICE_GPU>()(box, n, nd, (rbmd::Real)qqr2e, dx, dy, dz,
                                                      fb, fb_npt, drho_re, drho_im, q, x, y, z,
                                                      fdx, fdy, fdz, virial_direct,
                                                      energy_parts + 1);
  return ref_sync();
}

}  // extern "C"
