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

}  // extern "C"
