/* Reference-kernel harness, real space: RBMD's own op functors from
 * src/force/src/cvff_op/rocm/cvff_op.hip.cu (which includes
 * lj_cut_coul_kspace_op.hip.cu and, through it, lj_op.hip.cu) and
 * force_op.hip.cu, compiled in place.  Test infrastructure only. */
#include "force/src/cvff_op/rocm/cvff_op.hip.cu"
#include "force/src/force_op/rocm/force_op.hip.cu"
#include "ref_common.h"

extern "C" {

int ref_pair_rbl(const double* lo, const double* hi, double rs, double rc, int n, int sample_num,
                 int pice, double alpha, double qqr2e, const int* type, const rbmd::Real* sigma,
                 const rbmd::Real* eps, const int* start, const int* end, const int* core,
                 const int* shell, const int* shell_num, const rbmd::Real* q, const rbmd::Real* x,
                 const rbmd::Real* y, const rbmd::Real* z, rbmd::Real* fx, rbmd::Real* fy,
                 rbmd::Real* fz) {
  op::LJCutCoulRBLForceOp<device::DEVICE_GPU>()(
      ref_make_box(lo, hi), (rbmd::Real)rs, (rbmd::Real)rc, n, sample_num, pice,
      (rbmd::Real)alpha, (rbmd::Real)qqr2e, type, sigma, eps, start, end, core, shell, shell_num,
      q, x, y, z, fx, fy, fz);
  return ref_sync();
}

int ref_fix_rbl(int n, double cx, double cy, double cz, rbmd::Real* fx, rbmd::Real* fy,
                rbmd::Real* fz) {
  op::FixRBLForceOp<device::DEVICE_GPU>()(n, (rbmd::Real)cx, (rbmd::Real)cy, (rbmd::Real)cz, fx,
                                          fy, fz);
  return ref_sync();
}

int ref_pair_verlet(const double* lo, const double* hi, double rc, int n, double alpha,
                    double qqr2e, const int* type, const rbmd::Real* sigma, const rbmd::Real* eps,
                    const int* start, const int* end, const int* nbrs, const rbmd::Real* q,
                    const rbmd::Real* x, const rbmd::Real* y, const rbmd::Real* z, rbmd::Real* fx,
                    rbmd::Real* fy, rbmd::Real* fz, rbmd::Real* flat_virial, rbmd::Real* evdwl,
                    rbmd::Real* ecoul) {
  op::LJCutCoulForceOp<device::DEVICE_GPU>()(ref_make_box(lo, hi), (rbmd::Real)rc, n,
                                             (rbmd::Real)alpha, (rbmd::Real)qqr2e, type, sigma,
                                             eps, start, end, nbrs, q, x, y, z, fx, fy, fz,
                                             flat_virial, evdwl, ecoul);
  return ref_sync();
}

/* SpecialLJCutCoulRBLForceOp (cvff_op.hip.cu:3978-4040): the CVFF RBL pair
 * force with special-bond weights over the core list (start / end / core) and
 * the column-major shell list (shell[k * n + i]).  lj_force12 / lj_force6 are
 * the [ntypes x ntypes] tables of CVFF::Init (cvff.cpp:855-872); nspecial
 * [n][3] and special [n][maxspecial] (partner global ids) follow the atoms.
 * The functor runs the kernel named by RBMD_PAIR_KERNEL (unset: optimized). */
int ref_pair_rbl_special(const double* lo, const double* hi, double rs, double rc, int n,
                         int sample_num, int pice, double alpha, double qqr2e, const int* type,
                         const int* gid, int ntypes, const rbmd::Real* lj12,
                         const rbmd::Real* lj6, const int* start, const int* end,
                         const int* core, const int* shell, const int* shell_num,
                         const int* nspecial, const int* special, int maxspecial, double w12,
                         double w13, double w14, const rbmd::Real* q, const rbmd::Real* x,
                         const rbmd::Real* y, const rbmd::Real* z, rbmd::Real* fx,
                         rbmd::Real* fy, rbmd::Real* fz) {
  op::SpecialLJCutCoulRBLForceOp<device::DEVICE_GPU>()(
      ref_make_box(lo, hi), (rbmd::Real)rs, (rbmd::Real)rc, n, sample_num, pice,
      (rbmd::Real)alpha, (rbmd::Real)qqr2e, type, gid, ntypes, lj12, lj6, start, end, core, shell,
      shell_num, nspecial, special, maxspecial, (rbmd::Real)w12, (rbmd::Real)w13,
      (rbmd::Real)w14, q, x, y, z, fx, fy, fz);
  return ref_sync();
}

}  // extern "C"
