/* Reference-kernel harness, SHAKE / RATTLE: RBMD's own ShakeAOp / ShakeBOp
 * (src/simulate_pipeline/src/controller/shake_controller/shake_controller_op/
 * rocm/shake_controller_op.hip.cu:19-660, 1188-1238), compiled in place.
 * Device arrays; angles are (H, O, H) global-id triples, id2idx maps a global
 * id to its atom index.  Test infrastructure only. */
#include "simulate_pipeline/src/controller/shake_controller/shake_controller_op/rocm/shake_controller_op.hip.cu"
#include "ref_common.h"

extern "C" {

int ref_shake_a(const double* lo, const double* hi, int nangle, double dt, double fmt2v,
                const int* id2idx, const rbmd::Real* mass, const int* type, const int* angles,
                rbmd::Real* px, rbmd::Real* py, rbmd::Real* pz, rbmd::Real* vx, rbmd::Real* vy,
                rbmd::Real* vz, const rbmd::Real* fx, const rbmd::Real* fy,
                const rbmd::Real* fz, int* flagx, int* flagy, int* flagz) {
  op::ShakeAOp<device::DEVICE_GPU>()(nangle, (rbmd::Real)dt, (rbmd::Real)fmt2v,
                                     ref_make_box(lo, hi), id2idx, mass, type,
                                     reinterpret_cast<const Id3*>(angles), px, py, pz, vx, vy, vz,
                                     fx, fy, fz, flagx, flagy, flagz);
  return ref_sync();
}

int ref_shake_b(const double* lo, const double* hi, int nangle, double dt, double fmt2v,
                const int* id2idx, const rbmd::Real* mass, const int* type, const int* angles,
                const rbmd::Real* px, const rbmd::Real* py, const rbmd::Real* pz,
                rbmd::Real* vx, rbmd::Real* vy, rbmd::Real* vz, const rbmd::Real* fx,
                const rbmd::Real* fy, const rbmd::Real* fz) {
  op::ShakeBOp<device::DEVICE_GPU>()(nangle, (rbmd::Real)dt, (rbmd::Real)fmt2v,
                                     ref_make_box(lo, hi), id2idx, mass, type,
                                     reinterpret_cast<const Id3*>(angles), px, py, pz, vx, vy, vz,
                                     fx, fy, fz);
  return ref_sync();
}

}  // extern "C"
