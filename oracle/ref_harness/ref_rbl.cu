/* Reference-kernel harness, RBL lists: RBMD's own FilterRblNeighborCandidatesOp
 * (src/neighbor_list/src/op/rocm/rbl_full_neighbor_list_op.hip.cu:237-334),
 * compiled in place.  Test infrastructure only. */
#include "neighbor_list/src/op/rocm/rbl_full_neighbor_list_op.hip.cu"
#include "ref_common.h"

extern "C" int ref_rbl_filter(double core2, double force2, int n, const int* gid,
                              const rbmd::Real* x, const rbmd::Real* y, const rbmd::Real* z,
                              const int* cstart, const int* cend, const int* cand,
                              const int* core_cap, const int* core_start, int* core_end, int* core,
                              int shell_cap, int* shell, int* shell_num, int* required,
                              const double* lo, const double* hi, int* realloc, int freq,
                              int epoch) {
  op::FilterRblNeighborCandidatesOp<device::DEVICE_GPU>()(
      (rbmd::Real)core2, (rbmd::Real)force2, n, gid, x, y, z, cstart, cend, cand, core_cap,
      core_start, core_end, core, shell_cap, shell, shell_num, required, ref_make_box(lo, hi),
      realloc, freq, epoch);
  return ref_sync();
}
