// rbx_capi_f32.cu -- the op-level entry points for the reference's default
// build, where rbmd::Real is float (cmake/option.cmake: ENABLE_DOUBLE OFF,
// src/common/types.h:4-8).  Same argument order as the FP64 entries; every
// Real buffer and scalar is float.
//
// k-space: the structure factor and the RBE force run the mixed-form kernels
// (32-bit fixed-point fractional coordinates, exact integer phase m.u mod
// 2^32, FP32 sincos, FP64 cross-block reduction), so their error is that of
// the FP32 arithmetic on the phase, not of an FP32 k.r.  Energy and virial
// are summed in FP64.  Real space: every membership test (list predicate,
// force windows) is evaluated in float exactly as the float build evaluates
// it, so lists and kept pairs are the float build's; force values are FP64
// sums stored in float.
#include <cuda_runtime.h>

#include <initializer_list>

#include "rbx.h"
#include "rbx_capi_util.h"
#include "rbx_common.cuh"
#include "rbx_kernels.h"

namespace rbx {

__global__ void k_widen(int n, const float* __restrict__ src, double* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (double)src[i];
}
__global__ void k_narrow(int n, const double* __restrict__ src, float* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (float)src[i];
}

int launch_widen(int n, const float* src, double* dst, cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_widen<<<(n + 255) / 256, 256, 0, st>>>(n, src, dst);
  count_launch();
  return check_launch("widen");
}
int launch_narrow(int n, const double* src, float* dst, cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_narrow<<<(n + 255) / 256, 256, 0, st>>>(n, src, dst);
  count_launch();
  return check_launch("narrow");
}

namespace {
// Device scratch freed on the stream when the call returns.
struct Scratch {
  cudaStream_t st;
  void* p[8] = {};
  int k = 0;
  explicit Scratch(cudaStream_t s) : st(s) {}
  template <typename T>
  int get(T** out, size_t count) {
    RBX_TRY(async_alloc(out, count, st));
    p[k++] = *out;
    return RBX_OK;
  }
  ~Scratch() {
    for (int i = 0; i < k; ++i) cudaFreeAsync(p[i], st);
  }
};

// Widened copies of n-element float arrays (contiguous, in argument order).
int widen_all(Scratch& s, int n, std::initializer_list<const float*> src, double** dst) {
  double* w = nullptr;
  RBX_TRY(s.get(&w, (size_t)n * src.size()));
  *dst = w;
  int k = 0;
  for (const float* a : src) RBX_TRY(launch_widen(n, a, w + (size_t)n * k++, s.st));
  return RBX_OK;
}

// Fixed-point records {u_x, u_y, u_z, q} of float positions and charges.
int fixed_records(Scratch& s, const DBox& b, int n, const float* q, const float* x,
                  const float* y, const float* z, uint4** atoms) {
  double* w = nullptr;
  RBX_TRY(widen_all(s, n, {x, y, z, q}, &w));
  RBX_TRY(s.get(atoms, (size_t)n));
  return launch_to_fixed(b, n, w, w + n, w + 2 * (size_t)n, w + 3 * (size_t)n, *atoms, s.st);
}
}  // namespace
}  // namespace rbx

using namespace rbx;

extern "C" {

int rbx_rbe_structure_factor_f32(const rbx_box* box, int num_atoms, int p_number,
                                 const float* charge, const float* p_sample_x,
                                 const float* p_sample_y, const float* p_sample_z,
                                 const float* px, const float* py, const float* pz,
                                 float* density_real, float* density_imag, void* stream) {
  RBX_CHECK_BOX(box);
  if (num_atoms < 0 || p_number < 0) {
    set_error("rbx_rbe_structure_factor_f32: negative size");
    return RBX_ERR_INVALID;
  }
  if (p_number == 0) return RBX_OK;
  RBX_TRY(require_device());
  cudaStream_t st = (cudaStream_t)stream;
  Scratch s(st);
  const DBox b = make_dbox(*box);
  double* m = nullptr;  // samples widened: mx, my, mz
  RBX_TRY(widen_all(s, p_number, {p_sample_x, p_sample_y, p_sample_z}, &m));
  const int nb = rbe_partial_blocks(num_atoms);
  double *part = nullptr, *rho = nullptr;
  RBX_TRY(s.get(&part, (size_t)2 * nb * p_number));
  RBX_TRY(s.get(&rho, (size_t)2 * p_number));
  double *pr = part, *pi = part + (size_t)nb * p_number;
  if (num_atoms > 0) {
    uint4* atoms = nullptr;
    int* mi = nullptr;
    RBX_TRY(fixed_records(s, b, num_atoms, charge, px, py, pz, &atoms));
    RBX_TRY(s.get(&mi, (size_t)3 * p_number));
    RBX_TRY(launch_m_to_int(p_number, m, m + p_number, m + 2 * p_number, mi, st));
    RBX_TRY(launch_rbe_rho_partial_mixed(num_atoms, p_number, mi, atoms, pr, pi, nb, st));
  } else {
    cudaMemsetAsync(part, 0, sizeof(double) * 2 * nb * p_number, st);
  }
  RBX_TRY(launch_rbe_finalize(b, p_number, nb, pr, pi, m, m + p_number, m + 2 * p_number, 1.0,
                              0.0, 1.0, 0.0, 0.0, rho, rho + p_number, nullptr, nullptr, nullptr,
                              0, nullptr, 0, nullptr, nullptr, st));
  RBX_TRY(launch_narrow(p_number, rho, density_real, st));
  return launch_narrow(p_number, rho + p_number, density_imag, st);
}

int rbx_rbe_force_f32(const rbx_box* box, int num_atoms, int p_number, float alpha,
                      float rbe_sum_gauss, float qqr2e, const float* real_array,
                      const float* imag_array, const float* charge, const float* p_sample_x,
                      const float* p_sample_y, const float* p_sample_z, const float* px,
                      const float* py, const float* pz, float* fx, float* fy, float* fz,
                      void* stream) {
  RBX_CHECK_BOX(box);
  if (num_atoms < 0 || p_number <= 0) {
    set_error("rbx_rbe_force_f32: need num_atoms >= 0 and p_number > 0");
    return RBX_ERR_INVALID;
  }
  if (num_atoms == 0) return RBX_OK;
  RBX_TRY(require_device());
  cudaStream_t st = (cudaStream_t)stream;
  Scratch s(st);
  const DBox b = make_dbox(*box);
  double *m = nullptr, *rho = nullptr, *f = nullptr;
  RBX_TRY(widen_all(s, p_number, {p_sample_x, p_sample_y, p_sample_z}, &m));
  RBX_TRY(widen_all(s, p_number, {real_array, imag_array}, &rho));
  KTab* tab = nullptr;
  RBX_TRY(s.get(&tab, (size_t)p_number));
  RBX_TRY(launch_rbe_finalize(b, p_number, 1, rho, rho + p_number, m, m + p_number,
                              m + 2 * p_number, alpha, rbe_sum_gauss, qqr2e, 0.0, 0.0, nullptr,
                              nullptr, nullptr, nullptr, tab, 0, nullptr, 0, nullptr, nullptr,
                              st));
  uint4* atoms = nullptr;
  RBX_TRY(fixed_records(s, b, num_atoms, charge, px, py, pz, &atoms));
  RBX_TRY(s.get(&f, (size_t)3 * num_atoms));
  RbeForceOut o;
  o.f_out_x = f;
  o.f_out_y = f + num_atoms;
  o.f_out_z = f + 2 * (size_t)num_atoms;
  RBX_TRY(launch_rbe_force_mixed(num_atoms, p_number, tab, atoms, o, st));
  RBX_TRY(launch_narrow(num_atoms, o.f_out_x, fx, st));
  RBX_TRY(launch_narrow(num_atoms, o.f_out_y, fy, st));
  return launch_narrow(num_atoms, o.f_out_z, fz, st);
}

int rbx_rbe_energy_virial_f32(const rbx_box* box, int p, float alpha, float rbe_sum_gauss,
                              float qqrd2e, float qsqsum, float qsum, const float* real_array,
                              const float* imag_array, const float* p_sample_x,
                              const float* p_sample_y, const float* p_sample_z,
                              float* virial_tensor, float* energy, void* stream) {
  RBX_CHECK_BOX(box);
  if (p <= 0 || !virial_tensor || !energy) {
    set_error("rbx_rbe_energy_virial_f32: need p > 0 and output pointers");
    return RBX_ERR_INVALID;
  }
  RBX_TRY(require_device());
  cudaStream_t st = (cudaStream_t)stream;
  Scratch s(st);
  const DBox b = make_dbox(*box);
  double *m = nullptr, *rho = nullptr, *out = nullptr;
  RBX_TRY(widen_all(s, p, {p_sample_x, p_sample_y, p_sample_z}, &m));
  RBX_TRY(widen_all(s, p, {real_array, imag_array}, &rho));
  RBX_TRY(s.get(&out, 7));  // virial[6], energy
  RBX_TRY(launch_rbe_finalize(b, p, 1, rho, rho + p, m, m + p, m + 2 * p, alpha, rbe_sum_gauss,
                              qqrd2e, qsqsum, qsum, nullptr, nullptr, out + 6, out, nullptr, 0,
                              nullptr, 0, nullptr, nullptr, st));
  RBX_TRY(launch_narrow(6, out, virial_tensor, st));
  return launch_narrow(1, out + 6, energy, st);
}

int rbx_rbl_filter_f32(float core_cutoff_2, float force_cutoff_2, int total_atom_num,
                       const int* atoms_id, const float* px, const float* py, const float* pz,
                       const int* candidate_start, const int* candidate_end,
                       const int* candidate_neighbors, const int* max_core_neighbor_num,
                       const int* core_start, int* core_end, int* core_neighbors,
                       int random_neighbor_capacity, int* random_neighbors,
                       int* random_neighbors_num, int* required_random_neighbor_capacity,
                       const rbx_box* box, int* should_realloc, int selection_frequency,
                       int sample_epoch, void* stream) {
  RBX_CHECK_BOX(box);
  if (total_atom_num < 0 || random_neighbor_capacity < 0) {
    set_error("rbx_rbl_filter_f32: negative size");
    return RBX_ERR_INVALID;
  }
  RBX_TRY(require_device());
  return launch_ref_rbl_filter(core_cutoff_2, force_cutoff_2, total_atom_num, atoms_id, px, py,
                               pz, candidate_start, candidate_end, candidate_neighbors,
                               max_core_neighbor_num, core_start, core_end, core_neighbors,
                               random_neighbor_capacity, random_neighbors, random_neighbors_num,
                               required_random_neighbor_capacity, make_dbox(*box), should_realloc,
                               make_divtest(selection_frequency), sample_epoch,
                               (cudaStream_t)stream);
}

int rbx_pair_force_rbl_f32(const rbx_box* box, float rs, float rc, int num_atoms,
                           int neighbor_sample_num, int pice_num, float alpha, float qqr2e,
                           const int* atoms_type, const float* sigma, const float* eps,
                           const int* start_id, const int* end_id, const int* id_verletlist,
                           const int* id_random_neighbor, const int* random_neighbor_num,
                           const float* charge, const float* px, const float* py,
                           const float* pz, float* fx, float* fy, float* fz, void* stream) {
  (void)neighbor_sample_num;
  RBX_CHECK_BOX(box);
  if (num_atoms < 0) {
    set_error("rbx_pair_force_rbl_f32: negative num_atoms");
    return RBX_ERR_INVALID;
  }
  RBX_TRY(require_device());
  return launch_ref_pair_rbl(make_dbox(*box), rs, rc, num_atoms, pice_num, alpha, qqr2e,
                             atoms_type, sigma, eps, start_id, end_id, id_verletlist,
                             id_random_neighbor, random_neighbor_num, charge, px, py, pz, fx, fy,
                             fz, (cudaStream_t)stream);
}

int rbx_fix_rbl_force_f32(int num_atoms, float* fx, float* fy, float* fz, float* mean_out,
                          void* stream) {
  if (num_atoms <= 0) {
    set_error("rbx_fix_rbl_force_f32: num_atoms must be > 0");
    return RBX_ERR_INVALID;
  }
  RBX_TRY(require_device());
  cudaStream_t st = (cudaStream_t)stream;
  Scratch s(st);
  double* mean = nullptr;
  RBX_TRY(s.get(&mean, 3));
  RBX_TRY(launch_reduce_cols(num_atoms, 1, fx, mean, 1.0 / num_atoms, st));
  RBX_TRY(launch_reduce_cols(num_atoms, 1, fy, mean + 1, 1.0 / num_atoms, st));
  RBX_TRY(launch_reduce_cols(num_atoms, 1, fz, mean + 2, 1.0 / num_atoms, st));
  RBX_TRY(launch_sub_mean(num_atoms, fx, fy, fz, mean, st));
  if (mean_out) RBX_TRY(launch_narrow(3, mean, mean_out, st));
  return RBX_OK;
}

int rbx_pair_force_verlet_f32(const rbx_box* box, float cut_off, int num_atoms, float alpha,
                              float qqr2e, const int* atoms_type, const float* sigma,
                              const float* eps, const int* start_id, const int* end_id,
                              const int* id_verletlist, const float* charge, const float* px,
                              const float* py, const float* pz, float* fx, float* fy, float* fz,
                              float* flat_virial, float* total_evdwl, float* total_ecoul,
                              void* stream) {
  RBX_CHECK_BOX(box);
  if (num_atoms < 0) {
    set_error("rbx_pair_force_verlet_f32: negative num_atoms");
    return RBX_ERR_INVALID;
  }
  if (num_atoms == 0) return RBX_OK;
  RBX_TRY(require_device());
  cudaStream_t st = (cudaStream_t)stream;
  Scratch s(st);
  double *epart = nullptr, *tot = nullptr;
  RBX_TRY(s.get(&epart, (size_t)2 * num_atoms));
  RBX_TRY(s.get(&tot, 2));
  RBX_TRY(launch_ref_pair_verlet(make_dbox(*box), cut_off, num_atoms, alpha, qqr2e, atoms_type,
                                 sigma, eps, start_id, end_id, id_verletlist, charge, px, py, pz,
                                 fx, fy, fz, flat_virial, epart, st));
  RBX_TRY(launch_reduce_cols(num_atoms, 2, epart, tot, 1.0, st));
  if (total_evdwl) RBX_TRY(launch_narrow(1, tot, total_evdwl, st));
  if (total_ecoul) RBX_TRY(launch_narrow(1, tot + 1, total_ecoul, st));
  return RBX_OK;
}

}  // extern "C"
