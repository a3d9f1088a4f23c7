// rbx_capi.cu -- error plumbing and the op-level C ABI (include/rbx.h).
#include <math.h>
#include <stdarg.h>
#include <stdio.h>

#include <atomic>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "rbx.h"
#include "rbx_common.cuh"
#include "rbx_kernels.h"
#include "rbx_capi_util.h"

namespace rbx {

static thread_local std::string g_err;
static std::atomic<uint64_t> g_launches{0};

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
}

void count_launch(int n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }

int check_launch(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("%s: %s", what, cudaGetErrorString(e));
    return RBX_ERR_CUDA;
  }
  return RBX_OK;
}

int sm_count() {
  static thread_local int cached_dev = -1, cached = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return cached;
  if (dev != cached_dev) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0)
      cached = v;
    cached_dev = dev;
  }
  return cached;
}

int grid_for(long long work, int per_block, int max_blocks) {
  long long b = (work + per_block - 1) / per_block;
  if (b > max_blocks) b = max_blocks;
  return b < 1 ? 1 : (int)b;
}

// The library runs only on sm_100-class devices; there is no CPU path.
int require_device() {
  int dev = 0, count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count <= 0) {
    cudaGetLastError();
    set_error("no CUDA device available (librbx has no CPU fallback)");
    return RBX_ERR_DEVICE;
  }
  if (cudaGetDevice(&dev) != cudaSuccess) {
    set_error("cudaGetDevice failed");
    return RBX_ERR_DEVICE;
  }
  int major = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  if (major != 10) {
    set_error("device %d has compute capability %d.x; librbx is built for sm_100a only", dev,
              major);
    return RBX_ERR_DEVICE;
  }
  return RBX_OK;
}

// Per-axis inverse-CDF table of the RBE importance density (see the oracle's
// restatement): order m = 0, +1, -1, +2, -2, ... down to weight 1e-20,
// returned as cumulative sums.
int rbe_axis_table(double L, double alpha, double* w, int max_entries, double* total) {
  const double c = (M_PI * M_PI) / (alpha * L * L);
  int cnt = 0;
  double z = 0.0;
  for (int m = 0;; ++m) {
    const double v = exp(-c * (double)m * (double)m);
    if (m > 0 && v < 1e-20) break;
    if (cnt + (m == 0 ? 1 : 2) > max_entries) return -1;
    if (m == 0) {
      w[cnt++] = v;
      z += v;
    } else {
      w[cnt++] = v;
      w[cnt++] = v;
      z += v;
      z += v;
    }
  }
  *total = z;
  // cumulative form (left-to-right sums, the oracle's scan order)
  double acc = 0.0;
  for (int t = 0; t < cnt; ++t) {
    acc += w[t];
    w[t] = acc;
  }
  return cnt;
}

double gauss_sum(const rbx_box& b, double alpha) {
  double h[3] = {0, 0, 0};
  for (int d = 0; d < 3; ++d) {
    const double L = b.hi[d] - b.lo[d];
    const double factor = -(alpha * L * L);
    for (int m = -10; m <= 10; ++m) h[d] += exp((double)(m * m) * factor);
    h[d] *= sqrt(-(factor) / M_PI);
  }
  return h[0] * h[1] * h[2] - 1.0;
}

// dS/dalpha of gauss_sum: H_d = sqrt(alpha L^2 / pi) sum_m e^{-alpha L^2 m^2}.
double gauss_sum_dalpha(const rbx_box& b, double alpha) {
  double h[3], dh[3];
  for (int d = 0; d < 3; ++d) {
    const double L = b.hi[d] - b.lo[d];
    double w = 0.0, w2 = 0.0;
    for (int m = -10; m <= 10; ++m) {
      const double e = exp(-alpha * L * L * (double)(m * m));
      w += e;
      w2 += L * L * (double)(m * m) * e;
    }
    const double pre = sqrt(alpha * L * L / M_PI);
    h[d] = pre * w;
    dh[d] = pre * w / (2.0 * alpha) - pre * w2;
  }
  return dh[0] * h[1] * h[2] + h[0] * dh[1] * h[2] + h[0] * h[1] * dh[2];
}

int rbl_freq(int n_global, const rbx_box& b, double r_core, double cut_off, int sample_num) {
  const double V = (b.hi[0] - b.lo[0]) * (b.hi[1] - b.lo[1]) * (b.hi[2] - b.lo[2]);
  const double rho = (double)n_global / V;
  const double coeff = 1.0 + (0.05 / rho - 0.05);
  const int icoeff = (int)round(coeff);
  const int rs = (int)(icoeff * rho * ceil(4.0 / 3.0 * M_PI * pow(r_core, 3)) + 1);
  const int rc = (int)(icoeff * rho * ceil(4.0 / 3.0 * M_PI * pow(cut_off, 3)) + 1);
  const int shell = rc - rs;
  return shell <= sample_num ? 1 : (int)ceil((double)shell / (double)sample_num);
}


}  // namespace rbx

using namespace rbx;

extern "C" {

const char* rbx_last_error(void) { return g_err.c_str(); }
int rbx_version(void) { return RBX_VERSION; }
uint64_t rbx_launch_count(void) { return g_launches.load(); }

int rbx_rbe_gauss_sum(const rbx_box* box, double alpha, double* S) {
  RBX_CHECK_BOX(box);
  if (!(alpha > 0.0) || !S) {
    set_error("rbx_rbe_gauss_sum: alpha must be > 0");
    return RBX_ERR_INVALID;
  }
  *S = gauss_sum(*box, alpha);
  return RBX_OK;
}

int rbx_rbl_params(int n_global, const rbx_box* box, double r_core, double cut_off,
                   int neighbor_sample_num, int* freq) {
  RBX_CHECK_BOX(box);
  if (n_global <= 0 || neighbor_sample_num <= 0 || !freq) {
    set_error("rbx_rbl_params: invalid RBL global density inputs");
    return RBX_ERR_INVALID;
  }
  *freq = rbl_freq(n_global, *box, r_core, cut_off, neighbor_sample_num);
  return RBX_OK;
}

int rbx_rbe_sample(const rbx_box* box, double alpha, int p, uint64_t seed, int64_t step,
                   double* p_sample_x, double* p_sample_y, double* p_sample_z, void* stream) {
  RBX_CHECK_BOX(box);
  if (p < 0 || !(alpha > 0.0)) {
    set_error("rbx_rbe_sample: need p >= 0 and alpha > 0");
    return RBX_ERR_INVALID;
  }
  RBX_TRY(require_device());
  cudaStream_t st = (cudaStream_t)stream;
  enum { MAXT = 4096 };
  static thread_local double w[3 * MAXT];
  int cnt[3];
  double tot[3];
  int off = 0;
  for (int d = 0; d < 3; ++d) {
    cnt[d] = rbe_axis_table(box->hi[d] - box->lo[d], alpha, w + off, MAXT, &tot[d]);
    if (cnt[d] < 0) {
      set_error("rbx_rbe_sample: k-sampler table too large");
      return RBX_ERR_SAMPLER;
    }
    off += cnt[d];
  }
  double* dtab = nullptr;
  int* dstatus = nullptr;
  RBX_TRY(async_alloc(&dtab, (size_t)off, st));
  RBX_TRY(async_alloc(&dstatus, 1, st));
  cudaMemcpyAsync(dtab, w, sizeof(double) * off, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(dstatus, 0, sizeof(int), st);
  int rc = launch_rbe_sample(p, dtab, cnt, tot, seed, step, nullptr, p_sample_x, p_sample_y,
                             p_sample_z, nullptr, dstatus, st);
  int hstatus = 0;
  if (!rc) {
    cudaMemcpyAsync(&hstatus, dstatus, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) rc = check_launch("rbe_sample sync");
  }
  cudaFreeAsync(dtab, st);
  cudaFreeAsync(dstatus, st);
  if (!rc && hstatus) {
    set_error("rbx_rbe_sample: a sample needed more than 64 draws to avoid m = 0");
    return RBX_ERR_SAMPLER;
  }
  return rc;
}

int rbx_rbe_structure_factor(const rbx_box* box, int num_atoms, int p_number,
                             const double* charge, const double* p_sample_x,
                             const double* p_sample_y, const double* p_sample_z,
                             const double* px, const double* py, const double* pz,
                             double* density_real, double* density_imag, void* stream) {
  RBX_CHECK_BOX(box);
  if (num_atoms < 0 || p_number < 0) {
    set_error("rbx_rbe_structure_factor: negative size");
    return RBX_ERR_INVALID;
  }
  if (p_number == 0) return RBX_OK;
  RBX_TRY(require_device());
  cudaStream_t st = (cudaStream_t)stream;
  const DBox b = make_dbox(*box);
  const int nb = rbe_partial_blocks(num_atoms);
  double *pr = nullptr, *pi = nullptr;
  RBX_TRY(async_alloc(&pr, (size_t)nb * p_number, st));
  RBX_TRY(async_alloc(&pi, (size_t)nb * p_number, st));
  int rc = RBX_OK;
  if (num_atoms > 0) {
    rc = launch_rbe_rho_partial_f64(b, num_atoms, p_number, p_sample_x, p_sample_y, p_sample_z,
                                    charge, px, py, pz, pr, pi, nb, st);
  } else {
    cudaMemsetAsync(pr, 0, sizeof(double) * nb * p_number, st);
    cudaMemsetAsync(pi, 0, sizeof(double) * nb * p_number, st);
  }
  if (!rc)
    rc = launch_rbe_finalize(b, p_number, nb, pr, pi, p_sample_x, p_sample_y, p_sample_z, 1.0,
                             0.0, 1.0, 0.0, 0.0, density_real, density_imag, nullptr, nullptr,
                             nullptr, 0, nullptr, 0, nullptr, nullptr, st);
  cudaFreeAsync(pr, st);
  cudaFreeAsync(pi, st);
  return rc;
}

int rbx_rbe_force(const rbx_box* box, int num_atoms, int p_number, double alpha,
                  double rbe_sum_gauss, double qqr2e, const double* real_array,
                  const double* imag_array, const double* charge, const double* p_sample_x,
                  const double* p_sample_y, const double* p_sample_z, const double* px,
                  const double* py, const double* pz, double* fx, double* fy, double* fz,
                  void* stream) {
  RBX_CHECK_BOX(box);
  if (num_atoms < 0 || p_number <= 0) {
    set_error("rbx_rbe_force: need num_atoms >= 0 and p_number > 0");
    return RBX_ERR_INVALID;
  }
  if (num_atoms == 0) return RBX_OK;
  RBX_TRY(require_device());
  cudaStream_t st = (cudaStream_t)stream;
  const DBox b = make_dbox(*box);
  KTab* tab = nullptr;
  RBX_TRY(async_alloc(&tab, (size_t)p_number, st));
  int rc = launch_rbe_finalize(b, p_number, 1, real_array, imag_array, p_sample_x, p_sample_y,
                               p_sample_z, alpha, rbe_sum_gauss, qqr2e, 0.0, 0.0, nullptr,
                               nullptr, nullptr, nullptr, tab, 0, nullptr, 0, nullptr, nullptr, st);
  if (!rc) {
    RbeForceOut o;
    o.f_out_x = fx;
    o.f_out_y = fy;
    o.f_out_z = fz;
    rc = launch_rbe_force_f64(num_atoms, p_number, tab, charge, px, py, pz, o, st);
  }
  cudaFreeAsync(tab, st);
  return rc;
}

int rbx_rbe_energy_virial(const rbx_box* box, int p, double alpha, double rbe_sum_gauss,
                          double qqrd2e, double qsqsum, double qsum, const double* real_array,
                          const double* imag_array, const double* p_sample_x,
                          const double* p_sample_y, const double* p_sample_z,
                          double* virial_tensor, double* energy, void* stream) {
  RBX_CHECK_BOX(box);
  if (p <= 0 || !virial_tensor || !energy) {
    set_error("rbx_rbe_energy_virial: need p > 0 and output pointers");
    return RBX_ERR_INVALID;
  }
  RBX_TRY(require_device());
  const DBox b = make_dbox(*box);
  return launch_rbe_finalize(b, p, 1, real_array, imag_array, p_sample_x, p_sample_y, p_sample_z,
                             alpha, rbe_sum_gauss, qqrd2e, qsqsum, qsum, nullptr, nullptr, energy,
                             virial_tensor, nullptr, 0, nullptr, 0, nullptr, nullptr,
                             (cudaStream_t)stream);
}

int rbx_ewald_force(const rbx_box* box, int num_atoms, const int kmax[3], double alpha,
                    double qqr2e, const double* charge, const double* px, const double* py,
                    const double* pz, double* fx, double* fy, double* fz, double* energy,
                    void* stream) {
  RBX_CHECK_BOX(box);
  if (!kmax || kmax[0] < 0 || kmax[1] < 0 || kmax[2] < 0 || !(alpha > 0.0) || num_atoms < 0) {
    set_error("rbx_ewald_force: invalid kmax/alpha/num_atoms");
    return RBX_ERR_INVALID;
  }
  RBX_TRY(require_device());
  cudaStream_t st = (cudaStream_t)stream;
  const int nk = (2 * kmax[0] + 1) * (2 * kmax[1] + 1) * (2 * kmax[2] + 1) - 1;
  if (nk <= 0) return RBX_OK;
  double *re = nullptr, *im = nullptr, *kv = nullptr;
  RBX_TRY(async_alloc(&re, nk, st));
  RBX_TRY(async_alloc(&im, nk, st));
  RBX_TRY(async_alloc(&kv, (size_t)3 * nk, st));
  double qsq = 0.0;
  int rc = RBX_OK;
  if (energy && num_atoms > 0) {  // sum q^2 for the self-energy term
    std::vector<double> hq(num_atoms);
    rc = cudaMemcpyAsync(hq.data(), charge, sizeof(double) * num_atoms, cudaMemcpyDeviceToHost,
                         st) == cudaSuccess && cudaStreamSynchronize(st) == cudaSuccess
             ? RBX_OK
             : check_launch("ewald charge copy");
    for (int i = 0; i < num_atoms; ++i) qsq += hq[i] * hq[i];
  }
  const DBox b = make_dbox(*box);
  if (!rc)
    rc = launch_ewald(b, num_atoms, kmax, alpha, qqr2e, qsq, charge, px, py, pz, re, im, kv, fx,
                      fy, fz, energy, st);
  cudaFreeAsync(re, st);
  cudaFreeAsync(im, st);
  cudaFreeAsync(kv, st);
  return rc;
}

int rbx_cell_grid(const rbx_box* box, double neighbor_cutoff, int dims[3]) {
  RBX_CHECK_BOX(box);
  if (!(neighbor_cutoff > 0.0) || !dims) {
    set_error("rbx_cell_grid: invalid neighbor cutoff");
    return RBX_ERR_INVALID;
  }
  for (int d = 0; d < 3; ++d) {
    const double nd = floor((box->hi[d] - box->lo[d]) / neighbor_cutoff);
    dims[d] = nd >= 1.0 ? (int)nd : 0;
    if (dims[d] < 3) {
      set_error("The current simulation domain is too small for PBC: dimension %d has %d cells "
                "of edge >= %g (need 3)",
                d, dims[d], neighbor_cutoff);
      return RBX_ERR_INVALID;
    }
  }
  return RBX_OK;
}

size_t rbx_cells_scratch_bytes(int n, int ncell) { return cells_scratch_bytes(n, ncell); }

int rbx_cells_sort(const rbx_box* box, double neighbor_cutoff, int n, const double* px,
                   const double* py, const double* pz, int* perm, int* cell_of_sorted,
                   int* cell_start, void* scratch, void* stream) {
  int dims[3];
  RBX_TRY(rbx_cell_grid(box, neighbor_cutoff, dims));
  if (n < 0 || !scratch) {
    set_error("rbx_cells_sort: invalid n or scratch");
    return RBX_ERR_INVALID;
  }
  RBX_TRY(require_device());
  cudaStream_t st = (cudaStream_t)stream;
  int* status = nullptr;
  RBX_TRY(async_alloc(&status, 1, st));
  cudaMemsetAsync(status, 0, sizeof(int), st);
  int rc = launch_cells_sort(make_dbox(*box), dims, n, px, py, pz, perm, cell_of_sorted,
                             cell_start, scratch, status, st);
  int h = 0;
  cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && !rc) rc = check_launch("cells_sort sync");
  cudaFreeAsync(status, st);
  if (!rc && h) {
    set_error("rbx_cells_sort: a cell holds more than 2048 atoms");
    return RBX_ERR_CAPACITY;
  }
  return rc;
}

int rbx_nlist_should_reuse(const rbx_box* box, int n, const double* px, const double* py,
                           const double* pz, const double* cached_px, const double* cached_py,
                           const double* cached_pz, double skin, int* reuse,
                           double* max_disp_sq, void* stream) {
  if (!box || n < 0 || !reuse || !(skin >= 0.0)) {
    set_error("rbx_nlist_should_reuse: invalid box/n/skin/reuse");
    return RBX_ERR_INVALID;
  }
  RBX_TRY(require_device());
  cudaStream_t st = (cudaStream_t)stream;
  unsigned long long* d = nullptr;
  RBX_TRY(async_alloc(&d, 1, st));
  cudaMemsetAsync(d, 0, sizeof(unsigned long long), st);
  int rc = launch_max_disp(make_dbox(*box), n, px, py, pz, cached_px, cached_py, cached_pz, d, st);
  unsigned long long bits = 0;
  if (!rc) {
    cudaMemcpyAsync(&bits, d, sizeof(bits), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) rc = check_launch("should_reuse sync");
  }
  cudaFreeAsync(d, st);
  if (rc) return rc;
  double d2;
  memcpy(&d2, &bits, sizeof(d2));
  const double thr = 0.5 * skin;
  *reuse = d2 <= thr * thr ? 1 : 0;
  if (max_disp_sq) *max_disp_sq = d2;
  return RBX_OK;
}

int rbx_full_list(const rbx_box* box, double neighbor_cutoff, int n, const double* px,
                  const double* py, const double* pz, const int* cell_start, int cap, int* count,
                  int* nbrs, int* overflow, void* stream) {
  int dims[3];
  RBX_TRY(rbx_cell_grid(box, neighbor_cutoff, dims));
  if (n < 0 || cap <= 0 || !overflow) {
    set_error("rbx_full_list: invalid n/cap/overflow");
    return RBX_ERR_INVALID;
  }
  RBX_TRY(require_device());
  if (n == 0) return RBX_OK;
  cudaStream_t st = (cudaStream_t)stream;
  char* scratch = nullptr;
  RBX_TRY(async_alloc(&scratch, full_list_scratch_bytes(n, dims[0] * dims[1] * dims[2]), st));
  const int rc = launch_full_list(make_dbox(*box), dims, neighbor_cutoff, n, px, py, pz,
                                  cell_start, cap, count, nbrs, overflow, scratch, st);
  cudaFreeAsync(scratch, st);
  return rc;
}

int rbx_rbl_filter(double core_cutoff_2, double force_cutoff_2, int total_atom_num,
                   const int* atoms_id, const double* px, const double* py, const double* pz,
                   const int* candidate_start, const int* candidate_end,
                   const int* candidate_neighbors, const int* max_core_neighbor_num,
                   const int* core_start, int* core_end, int* core_neighbors,
                   int random_neighbor_capacity, int* random_neighbors, int* random_neighbors_num,
                   int* required_random_neighbor_capacity, const rbx_box* box,
                   int* should_realloc, int selection_frequency, int sample_epoch, void* stream) {
  RBX_CHECK_BOX(box);
  if (total_atom_num < 0 || random_neighbor_capacity < 0) {
    set_error("rbx_rbl_filter: negative size");
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

int rbx_pair_force_rbl(const rbx_box* box, double rs, double rc, int num_atoms,
                       int neighbor_sample_num, int pice_num, double alpha, double qqr2e,
                       const int* atoms_type, const double* sigma, const double* eps,
                       const int* start_id, const int* end_id, const int* id_verletlist,
                       const int* id_random_neighbor, const int* random_neighbor_num,
                       const double* charge, const double* px, const double* py,
                       const double* pz, double* fx, double* fy, double* fz, void* stream) {
  (void)neighbor_sample_num;
  RBX_CHECK_BOX(box);
  if (num_atoms < 0) {
    set_error("rbx_pair_force_rbl: negative num_atoms");
    return RBX_ERR_INVALID;
  }
  RBX_TRY(require_device());
  return launch_ref_pair_rbl(make_dbox(*box), rs, rc, num_atoms, pice_num, alpha, qqr2e,
                             atoms_type, sigma, eps, start_id, end_id, id_verletlist,
                             id_random_neighbor, random_neighbor_num, charge, px, py, pz, fx, fy,
                             fz, (cudaStream_t)stream);
}

int rbx_fix_rbl_force(int num_atoms, double* fx, double* fy, double* fz, double* mean_out,
                      void* stream) {
  if (num_atoms <= 0) {
    set_error("rbx_fix_rbl_force: num_atoms must be > 0");
    return RBX_ERR_INVALID;
  }
  RBX_TRY(require_device());
  cudaStream_t st = (cudaStream_t)stream;
  double* mean = mean_out;
  if (!mean) RBX_TRY(async_alloc(&mean, 3, st));
  int rc = launch_reduce_cols(num_atoms, 1, fx, mean, 1.0 / num_atoms, st);
  if (!rc) rc = launch_reduce_cols(num_atoms, 1, fy, mean + 1, 1.0 / num_atoms, st);
  if (!rc) rc = launch_reduce_cols(num_atoms, 1, fz, mean + 2, 1.0 / num_atoms, st);
  if (!rc) rc = launch_sub_mean(num_atoms, fx, fy, fz, mean, st);
  if (!mean_out) cudaFreeAsync(mean, st);
  return rc;
}

int rbx_pair_force_verlet(const rbx_box* box, double cut_off, int num_atoms, double alpha,
                          double qqr2e, const int* atoms_type, const double* sigma,
                          const double* eps, const int* start_id, const int* end_id,
                          const int* id_verletlist, const double* charge, const double* px,
                          const double* py, const double* pz, double* fx, double* fy, double* fz,
                          double* flat_virial, double* total_evdwl, double* total_ecoul,
                          void* stream) {
  RBX_CHECK_BOX(box);
  if (num_atoms < 0) {
    set_error("rbx_pair_force_verlet: negative num_atoms");
    return RBX_ERR_INVALID;
  }
  if (num_atoms == 0) return RBX_OK;
  RBX_TRY(require_device());
  cudaStream_t st = (cudaStream_t)stream;
  double* epart = nullptr;
  RBX_TRY(async_alloc(&epart, (size_t)2 * num_atoms, st));
  int rc = launch_ref_pair_verlet(make_dbox(*box), cut_off, num_atoms, alpha, qqr2e, atoms_type,
                                  sigma, eps, start_id, end_id, id_verletlist, charge, px, py, pz,
                                  fx, fy, fz, flat_virial, epart, st);
  if (!rc && total_evdwl) rc = launch_reduce_cols(num_atoms, 1, epart, total_evdwl, 1.0, st);
  if (!rc && total_ecoul)
    rc = launch_reduce_cols(num_atoms, 1, epart + num_atoms, total_ecoul, 1.0, st);
  cudaFreeAsync(epart, st);
  return rc;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// rbx_rbe_structure_factor_noalloc: the structure-factor pass for callers that
// cannot let a library allocate device memory.  Its per-block partial sums
// live in a fixed array compiled into the library instead of a temporary.
// ---------------------------------------------------------------------------
namespace {

constexpr int kNoallocBlocks = RBX_NOALLOC_RHO_BLOCKS;  // partial blocks per call
constexpr int kNoallocMaxP = RBX_NOALLOC_RHO_MAX_P;     // largest p_number accepted

// Re and Im partials, k-major: [2][kNoallocMaxP][kNoallocBlocks] doubles (2 MiB).
// Every GPU that loads the library holds this array until the process exits.
static __device__ __align__(256) double g_noalloc_rho_scratch[2 * kNoallocMaxP * kNoallocBlocks];

std::mutex g_noalloc_mu;
double* g_noalloc_addr[256] = {};  // last looked-up device address, per device ordinal

// Device address of the scratch array on the current device.  The array's name
// in host code is only a host-side handle; kernels must be given this address.
// Outside a stream capture the address is looked up on every call (the lookup
// allocates nothing), so a context torn down and created again, e.g. after
// cudaDeviceReset, is picked up; inside a capture, where the lookup may not be
// issued, the address of the last call outside a capture on this device is used.
int noalloc_scratch(cudaStream_t st, double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) {
    cudaGetLastError();
    set_error("rbx_rbe_structure_factor_noalloc: no current CUDA device");
    return RBX_ERR_DEVICE;
  }
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) {
    cudaGetLastError();
    cap = cudaStreamCaptureStatusNone;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (cap != cudaStreamCaptureStatusNone) {
    if (!g_noalloc_addr[dev]) {
      set_error("rbx_rbe_structure_factor_noalloc: the first call on device %d must come before "
                "any stream capture",
                dev);
      return RBX_ERR_INVALID;
    }
  } else {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_rho_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      set_error("rbx_rbe_structure_factor_noalloc: cudaGetSymbolAddress failed on device %d: %s",
                dev, cudaGetErrorString(e));
      return RBX_ERR_CUDA;
    }
    g_noalloc_addr[dev] = (double*)p;
  }
  *out = g_noalloc_addr[dev];
  return RBX_OK;
}

}  // namespace

extern "C" int rbx_rbe_structure_factor_noalloc(const rbx_box* box, int num_atoms, int p_number,
                                                const double* charge, const double* p_sample_x,
                                                const double* p_sample_y,
                                                const double* p_sample_z, const double* px,
                                                const double* py, const double* pz,
                                                double* density_real, double* density_imag,
                                                void* stream) {
  RBX_CHECK_BOX(box);
  if (num_atoms < 0 || p_number < 0) {
    set_error("rbx_rbe_structure_factor_noalloc: negative size");
    return RBX_ERR_INVALID;
  }
  if (p_number > kNoallocMaxP) {
    set_error("rbx_rbe_structure_factor_noalloc: p_number %d exceeds the built-in scratch limit "
              "of %d k-vectors; use rbx_rbe_structure_factor",
              p_number, kNoallocMaxP);
    return RBX_ERR_INVALID;
  }
  if (p_number == 0) return RBX_OK;
  RBX_TRY(require_device());
  cudaStream_t st = (cudaStream_t)stream;
  double* scratch = nullptr;
  RBX_TRY(noalloc_scratch(st, &scratch));
  const DBox b = make_dbox(*box);
  int nb = rbe_partial_blocks(num_atoms);
  if (nb > kNoallocBlocks) nb = kNoallocBlocks;
  double* pr = scratch;
  double* pi = scratch + (size_t)kNoallocMaxP * kNoallocBlocks;
  // Every (k, block) slot the finalize reads is written below, so no clearing
  // is needed; slots left from an earlier, larger call are never read.
  if (num_atoms > 0) {
    RBX_TRY(launch_rbe_rho_partial_f64(b, num_atoms, p_number, p_sample_x, p_sample_y, p_sample_z,
                                       charge, px, py, pz, pr, pi, nb, st));
  } else {
    nb = 1;
    if (cudaMemsetAsync(pr, 0, sizeof(double) * p_number, st) != cudaSuccess ||
        cudaMemsetAsync(pi, 0, sizeof(double) * p_number, st) != cudaSuccess)
      return check_launch("rbx_rbe_structure_factor_noalloc memset");
  }
  return launch_rbe_finalize(b, p_number, nb, pr, pi, p_sample_x, p_sample_y, p_sample_z, 1.0, 0.0,
                             1.0, 0.0, 0.0, density_real, density_imag, nullptr, nullptr, nullptr,
                             0, nullptr, 0, nullptr, nullptr, st);
}

// ---------------------------------------------------------------------------
// RBSOG k-space and VERLET-SOG real space (op level)
// ---------------------------------------------------------------------------
#include <stdexcept>

#include "host/rbsog.h"

namespace {

int cuda_ok(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return RBX_OK;
  set_error("%s: %s", what, cudaGetErrorString(e));
  return RBX_ERR_DEVICE;
}

int rbsog_setup_checked(int level, double cut_off, const rbx_box* box,
                        rbx_host::RbsogSetup* out) {
  try {
    *out = rbx_host::rbsog_setup(level, cut_off, *box);
  } catch (const std::exception& ex) {
    set_error("%s", ex.what());
    return RBX_ERR_INVALID;
  }
  return RBX_OK;
}

}  // namespace

int rbx_rbsog_params(int level, double cut_off, const rbx_box* box, rbx_rbsog_info* out,
                     double* coef, int* direct_m, double* direct_fb) {
  RBX_CHECK_BOX(box);
  if (!out) {
    set_error("rbx_rbsog_params: null output");
    return RBX_ERR_INVALID;
  }
  rbx_host::RbsogSetup s;
  RBX_TRY(rbsog_setup_checked(level, cut_off, box, &s));
  out->level = s.level;
  out->mmax = s.mmax;
  out->b = s.b;
  out->sigma = s.sigma;
  out->w0 = s.w0;
  out->S = s.S;
  out->S_npt = s.S_npt;
  out->self_coeff = s.self_coeff;
  for (int i = 0; i < 6; ++i) out->taylor[i] = s.taylor[i];
  out->n_direct = (int)s.direct_fb.size();
  out->S_full = s.S_full;
  if (coef) std::copy(s.coef.begin(), s.coef.end(), coef);
  if (direct_m) std::copy(s.direct_m.begin(), s.direct_m.end(), direct_m);
  if (direct_fb) std::copy(s.direct_fb.begin(), s.direct_fb.end(), direct_fb);
  return RBX_OK;
}

int rbx_rbsog_sample(const rbx_box* box, int level, double cut_off, int p, uint64_t seed,
                     int64_t step, double* mx, double* my, double* mz, void* stream) {
  RBX_CHECK_BOX(box);
  if (p <= 0 || !mx || !my || !mz) {
    set_error("rbx_rbsog_sample: need p > 0 and output arrays");
    return RBX_ERR_INVALID;
  }
  rbx_host::RbsogSetup s;
  RBX_TRY(rbsog_setup_checked(level, cut_off, box, &s));
  RBX_TRY(require_device());
  cudaStream_t st = (cudaStream_t)stream;
  double *cdf = nullptr, *tables = nullptr, *tot = nullptr;
  int *off = nullptr, *cnt = nullptr, *status = nullptr;
  int rc = async_alloc(&cdf, s.comp_cdf.size(), st);
  if (!rc) rc = async_alloc(&tables, s.tables.size(), st);
  if (!rc) rc = async_alloc(&tot, s.tab_tot.size(), st);
  if (!rc) rc = async_alloc(&off, s.tab_off.size(), st);
  if (!rc) rc = async_alloc(&cnt, s.tab_cnt.size(), st);
  if (!rc) rc = async_alloc(&status, 1, st);
  if (!rc) {
    cudaMemcpyAsync(cdf, s.comp_cdf.data(), sizeof(double) * s.comp_cdf.size(),
                    cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(tables, s.tables.data(), sizeof(double) * s.tables.size(),
                    cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(tot, s.tab_tot.data(), sizeof(double) * s.tab_tot.size(),
                    cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(off, s.tab_off.data(), sizeof(int) * s.tab_off.size(),
                    cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(cnt, s.tab_cnt.data(), sizeof(int) * s.tab_cnt.size(),
                    cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(status, 0, sizeof(int), st);
    RbsogTables t{cdf, (int)s.comp_cdf.size(), s.comp_cdf.back(), tables, off, cnt, tot};
    rc = launch_rbsog_sample(p, t, seed, (uint64_t)step, nullptr, mx, my, mz, nullptr, status, st);
  }
  int hs = 0;
  if (!rc) {
    cudaMemcpyAsync(&hs, status, sizeof(int), cudaMemcpyDeviceToHost, st);
    rc = cuda_ok(cudaStreamSynchronize(st), "rbx_rbsog_sample");
  }
  for (void* ptr : {(void*)cdf, (void*)tables, (void*)tot, (void*)off, (void*)cnt, (void*)status})
    if (ptr) cudaFreeAsync(ptr, st);
  if (!rc && hs) {
    set_error("rbx_rbsog_sample: a sample found no |m|^2 > 1 draw in 64 tries");
    return RBX_ERR_SAMPLER;
  }
  return rc;
}

int rbx_rbsog_force(const rbx_box* box, int level, double cut_off, double qqr2e, double S,
                    double qsqsum, int num_atoms, int p, const double* charge, const double* mx,
                    const double* my, const double* mz, const double* px, const double* py,
                    const double* pz, double* fx, double* fy, double* fz, double* energy,
                    void* stream) {
  RBX_CHECK_BOX(box);
  if (num_atoms < 0 || p <= 0 || !mx || !my || !mz || !fx || !fy || !fz) {
    set_error("rbx_rbsog_force: need num_atoms >= 0, p > 0 and the arrays");
    return RBX_ERR_INVALID;
  }
  rbx_host::RbsogSetup s;
  RBX_TRY(rbsog_setup_checked(level, cut_off, box, &s));
  if (num_atoms == 0) return RBX_OK;
  RBX_TRY(require_device());
  cudaStream_t st = (cudaStream_t)stream;
  const DBox b = make_dbox(*box);
  const double V = b.len[0] * b.len[1] * b.len[2];
  const double Suse = S > 0 ? S : (S < 0 ? s.S_full : s.S);
  const int nd = (int)s.direct_fb.size(), pt = p + nd;
  std::vector<double4> w(pt);
  std::vector<double> dm(3 * (size_t)nd);
  for (int k = 0; k < p; ++k) w[k] = make_double4(-Suse * qqr2e / p, 0.0, Suse * qqr2e / (2.0 * p * V), 0.0);
  for (int k = 0; k < nd; ++k) {
    w[p + k] = make_double4(0.0, -qqr2e * s.direct_fb[k], 0.0, qqr2e * s.direct_fb[k] / (2.0 * V));
    for (int d = 0; d < 3; ++d) dm[3 * k + d] = s.direct_m[3 * k + d];
  }
  const int nparts = rbe_partial_blocks(num_atoms);
  double *m3 = nullptr, *pre = nullptr, *pim = nullptr, *kterm = nullptr, *en = nullptr;
  double4* wd = nullptr;
  KTab* tab = nullptr;
  int rc = async_alloc(&m3, 3 * (size_t)pt, st);
  if (!rc) rc = async_alloc(&wd, (size_t)pt, st);
  if (!rc) rc = async_alloc(&pre, (size_t)pt * nparts, st);
  if (!rc) rc = async_alloc(&pim, (size_t)pt * nparts, st);
  if (!rc) rc = async_alloc(&tab, (size_t)pt, st);
  if (!rc) rc = async_alloc(&kterm, (size_t)pt, st);
  if (!rc) rc = async_alloc(&en, 1, st);
  if (!rc) {
    double* mxs[3] = {m3, m3 + pt, m3 + 2 * pt};
    const double* src[3] = {mx, my, mz};
    for (int d = 0; d < 3; ++d) {
      cudaMemcpyAsync(mxs[d], src[d], sizeof(double) * p, cudaMemcpyDeviceToDevice, st);
      std::vector<double> col(nd);
      for (int k = 0; k < nd; ++k) col[k] = dm[3 * k + d];
      cudaMemcpyAsync(mxs[d] + p, col.data(), sizeof(double) * nd, cudaMemcpyHostToDevice, st);
      cudaStreamSynchronize(st);  // col is a host temporary
    }
    cudaMemcpyAsync(wd, w.data(), sizeof(double4) * pt, cudaMemcpyHostToDevice, st);
    rc = launch_rbe_rho_partial_f64(b, num_atoms, pt, mxs[0], mxs[1], mxs[2], charge, px, py, pz,
                                    pre, pim, nparts, st);
    if (!rc)
      rc = launch_rbsog_finalize(b, pt, nparts, pre, pim, mxs[0], mxs[1], mxs[2], wd, nullptr,
                                 nullptr, tab, kterm, -s.self_coeff * qsqsum * qqr2e,
                                 energy ? en : nullptr, 0, nullptr, 0, nullptr, st);
    if (!rc) {
      RbeForceOut o;
      o.f_out_x = fx;
      o.f_out_y = fy;
      o.f_out_z = fz;
      rc = launch_rbe_force_f64(num_atoms, pt, tab, charge, px, py, pz, o, st);
    }
    if (!rc && energy) {
      cudaMemcpyAsync(energy, en, sizeof(double), cudaMemcpyDeviceToHost, st);
      rc = cuda_ok(cudaStreamSynchronize(st), "rbx_rbsog_force");
    }
  }
  for (void* ptr : {(void*)m3, (void*)wd, (void*)pre, (void*)pim, (void*)tab, (void*)kterm,
                    (void*)en})
    if (ptr) cudaFreeAsync(ptr, st);
  return rc;
}

static SogGauss sog_gauss_upload(const rbx_host::RbsogSetup& s, double** coef, cudaStream_t st,
                                 int* rc) {
  *rc = async_alloc(coef, 2 * (size_t)s.mmax, st);
  if (*rc) return SogGauss{};
  cudaMemcpyAsync(*coef, s.coef.data(), sizeof(double) * s.mmax, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(*coef + s.mmax, s.coef_npt.data(), sizeof(double) * s.mmax,
                  cudaMemcpyHostToDevice, st);
  return SogGauss{*coef, *coef + s.mmax, s.mmax, s.b * s.b, s.sigma * s.sigma};
}

int rbx_rbsog_npt_chain(const rbx_box* box, int level, double cut_off, int p, const double* mx,
                        const double* my, const double* mz, uint64_t seed, int64_t step,
                        int* idx_npt, void* stream) {
  RBX_CHECK_BOX(box);
  if (p <= 0 || !mx || !my || !mz || !idx_npt) {
    set_error("rbx_rbsog_npt_chain: need p > 0 and the arrays");
    return RBX_ERR_INVALID;
  }
  rbx_host::RbsogSetup s;
  RBX_TRY(rbsog_setup_checked(level, cut_off, box, &s));
  RBX_TRY(require_device());
  cudaStream_t st = (cudaStream_t)stream;
  double* coef = nullptr;
  int* mult = nullptr;
  int rc = 0;
  const SogGauss g = sog_gauss_upload(s, &coef, st, &rc);
  if (!rc) rc = async_alloc(&mult, (size_t)p, st);
  if (!rc)
    rc = launch_rbsog_npt_chain(make_dbox(*box), p, mx, my, mz, g, seed, (uint64_t)step, nullptr,
                                idx_npt, mult, st);
  if (!rc) rc = cuda_ok(cudaStreamSynchronize(st), "rbx_rbsog_npt_chain");
  for (void* ptr : {(void*)coef, (void*)mult})
    if (ptr) cudaFreeAsync(ptr, st);
  return rc;
}

int rbx_rbsog_virial(const rbx_box* box, int level, double cut_off, double qqr2e, double S,
                     double S_npt, int num_atoms, int p, const double* charge, const double* mx,
                     const double* my, const double* mz, const int* idx_npt, const double* px,
                     const double* py, const double* pz, double* virial, void* stream) {
  RBX_CHECK_BOX(box);
  if (num_atoms < 0 || p <= 0 || !mx || !my || !mz || !idx_npt || !virial) {
    set_error("rbx_rbsog_virial: need num_atoms >= 0, p > 0 and the arrays");
    return RBX_ERR_INVALID;
  }
  rbx_host::RbsogSetup s;
  RBX_TRY(rbsog_setup_checked(level, cut_off, box, &s));
  for (int c = 0; c < 6; ++c) virial[c] = 0.0;
  if (num_atoms == 0) return RBX_OK;
  RBX_TRY(require_device());
  cudaStream_t st = (cudaStream_t)stream;
  const DBox b = make_dbox(*box);
  const double V = b.len[0] * b.len[1] * b.len[2];
  const double Suse = S > 0 ? S : (S < 0 ? s.S_full : s.S);
  const double Snpt = S_npt > 0 ? S_npt : s.S_npt;
  const int nd = (int)s.direct_fb.size(), pt = p + nd;
  // multiplicity of each sample in the gather map
  std::vector<int> hidx(p), mult(p, 0);
  int rc = cuda_ok(cudaMemcpyAsync(hidx.data(), idx_npt, sizeof(int) * p, cudaMemcpyDeviceToHost,
                                   st), "D2H");
  if (!rc) rc = cuda_ok(cudaStreamSynchronize(st), "rbx_rbsog_virial");
  if (rc) return rc;
  for (int i = 0; i < p; ++i) {
    if (hidx[i] < 0 || hidx[i] >= p) {
      set_error("rbx_rbsog_virial: idx_npt[%d] = %d outside [0, %d)", i, hidx[i], p);
      return RBX_ERR_INVALID;
    }
    ++mult[hidx[i]];
  }
  std::vector<double4> w(pt);
  std::vector<double> wv(pt), dm(3 * (size_t)nd);
  for (int k = 0; k < p; ++k) {
    w[k] = make_double4(0.0, 0.0, Suse * qqr2e / (2.0 * p * V), 0.0);
    wv[k] = -Snpt * qqr2e / (4.0 * p * V);
  }
  for (int k = 0; k < nd; ++k) {
    w[p + k] = make_double4(0.0, 0.0, 0.0, qqr2e * s.direct_fb[k] / (2.0 * V));
    wv[p + k] = -qqr2e * s.direct_fb_npt[k] / (4.0 * V);
    for (int d = 0; d < 3; ++d) dm[3 * k + d] = s.direct_m[3 * k + d];
  }
  const int nparts = rbe_partial_blocks(num_atoms);
  double *m3 = nullptr, *pre = nullptr, *pim = nullptr, *kterm = nullptr, *vw = nullptr,
         *vout = nullptr;
  double4* wd = nullptr;
  int* dmult = nullptr;
  rc = async_alloc(&m3, 3 * (size_t)pt, st);
  if (!rc) rc = async_alloc(&wd, (size_t)pt, st);
  if (!rc) rc = async_alloc(&pre, (size_t)pt * nparts, st);
  if (!rc) rc = async_alloc(&pim, (size_t)pt * nparts, st);
  if (!rc) rc = async_alloc(&kterm, 7 * (size_t)pt, st);
  if (!rc) rc = async_alloc(&vw, (size_t)pt, st);
  if (!rc) rc = async_alloc(&vout, 6, st);
  if (!rc) rc = async_alloc(&dmult, (size_t)p, st);
  if (!rc) {
    double* mxs[3] = {m3, m3 + pt, m3 + 2 * pt};
    const double* src[3] = {mx, my, mz};
    std::vector<double> cols(3 * (size_t)nd);
    for (int d = 0; d < 3; ++d)
      for (int k = 0; k < nd; ++k) cols[(size_t)d * nd + k] = dm[3 * k + d];
    for (int d = 0; d < 3; ++d) {
      cudaMemcpyAsync(mxs[d], src[d], sizeof(double) * p, cudaMemcpyDeviceToDevice, st);
      cudaMemcpyAsync(mxs[d] + p, cols.data() + (size_t)d * nd, sizeof(double) * nd,
                      cudaMemcpyHostToDevice, st);
    }
    cudaMemcpyAsync(wd, w.data(), sizeof(double4) * pt, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(vw, wv.data(), sizeof(double) * pt, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dmult, mult.data(), sizeof(int) * p, cudaMemcpyHostToDevice, st);
    rc = launch_rbe_rho_partial_f64(b, num_atoms, pt, mxs[0], mxs[1], mxs[2], charge, px, py, pz,
                                    pre, pim, nparts, st);
    const SogVirial sv{p, dmult, vw, kterm + pt, vout};
    if (!rc)
      rc = launch_rbsog_finalize(b, pt, nparts, pre, pim, mxs[0], mxs[1], mxs[2], wd, nullptr,
                                 nullptr, nullptr, kterm, 0.0, nullptr, 0, nullptr, 0, nullptr, st,
                                 &sv);
    if (!rc) {
      cudaMemcpyAsync(virial, vout, sizeof(double) * 6, cudaMemcpyDeviceToHost, st);
      rc = cuda_ok(cudaStreamSynchronize(st), "rbx_rbsog_virial");
    }
  }
  for (void* ptr : {(void*)m3, (void*)wd, (void*)pre, (void*)pim, (void*)kterm, (void*)vw,
                    (void*)vout, (void*)dmult})
    if (ptr) cudaFreeAsync(ptr, st);
  return rc;
}

int rbx_pair_force_verlet_sog(const rbx_box* box, int level, double cut_off, double qqr2e,
                              int num_atoms, int ntypes, const double* sigma, const double* eps,
                              const int* type, const double* charge, const double* px,
                              const double* py, const double* pz, int cap, const int* cand_count,
                              const int* cand, double* fx, double* fy, double* fz,
                              double* energy, double* flat_virial, void* stream) {
  RBX_CHECK_BOX(box);
  if (num_atoms < 0 || ntypes <= 0 || !sigma || !eps || cap < 0) {
    set_error("rbx_pair_force_verlet_sog: invalid arguments");
    return RBX_ERR_INVALID;
  }
  rbx_host::RbsogSetup s;
  RBX_TRY(rbsog_setup_checked(level, cut_off, box, &s));
  if (num_atoms == 0) return RBX_OK;
  RBX_TRY(require_device());
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<double> he((size_t)ntypes * ntypes), hs((size_t)ntypes * ntypes);
  for (int a = 0; a < ntypes; ++a)
    for (int c = 0; c < ntypes; ++c) {
      he[a * ntypes + c] = sqrt(eps[a] * eps[c]);
      hs[a * ntypes + c] = pow((sigma[a] + sigma[c]) / 2, 6.0);
    }
  SogPairParams sp{};
  sp.box = make_dbox(*box);
  sp.cut_off = cut_off;
  sp.qqr2e = qqr2e;
  sp.ntypes = ntypes;
  for (int i = 0; i < 6; ++i) sp.taylor[i] = s.taylor[i];
  sp.sigma = s.sigma;
  sp.b = s.b;
  sp.w0 = s.w0;
  sp.norm = 2.0 * log(s.b) / sqrt(2.0 * RBX_PI * s.sigma * s.sigma);
  sp.mmax = s.mmax;
  double *tabs = nullptr, *epart = nullptr;
  const int nb = verlet_sog_blocks(num_atoms);
  int rc = async_alloc(&tabs, 2 * he.size(), st);
  if (!rc && energy) rc = async_alloc(&epart, 2 * (size_t)nb, st);
  if (!rc) {
    cudaMemcpyAsync(tabs, he.data(), sizeof(double) * he.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(tabs + he.size(), hs.data(), sizeof(double) * hs.size(),
                    cudaMemcpyHostToDevice, st);
    sp.lj_eps = tabs;
    sp.lj_s6 = tabs + he.size();
    rc = launch_verlet_sog(sp, num_atoms, px, py, pz, charge, type, cand_count, cand, cap, fx, fy,
                           fz, epart, st, flat_virial);
  }
  if (!rc) rc = cuda_ok(cudaStreamSynchronize(st), "rbx_pair_force_verlet_sog");
  if (!rc && energy) {
    std::vector<double> h(2 * (size_t)nb);
    rc = cuda_ok(cudaMemcpy(h.data(), epart, sizeof(double) * h.size(), cudaMemcpyDeviceToHost),
                 "D2H");
    energy[0] = energy[1] = 0.0;
    for (int k = 0; k < nb; ++k) {
      energy[0] += h[2 * k];
      energy[1] += h[2 * k + 1];
    }
  }
  for (void* ptr : {(void*)tabs, (void*)epart})
    if (ptr) cudaFreeAsync(ptr, st);
  return rc;
}
