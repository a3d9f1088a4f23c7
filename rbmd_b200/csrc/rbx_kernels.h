// rbx_kernels.h -- host launchers of the sm_100a kernels (internal).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "rbx_common.cuh"

namespace rbx {

// Per-k force table written by the finalize kernel.
struct KTab {
  double kx, ky, kz;
  double a, b;  // coef * Re rho, coef * Im rho, coef = -4 pi qqr2e S / (P V k^2)
  int m[4];     // integer m (mixed form)
};

// Destinations of the RBE force pass.
struct RbeForceOut {
  const double* f_pair_x = nullptr;  // add real-space force (combine), or null
  const double* f_pair_y = nullptr;
  const double* f_pair_z = nullptr;
  const double* mean = nullptr;      // subtract this mean from the pair force
  double* f_out_x = nullptr;
  double* f_out_y = nullptr;
  double* f_out_z = nullptr;
  double* fk_x = nullptr;            // optional copy of the k-space force
  double* fk_y = nullptr;
  double* fk_z = nullptr;
  double* vx = nullptr;              // optional half kick
  double* vy = nullptr;
  double* vz = nullptr;
  const int* type = nullptr;
  const double* inv_mass = nullptr;
  double half_dt = 0.0;
};

// ---- k-space (rbx_rbe.cu) ----
int rbe_partial_blocks(int n);
// The RBE k-sampler's inputs (launch_rbe_sample) for drawing the samples
// inside the structure-factor kernels: tables null = read the samples instead.
struct SampleArgs {
  const double* tables;  // the three cumulative per-axis tables, concatenated
  int c0, c1, c2;
  double t0, t1, t2;
  uint32_t key0, key1;   // the seed
  uint64_t step_arg;
  const int* step_dev;   // device step (inside a step graph), else step_arg
  double *mx, *my, *mz;  // samples out (block column 0)
  int* mi;               // integer copy (may be null)
  int* status;           // raised on a failed draw
};
SampleArgs make_sample_args(const double* tables, const int cnt[3], const double tot[3],
                            uint64_t seed, int64_t step, const int* step_dev, double* mx,
                            double* my, double* mz, int* mi, int* status);
int launch_rbe_rho_partial_f64(const DBox& b, int n, int p, const double* mx, const double* my,
                               const double* mz, const double* q, const double* x,
                               const double* y, const double* z, double* part_re,
                               double* part_im, int nblocks, cudaStream_t st, int kpt = 4,
                               const SampleArgs* sample = nullptr);
int launch_rbe_rho_partial_mixed(int n, int p, const int* mi, const uint4* atoms,
                                 double* part_re, double* part_im, int nblocks, cudaStream_t st,
                                 int kpt = 4, const SampleArgs* sample = nullptr);
int launch_rbe_finalize(const DBox& b, int p, int nparts, const double* part_re,
                        const double* part_im, const double* mx, const double* my,
                        const double* mz, double alpha, double S, double qqr2e, double qsq,
                        double qsum, double* rho_re, double* rho_im, double* energy,
                        double* virial, KTab* tab, int mean_parts, const double* fpart,
                        int n_atoms, double* mean_out, double* kterm, cudaStream_t st,
                        unsigned* sum_ctr = nullptr);
// kterm: scratch of 8 p doubles for the per-k energy/virial terms (parallel
// finalize); when null and energy is requested, one block does the finalize.
int launch_rbe_force_f64(int n, int p, const KTab* tab, const double* q, const double* x,
                         const double* y, const double* z, const RbeForceOut& out,
                         cudaStream_t st, int block = 256);
int launch_rbe_force_mixed(int n, int p, const KTab* tab, const uint4* atoms,
                           const RbeForceOut& out, cudaStream_t st, int block = 256);
// step_dev (may be null): read the step from device memory (step graphs).
int launch_rbe_sample(int p, const double* tables, const int cnt[3], const double tot[3],
                      uint64_t seed, int64_t step, const int* step_dev, double* mx, double* my,
                      double* mz, int* mi, int* status, cudaStream_t st);
int launch_m_to_int(int p, const double* mx, const double* my, const double* mz, int* mi,
                    cudaStream_t st);
int launch_ewald(const DBox& b, int n, const int kmax[3], double alpha, double qqr2e,
                 double qsq, const double* q, const double* x, const double* y, const double* z,
                 double* re, double* im, double* kvec, double* fx, double* fy, double* fz,
                 double* energy, cudaStream_t st);

// Host-side sampler tables (order m = 0, +1, -1, ...), identical to the oracle's.
int rbe_axis_table(double L, double alpha, double* w, int max_entries, double* total);

// Candidate rows of the list builder: row i (idx + i * cap) holds
// c = min(count[i], cap) entries, nf = c - nb in the near segment [0, nf) and
// nb = far[i] (0 when far is null) in the far segment [cap - nb, cap);
// count[i] > cap marks an overflowed build.
struct Rows {
  const int* count = nullptr;
  const int* far = nullptr;
  const int* idx = nullptr;
  int cap = 0;
};

__device__ __forceinline__ void row_extent(const Rows& r, int i, int& nf, int& nb) {
  const int c = min(r.count[i], r.cap);
  nb = r.far ? min(r.far[i], c) : 0;
  nf = c - nb;
}
// Entry k (0 <= k < nf + nb) of a row: the near segment, then the far one.
__device__ __forceinline__ int row_at(const int* row, int cap, int nf, int nb, int k) {
  return __ldg(row + (k < nf ? k : k + (cap - nf - nb)));
}

// ---- real space (rbx_pair.cu) ----
// Screen of "r^2 < C" on the fixed-point |d|^2 (FP32, units of s^2 with
// s = L/2^32, L the longest box edge): decided below lo and at or above hi,
// undecided in between (the FP64 predicate decides).
struct IntScreen {
  float lo, hi;
};
// Build the screen for threshold C (r^2 units) with L the longest box edge.
IntScreen make_screen(double C, double L, double band);

struct PairParams {
  DBox box;
  double rs2, rc2;            // force predicates: r_core^2, cut_off^2
  double core2_list;          // list predicates: r_core^2 - EPS, cut_off^2 - EPS
  double force2_list;
  double alpha, sqrt_alpha, qqr2e;
  int freq;                   // pice_num
  DivTest div;
  int ntypes;
  const double* lj_eps;       // ntypes^2 eps_ij
  const double* lj_s6;        // ntypes^2 sigma_ij^6
  // fixed-point screen: |u_j - u_i|^2 in units of (L_max / 2^32)^2 against
  // FP32 thresholds; on a box with unequal edges each difference is first
  // weighted by L_d / L_max (cubic: no weights)
  int cubic;
  float sw[3];                // L_d / L_max in FP32
  float sf[3];                // L_d / 2^32 in FP32 (mixed pair vector)
  IntScreen sc_eps, sc_core, sc_rs, sc_force, sc_rc;
};


// Fused RBL filter + pair force over a row-major candidate list.
// fpart (nblocks x 3) receives per-block force sums for the mean removal.
int rbl_fused_blocks(int n);
// Grid of the fused RBL kernel for this form: one wave of resident blocks,
// at most max_blocks (the capacity of the per-block partial buffer).
int rbl_fused_grid(bool mixed, int freq, int n, int cap, int max_blocks, int waves = 8,
                   int ntypes = 1);
// Dynamic shared memory of the pair kernels' per-type-pair LJ tables.
size_t type_table_bytes(int ntypes, bool mixed);
// Rows may be split (near / far segments, the far pairs certainly outside
// r_core until the next rebuild) or not (far null: every pair classified).
int launch_rbl_fused(bool mixed, const PairParams& pp, int n, const uint4* atoms,
                     const double* x, const double* y, const double* z, const double* q,
                     const int* type, const unsigned long long* key_a,
                     const unsigned long long* key_b, int epoch, const int* epoch_dev,
                     const Rows& rows, double* fx, double* fy, double* fz, double* fpart,
                     int nblocks, cudaStream_t st);
// Verlet pair force over the candidate list, cut at cut_off (force predicate).
int launch_verlet_fused_f64(const PairParams& pp, int n, const uint4* atoms, const double* x,
                            const double* y, const double* z, const double* q, const int* type,
                            const Rows& rows, double* fx,
                            double* fy, double* fz, double* fpart, double* epart, int nblocks,
                            cudaStream_t st);
// Emit RBL lists (parity checks / export): core and shell rows (cap stride).
int launch_rbl_lists(const PairParams& pp, int n, const uint4* atoms, const double* x,
                     const double* y, const double* z, const unsigned long long* key_a,
                     const unsigned long long* key_b, int epoch, const Rows& rows,
                     int* core_count, int* core, int* shell_count, int* shell,
                     cudaStream_t st);
int launch_rbl_keys(int n, const int* gid, unsigned long long* key_a, unsigned long long* key_b,
                    cudaStream_t st);
// Drop-in ops with the reference layouts.
int launch_ref_rbl_filter(double core2, double force2, int n, const int* gid, const double* x,
                          const double* y, const double* z, const int* cstart, const int* cend,
                          const int* cand, const int* core_cap, const int* core_start,
                          int* core_end, int* core, int shell_cap, int* shell, int* shell_num,
                          int* required, const DBox& b, int* realloc, const DivTest& div,
                          int epoch, cudaStream_t st);
int launch_ref_pair_rbl(const DBox& b, double rs, double rc, int n, int pice_num, double alpha,
                        double qqr2e, const int* type, const double* sigma, const double* eps,
                        const int* start, const int* end, const int* core, const int* shell,
                        const int* shell_num, const double* q, const double* x, const double* y,
                        const double* z, double* fx, double* fy, double* fz, cudaStream_t st);
int launch_ref_pair_verlet(const DBox& b, double cut_off, int n, double alpha, double qqr2e,
                           const int* type, const double* sigma, const double* eps,
                           const int* start, const int* end, const int* nbrs, const double* q,
                           const double* x, const double* y, const double* z, double* fx,
                           double* fy, double* fz, double* flat_virial, double* epart,
                           cudaStream_t st);
// FP32 overloads of the drop-in ops (the reference's default build,
// rbmd::Real = float): membership tests in float as that build evaluates
// them, force values computed in FP64 and stored in float.
int launch_ref_rbl_filter(float core2, float force2, int n, const int* gid, const float* x,
                          const float* y, const float* z, const int* cstart, const int* cend,
                          const int* cand, const int* core_cap, const int* core_start,
                          int* core_end, int* core, int shell_cap, int* shell, int* shell_num,
                          int* required, const DBox& b, int* realloc, const DivTest& div,
                          int epoch, cudaStream_t st);
int launch_ref_pair_rbl(const DBox& b, float rs, float rc, int n, int pice_num, double alpha,
                        double qqr2e, const int* type, const float* sigma, const float* eps,
                        const int* start, const int* end, const int* core, const int* shell,
                        const int* shell_num, const float* q, const float* x, const float* y,
                        const float* z, float* fx, float* fy, float* fz, cudaStream_t st);
int launch_ref_pair_verlet(const DBox& b, float cut_off, int n, double alpha, double qqr2e,
                           const int* type, const float* sigma, const float* eps,
                           const int* start, const int* end, const int* nbrs, const float* q,
                           const float* x, const float* y, const float* z, float* fx,
                           float* fy, float* fz, float* flat_virial, double* epart,
                           cudaStream_t st);
int launch_reduce_cols(int n, int ncols, const float* cols, double* out, double scale,
                       cudaStream_t st);
int launch_sub_mean(int n, float* fx, float* fy, float* fz, const double* mean,
                    cudaStream_t st);
// Element-wise conversions between float and double device arrays.
int launch_widen(int n, const float* src, double* dst, cudaStream_t st);
int launch_narrow(int n, const double* src, float* dst, cudaStream_t st);
int launch_sum_i32(int n, const int* src, long long* out, cudaStream_t st);
int launch_reduce_cols(int n, int ncols, const double* cols, double* out, double scale,
                       cudaStream_t st);
int launch_sub_mean(int n, double* fx, double* fy, double* fz, const double* mean,
                    cudaStream_t st);

// ---- cells, lists, integration (rbx_cells.cu) ----
// Bookkeeping of an engine rebuild folded into its kernels (each member may be
// null): the cell sort's first kernel zeroes flags[0..1] (sort status, list
// overflow) and *total and adds one to *counter; the list builder then adds
// every row's candidate count to *total.
struct RebuildBook {
  int* flags;
  long long* total;
  int* counter;
};
int launch_cells_sort(const DBox& b, const int dims[3], int n, const double* x, const double* y,
                      const double* z, int* perm, int* cell_of_sorted, int* cell_start,
                      void* scratch, int* status, cudaStream_t st,
                      const RebuildBook* book = nullptr);
size_t cells_scratch_bytes(int n, int ncell);
// Scratch of launch_full_list: per-chunk boxes and cells, full_list_scratch_bytes(n, ncell).
size_t full_list_scratch_bytes(int n, int ncell);
// Split of the candidate rows for RBL engines: candidates whose build distance
// is certainly at least r_near go to the far segment at the back of the row,
// far[i] of them (see Rows); the others, and any within the FP32 error of
// r_near, to the near segment.
struct FarSplit {
  double r_near;
  int* far;
};
int launch_full_list(const DBox& b, const int dims[3], double cutoff, int n, const double* x,
                     const double* y, const double* z, const int* cell_start, int cap,
                     int* count, int* nbrs, int* overflow, void* scratch, cudaStream_t st,
                     const FarSplit* split = nullptr, long long* total = nullptr);
// Force adjoint (rbx_adjoint.cu).  Pair part: per-atom dL/dr, dL/dq and
// per-block partials [nblocks][2 ntypes + 1] (d_eps, d_sigma, d_alpha).
int adj_pair_blocks(int n);
int launch_adj_pair(const PairParams& pp, int n, const double* x, const double* y,
                    const double* z, const double* q, const int* type, const double* sigma_t,
                    const double* eps_t, const unsigned long long* key_a,
                    const unsigned long long* key_b, int epoch, const Rows& rows,
                    const double* gx, const double* gy,
                    const double* gz, const double mean_g[3], double* d_rx, double* d_ry,
                    double* d_rz, double* d_q, double* part, int nblocks, cudaStream_t st,
                    bool f32 = false);
// k-space part, added to d_r and d_q; part_gk[adj_k_blocks(n)] = block sums of g . K.
// cscale = -4 pi qqr2e S / (P V); ab: 2p scratch; part_a/b: p * nparts scratch.
int adj_k_blocks(int n);
int launch_adj_kspace(int n, int p, double cscale, const KTab* tab, const double* q,
                      const double* x, const double* y, const double* z, const double* gx,
                      const double* gy, const double* gz, double* part_a, double* part_b,
                      int nparts, double* ab, double* d_rx, double* d_ry, double* d_rz,
                      double* d_q, double* part_gk, cudaStream_t st);
// Mixed form: phases from the fixed-point records, FP32 terms, FP64 sums.
int launch_adj_kspace_mixed(int n, int p, double cscale, const KTab* tab, const uint4* atoms,
                            const double* gx, const double* gy, const double* gz, double* part_a,
                            double* part_b, int nparts, double* ab, double* d_rx, double* d_ry,
                            double* d_rz, double* d_q, double* part_gk, cudaStream_t st);
// [n][3] interleaved host-order rows -> three cell-order arrays (orig[i] = host index).
int launch_gather_vec3(int n, const int* orig, const double* src, double* x, double* y, double* z,
                       cudaStream_t st);

// RBSOG k-space and VERLET-SOG real space (rbx_rbsog.cu).
struct RbsogTables {         // device views of the mixture sampler's tables
  const double* comp_cdf;    // [ncomp = 3 mmax] cumulative component weights
  int ncomp;
  double comp_tot;
  const double* tables;      // concatenated cumulative per-axis tables
  const int* off;            // [mmax][3][2] offsets, counts and totals
  const int* cnt;
  const double* tot;
};
struct SogPairParams {
  DBox box;
  double cut_off, qqr2e;
  int ntypes;
  const double* lj_eps;      // ntypes^2
  const double* lj_s6;
  double taylor[6];          // short-range force polynomial in r^2
  double sigma, b, w0, norm; // energy: norm w_l exp(-r^2 / (2 sigma^2 b^(2l)))
  int mmax;
};
int launch_rbsog_sample(int p, const RbsogTables& t, uint64_t seed, uint64_t step,
                        const int* step_dev, double* mx, double* my, double* mz, int* mi,
                        int* status, cudaStream_t st);
// w[k] = {wa, wb, ea, eb}: c_k = (wa / k^2 + wb) / V, e_k = (ea / k^2 + eb) |rho|^2.
// energy (may be null) needs kterm [p]; E = sum_k e_k + self_energy.
// Virial (optional): vir = {psamp, mult, vw, vterm, out}.  Sample k < psamp
// adds e_k to each diagonal entry plus mult[k] vw[k] |rho_k|^2 / |k|^4 k_a k_b;
// a direct vector k >= psamp adds e_k to the diagonal plus
// vw[k] |rho_k|^2 k_a k_b; the per-k terms vterm [p][6] are summed in k order
// into out[6] (xx, yy, zz, xy, xz, yz).
struct SogVirial {
  int psamp;
  const int* mult;
  const double* vw;
  double* vterm;
  double* out;
};
int launch_rbsog_finalize(const DBox& b, int p, int nparts, const double* part_re,
                          const double* part_im, const double* mx, const double* my,
                          const double* mz, const double4* w, double* rho_re, double* rho_im,
                          KTab* tab, double* kterm, double self_energy, double* energy,
                          int mean_parts, const double* fpart, int n_atoms, double* mean_out,
                          cudaStream_t st, const SogVirial* vir = nullptr);
// The NPT gather chain of RBSOGSampleKSpace over the p samples: one block;
// r_i = G_npt(m_i) |k_i|^4 / (G(m_i) |k_i|^2) and a Philox uniform u_i per
// sample, then idx_0 = 0, idx_i = i when u_i r_(idx_(i-1)) < r_i else
// idx_(i-1).  mult[k] = #{i : idx_i = k}; idx (may be null) the map itself.
struct SogGauss {
  const double* coef;      // [mmax] Gaussian weights
  const double* coef_npt;  // [mmax] their NPT counterparts
  int mmax;
  double b2, sig2;         // b^2, sigma^2
};
int launch_rbsog_npt_chain(const DBox& b, int p, const double* mx, const double* my,
                           const double* mz, const SogGauss& g, uint64_t seed, uint64_t step,
                           const int* step_dev, int* idx, int* mult, cudaStream_t st);
int verlet_sog_blocks(int n);
// epart (may be null) receives [blocks][2] = {E_LJ, E_coul} per-block sums.
// Mixed form: fixed-point records, FP32 pair terms, no energies.
int launch_verlet_sog_mixed(const SogPairParams& sp, const float sf[3], int n, const uint4* atoms,
                            const int* type, const int* cand_count, const int* cand, int cap,
                            double* fx, double* fy, double* fz, cudaStream_t st);
// flat_virial (may be null): per-atom virial [6][n] (xx, yy, zz, xy, xz, yz).
int launch_verlet_sog(const SogPairParams& sp, int n, const double* x, const double* y,
                      const double* z, const double* q, const int* type, const int* cand_count,
                      const int* cand, int cap, double* fx, double* fy, double* fz, double* epart,
                      cudaStream_t st, double* flat_virial = nullptr);

// Nose-Hoover chain (rbx_thermo.cu): parameters and the device state layout.
constexpr int NH_CHAIN = 3;
enum NHSlot {
  NH_ETA = 0,                            // [NH_CHAIN]
  NH_ETA_DOT = NH_ETA + NH_CHAIN,        // [NH_CHAIN + 1], last entry 0
  NH_ETA_DOTDOT = NH_ETA_DOT + NH_CHAIN + 1,
  NH_ETA_MASS = NH_ETA_DOTDOT + NH_CHAIN,
  NH_TEMP = NH_ETA_MASS + NH_CHAIN,      // current temperature
  NH_T_TARGET, NH_KE_TARGET, NH_FACTOR,  // target, tdof kB T_target, last scale
  NH_SLOTS
};
struct NHParams {
  double t_start, t_stop, t_freq, dt, kb, mvv2e, tdof;
  long long num_steps;
};
constexpr int KE_PARTS = 296;  // fixed reduction grid (2 x 148 SMs)
int launch_ke_partials(int n, const int* type, const double* mass, const double* vx,
                       const double* vy, const double* vz, double mvv2e, double* part,
                       cudaStream_t st);
int launch_nh_chain(const NHParams& p, double* state, const double* part, const int* step_dev,
                    long long step_add, int mode, cudaStream_t st);
int launch_scale_v(int n, const double* state, double* vx, double* vy, double* vz,
                   cudaStream_t st);

// A set of per-atom arrays moved together: dst[a][i] = src[a][perm[i]].
struct ArraySet {
  static constexpr int kMaxF64 = 16, kMaxI32 = 8, kMaxU64 = 2;
  const double* src_f64[kMaxF64];
  double* dst_f64[kMaxF64];
  const int* src_i32[kMaxI32];
  int* dst_i32[kMaxI32];
  const unsigned long long* src_u64[kMaxU64];
  unsigned long long* dst_u64[kMaxU64];
  int nf64, ni32, nu64;
};
// perm may be null (plain copy).
int launch_move_set(int n, const int* perm, const ArraySet& set, cudaStream_t st);
// dst[a][idx[i]] = src[a][i] (host order <- cell order).
int launch_scatter_set(int n, const int* idx, const ArraySet& set, cudaStream_t st);
int launch_fill_i32(int n, int* p, int v, cudaStream_t st);
int launch_zero_u64(unsigned long long* p, cudaStream_t st);
int launch_add_i32(int* p, int v, cudaStream_t st);
// Step-graph decision: ++*epoch; rebuild branch iff max displacement^2 > thr2.
int launch_step_decide(const unsigned long long* max_d2, double thr2, int* epoch,
                       cudaGraphConditionalHandle rebuild, cudaStream_t st);
int launch_gather_f64(int n, const int* perm, const double* src, double* dst, cudaStream_t st);
int launch_gather_i32(int n, const int* perm, const int* src, int* dst, cudaStream_t st);
int launch_gather_u64(int n, const int* perm, const unsigned long long* src,
                      unsigned long long* dst, cudaStream_t st);
int launch_scatter_f64(int n, const int* idx, const double* src, double* dst, cudaStream_t st);
int launch_scatter_i32(int n, const int* idx, const int* src, int* dst, cudaStream_t st);
int launch_kick(int n, const double* fx, const double* fy, const double* fz, const int* type,
                const double* inv_mass, double half_dt, double* vx, double* vy, double* vz,
                cudaStream_t st);
// Drift + periodic wrap + max displacement since the last build (+ fixed point).
// Per-atom periodic image counters (may be null: not tracked).
// Three coordinate arrays (any may be null as a whole: x == nullptr).
struct Pos3 {
  double* x;
  double* y;
  double* z;
};
struct ImageRefs {
  int* c[3];
};
// kick (may be null): the step's first half kick v += F inv_mass[type] half_dt
// done in the same pass, before the drift.
struct KickArgs {
  const double *fx, *fy, *fz;
  const int* type;
  const double* inv_mass;
  double half_dt;
};
// decide (may be null; inside a step graph only): the step's rebuild decision
// taken by the drift's last block (k_step_decide's test on max_d2 > thr2,
// epoch += 1), which then clears max_d2 and ctr (zero before the first step).
struct DecideArgs {
  unsigned* ctr;
  double thr2;
  int* epoch;
  cudaGraphConditionalHandle cond;
};
int launch_drift(const DBox& b, int n, double dt, double* x, double* y, double* z,
                 double* vx, double* vy, double* vz, const double* x0,
                 const double* y0, const double* z0, unsigned long long* max_d2_bits,
                 uint4* atoms, const double* q, ImageRefs img, Pos3 old, cudaStream_t st,
                 const KickArgs* kick = nullptr, const DecideArgs* decide = nullptr);
// CVFF special-bond correction of the RBL pair force (rbx_special.cu): its
// SPEC_PARTS per-block force sums follow the fused kernel's in fpart.
constexpr int SPEC_PARTS = 1184;  // 8 blocks per SM of 148: about one atom per thread
int launch_special_rbl(const PairParams& pp, int natoms, const int* atoms_h, const int* cnt,
                       const int* part, int maxs, double w12, double w13, double w14,
                       const int* where, const double* x, const double* y, const double* z,
                       const double* q, const int* type, const unsigned long long* key_a,
                       const unsigned long long* key_b, int epoch, const int* epoch_dev,
                       double* fx, double* fy, double* fz, double* fpart, cudaStream_t st);
// SHAKE / RATTLE of rigid three-atom clusters (rbx_shake.cu).
struct ShakeParams {
  double dt, b1sq, b2sq, b12sq, tol;
  int max_iter;
};
int launch_inverse_perm(int n, const int* orig, int* where, cudaStream_t st);
int launch_shake_a(const DBox& b, const ShakeParams& sp, int nc, const int* cl, const int* where,
                   const int* type, const double* mass, Pos3 old, Pos3 pos, Pos3 vel,
                   ImageRefs img, const double* x0, const double* y0, const double* z0,
                   unsigned long long* max_d2, uint4* atoms, const double* q, int* status,
                   cudaStream_t st);
int launch_shake_b(const DBox& b, int nc, const int* cl, const int* where, const int* type,
                   const double* mass, Pos3 pos, Pos3 vel, int* status, cudaStream_t st);
int launch_to_fixed(const DBox& b, int n, const double* x, const double* y, const double* z,
                    const double* q, uint4* atoms, cudaStream_t st);
int launch_max_disp(const DBox& b, int n, const double* x, const double* y, const double* z,
                    const double* x0, const double* y0, const double* z0,
                    unsigned long long* max_d2_bits, cudaStream_t st);

// ---- phase-batched replicas (rbx_batch.cu) ----
// While a recorder is installed on the calling thread, the launchers of the
// step kernels that have a batched form -- drift, fused RBL, mixed structure
// factor, finalize, mixed RBE force -- append their argument block to it
// instead of launching.  A batch then launches each phase once over the
// blocks of every replica: block b belongs to replica r when start[r] <= b <
// start[r + 1], and runs as block b - start[r] of that replica's own grid.
enum PhaseKind { PH_DRIFT = 0, PH_RBL = 1, PH_RHO = 2, PH_FINALIZE = 3, PH_FORCE = 4 };
struct PhaseRecord {
  int kind = 0;
  int variant = 0;  // template instance of the kernel
  int blocks = 0;   // the replica's grid
  int threads = 0;
  size_t smem = 0;
  std::vector<unsigned char> args;
};
struct BatchRecorder {
  std::vector<PhaseRecord> recs;
};
BatchRecorder*& batch_recorder();  // the calling thread's recorder (null: launch)
int record_phase(int kind, int variant, int blocks, int threads, size_t smem, const void* args,
                 size_t bytes);
// One launch of phase `kind` over nrep replicas: args holds their argument
// blocks back to back, start[0..nrep] their first blocks (device arrays).
int launch_phase_batch(int kind, int variant, const void* args, const int* start, int nrep,
                       int total, int threads, size_t smem, cudaStream_t st);
int launch_drift_batch(const void* args, const int* start, int nrep, int total, cudaStream_t st);
int launch_rbl_batch(int variant, const void* args, const int* start, int nrep, int total,
                     size_t smem, cudaStream_t st);
int launch_rho_mixed_batch(int variant, const void* args, const int* start, int nrep, int total,
                           cudaStream_t st);
int launch_finalize_batch(const void* args, const int* start, int nrep, int total,
                          cudaStream_t st);
int launch_force_mixed_batch(int variant, const void* args, const int* start, int nrep,
                             int total, cudaStream_t st);

#ifdef __CUDACC__
// Replica of block b (binary search over start[0..nrep), start[0] = 0).
__device__ __forceinline__ int batch_replica(const int* __restrict__ start, int nrep, int b) {
  int lo = 0, hi = nrep - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(start + mid) <= b)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}
#endif

}  // namespace rbx
