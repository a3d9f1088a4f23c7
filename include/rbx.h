/*
 * rbx.h -- C ABI of the B200-native (sm_100a) RBE + LJ/erfc-Coulomb force
 * engine, a drop-in for RBMD 2.0's src/force (LJ/CUT/COUL/LONG + RBE k-space)
 * and src/neighbor_list (linked cells, full Verlet list, RBL core/shell lists).
 *
 * Conventions
 *  - Every function returns an rbx_status (0 = RBX_OK); rbx_last_error() gives
 *    the message of the last failure on the calling thread.  No C++ exception
 *    crosses this boundary.
 *  - Op-level functions take caller-owned DEVICE pointers (FP64 SoA, or FP32
 *    for the *_f32 twins of the float build; int32
 *    ids, the reference's rbmd::Real / rbmd::Id layout) and a cudaStream_t
 *    passed as void*; they enqueue work and return without synchronising
 *    unless stated.  Argument order follows the reference functor each one
 *    replaces (file:line given per entry, relative to the RBMD source tree).
 *  - Engine-level functions (rbx_engine_*) own their device memory and run
 *    the whole force evaluation / velocity-Verlet step on one GPU.
 *  - The library has no CPU fallback: without a usable sm_100 device every
 *    compute entry fails with RBX_ERR_DEVICE.
 */
#ifndef RBX_H
#define RBX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RBX_VERSION 1

typedef enum {
  RBX_OK = 0,
  RBX_ERR_INVALID = 1,   /* bad argument or configuration */
  RBX_ERR_CUDA = 2,      /* CUDA runtime / launch error */
  RBX_ERR_CAPACITY = 3,  /* a device list overflowed its capacity */
  RBX_ERR_NOMEM = 4,     /* device or host allocation failed */
  RBX_ERR_DEVICE = 5,    /* no usable sm_100 device */
  RBX_ERR_CONFIG = 6,    /* JSON key missing / unsupported value */
  RBX_ERR_SAMPLER = 7    /* k-sampler could not draw a non-zero vector */
} rbx_status;

/* Orthogonal periodic box: Box::_coord_min/_coord_max
 * (src/data_manager/include/model/box.h:5-49). */
typedef struct {
  double lo[3];
  double hi[3];
} rbx_box;

const char* rbx_last_error(void);
int rbx_version(void);
/* Number of kernel launches this thread issued through the library so far. */
uint64_t rbx_launch_count(void);

/* ------------------------------------------------------------------------ */
/* Host-side helpers                                                         */
/* ------------------------------------------------------------------------ */

/* S = prod_d H_d - 1.  Replaces ComputeRbeGaussianSum
 * (src/force/src/kspace_calculator.cpp:68-78). */
int rbx_rbe_gauss_sum(const rbx_box* box, double alpha, double* S);

/* RBL selection frequency ("pice_num").  Replaces
 * RblFullNeighborListBuilder::GetRblParams
 * (src/neighbor_list/src/neighbor_list_builder/rbl_full_neighbor_list_builder.cpp:193-228). */
int rbx_rbl_params(int n_global, const rbx_box* box, double r_core,
                   double cut_off, int neighbor_sample_num, int* freq);

/* ------------------------------------------------------------------------ */
/* k-space ops (device pointers)                                             */
/* ------------------------------------------------------------------------ */

/* Counter-based (Philox4x32-10) draw of P integer k-vectors m != 0 from the
 * RBE importance density P(m) ~ exp(-(2 pi m/L)^2/(4 alpha)); writes
 * m_x/m_y/m_z as doubles.  Replaces the host Metropolis-Hastings sampler
 * RBEPSAMPLE::Fetch_P_Sample (src/common/RBEPSample.h:150-188) called from
 * KSpaceCalculator::RBEInit (src/force/src/kspace_calculator.cpp:671-715). */
int rbx_rbe_sample(const rbx_box* box, double alpha, int p, uint64_t seed,
                   int64_t step, double* p_sample_x, double* p_sample_y,
                   double* p_sample_z, void* stream);

/* Re/Im rho(k_p) = sum_j q_j {cos,sin}(k_p . r_j).  Replaces
 * ComputePnumberChargeStructureFactorOp (kspace_calculator_op.h:106-121,
 * kernel kspace_calculator_op.hip.cu:238-289). Deterministic FP64 reduction. */
int rbx_rbe_structure_factor(const rbx_box* box, int num_atoms, int p_number,
                             const double* charge, const double* p_sample_x,
                             const double* p_sample_y, const double* p_sample_z,
                             const double* px, const double* py,
                             const double* pz, double* density_real,
                             double* density_imag, void* stream);

/* rbx_rbe_structure_factor without any device allocation.  No counterpart in
 * the reference: it exists for hosts that own all device memory themselves (a
 * pre-sized arena, a job-enforced memory cap, or a step loop whose footprint
 * must not change) and so cannot let a library call cudaMalloc or
 * cudaMallocAsync.  The per-block partial sums live in a fixed array built into
 * the library: RBX_NOALLOC_RHO_BLOCKS x RBX_NOALLOC_RHO_MAX_P doubles for Re and
 * for Im (2 MiB), held on every GPU that loads the library until the process
 * exits.  p_number above RBX_NOALLOC_RHO_MAX_P is rejected with RBX_ERR_INVALID.
 * Each call outside a stream capture looks up the array's device address on
 * the current device (no allocation), so a device reset is picked up by the
 * next such call; a call inside a capture reuses the address of the last call
 * outside one, so make one call on the device before any stream capture (and
 * again after a device reset).  All calls share the
 * one array: calls whose work can overlap on the GPU (other streams, other
 * host threads) race and must be serialised by the caller.  Results equal
 * rbx_rbe_structure_factor's up to FP64 summation order. */
#define RBX_NOALLOC_RHO_BLOCKS 256
#define RBX_NOALLOC_RHO_MAX_P 512
int rbx_rbe_structure_factor_noalloc(const rbx_box* box, int num_atoms, int p_number,
                                     const double* charge, const double* p_sample_x,
                                     const double* p_sample_y, const double* p_sample_z,
                                     const double* px, const double* py,
                                     const double* pz, double* density_real,
                                     double* density_imag, void* stream);

/* Per-atom RBE force.  Replaces ComputeRBEForceOp (kspace_calculator_op.h:123-135,
 * kernel kspace_calculator_op.hip.cu:678-738). */
int rbx_rbe_force(const rbx_box* box, int num_atoms, int p_number, double alpha,
                  double rbe_sum_gauss, double qqr2e, const double* real_array,
                  const double* imag_array, const double* charge,
                  const double* p_sample_x, const double* p_sample_y,
                  const double* p_sample_z, const double* px, const double* py,
                  const double* pz, double* fx, double* fy, double* fz,
                  void* stream);

/* RBE energy and 6-component virial (xx,yy,zz,xy,xz,yz), written to device
 * memory.  Replaces ComputeRBEForceVirialOp (kernel ComputeRBEVirial0,
 * kspace_calculator_op.hip.cu:573-674); deterministic order. */
int rbx_rbe_energy_virial(const rbx_box* box, int p, double alpha,
                          double rbe_sum_gauss, double qqrd2e, double qsqsum,
                          double qsum, const double* real_array,
                          const double* imag_array, const double* p_sample_x,
                          const double* p_sample_y, const double* p_sample_z,
                          double* virial_tensor, double* energy, void* stream);

/* Exact Ewald reciprocal force over the kmax box (+ per-atom virial).
 * Replaces ComputeEwaldForceOp / ComputeKspaceChargeStructureFactorOp
 * (kspace_calculator_op.hip.cu:176-213, 334-403). rho must hold num_k values;
 * num_k = (2kx+1)(2ky+1)(2kz+1)-1. energy (device, may be NULL) receives the
 * reciprocal + self energy of kspace_calculator.cpp:816-907. */
int rbx_ewald_force(const rbx_box* box, int num_atoms, const int kmax[3],
                    double alpha, double qqr2e, const double* charge,
                    const double* px, const double* py, const double* pz,
                    double* fx, double* fy, double* fz, double* energy,
                    void* stream);

/* RBSOG (random-batch sum of Gaussians) k-space, coulomb.type "RBSOG"
 * (KSpaceCalculator::Init RBSOG branch, kspace_calculator.cpp:253-330;
 * RBSOGInit / RBSOGSetup :988-1140; ComputeRBSOG :1331-1543).
 * Parameters of hyper_parameters.coulomb.rbsog_level (0..4) at this cut_off
 * and box: Gaussian base b, width sigma = sigma_at_rc10 cut_off / 10, count
 * mmax, w0, the sampling normalisation S (and S_npt) as RBSOGSetup computes
 * them, the self-energy coefficient (E_self = -self_coeff sum q^2 qqr2e) and
 * the VERLET-SOG Taylor coefficients (LJCoulSOGInit,
 * lj_cut_coul_kspace.cpp:651-711).  Host only. */
typedef struct {
  int level, mmax;
  double b, sigma, w0, S, S_npt, self_coeff;
  double taylor[6];
  int n_direct;             /* |m|^2 <= 1 vectors summed directly (6) */
  double S_full;            /* the sampled density's full normalisation,
                               sum of G^(m)|k|^2 over |m|^2 > 1.  RBSOGSetup's S
                               keeps only the l = 0 Gaussian's high-k sum (its
                               loop's stop value is not reset between
                               Gaussians), so S / S_full < 1 (0.44 - 0.89 by
                               level) scales the reference's sampled far field */
} rbx_rbsog_info;
/* coef [mmax], direct_m [n_direct][3], direct_fb [n_direct] may be NULL. */
int rbx_rbsog_params(int level, double cut_off, const rbx_box* box, rbx_rbsog_info* out,
                     double* coef, int* direct_m, double* direct_fb);
/* p integer k-samples (device arrays, values integral) from p(m) ~ G^(m)|k|^2
 * on |m|^2 > 1, the density RBSOGSampleKSpace's Metropolis chain targets
 * (kspace_calculator.cpp:1142-1240), drawn exactly and independently on the
 * device (Philox4x32-10, counter = sample, attempt, step; key = seed). */
int rbx_rbsog_sample(const rbx_box* box, int level, double cut_off, int p, uint64_t seed,
                     int64_t step, double* mx, double* my, double* mz, void* stream);
/* RBSOG k-space force of the p samples plus the six |m| = 1 vectors
 * (ComputeRBSOGSampleForceOp + ComputeRBSOGDirectForceOp + their energies
 * and the self energy, kspace_calculator.cpp:1380-1535, NVT/NVE factors
 * fac = 1).  S = 0 uses RBSOGSetup's S (the reference's forces), S < 0
 * the full normalisation S_full (an unbiased far field), S > 0 that value;
 * qsqsum = sum q^2.  Device arrays;
 * energy (host, may be NULL).  The virial is rbx_rbsog_virial. */
int rbx_rbsog_force(const rbx_box* box, int level, double cut_off, double qqr2e, double S,
                    double qsqsum, int num_atoms, int p, const double* charge, const double* mx,
                    const double* my, const double* mz, const double* px, const double* py,
                    const double* pz, double* fx, double* fy, double* fz, double* energy,
                    void* stream);
/* The NPT gather map of the p samples (the virial's chain in
 * RBSOGSampleKSpace, kspace_calculator.cpp:1242-1301): an independence
 * Metropolis chain over the samples with target Gaussian_modify(m) |k|^4 and
 * proposal Gaussian(m) |k|^2; idx_npt[0] = 0, idx_npt[i] = i when accepted,
 * else idx_npt[i - 1].  The uniforms are Philox4x32-10 draws of counter
 * {i, 0x4e505400, step} under key seed (the sampler's key).  Device arrays. */
int rbx_rbsog_npt_chain(const rbx_box* box, int level, double cut_off, int p, const double* mx,
                        const double* my, const double* mz, uint64_t seed, int64_t step,
                        int* idx_npt, void* stream);
/* RBSOG k-space virial[6] (host; xx, yy, zz, xy, xz, yz) of the p samples with
 * their gather map idx_npt (device) plus the six |m| = 1 vectors, at a fixed
 * box (fac = fac_npt = 1): ComputeRBSOGSampleVirialKernel +
 * ComputeRBSOGDirectVirialKernel (kspace_calculator_op.hip.cu:1133-1190,
 * 1308-1355).  S as rbx_rbsog_force; S_npt <= 0 uses RBSOGSetup's S_npt. */
int rbx_rbsog_virial(const rbx_box* box, int level, double cut_off, double qqr2e, double S,
                     double S_npt, int num_atoms, int p, const double* charge, const double* mx,
                     const double* my, const double* mz, const int* idx_npt, const double* px,
                     const double* py, const double* pz, double* virial, void* stream);
/* VERLET-SOG pair force over a full candidate list (LJCutCoulForceUserOp:
 * ComputeLJCutCoulForceUserKernel with lj126 and CoulCutForceUser,
 * lj_cut_coul_kspace_op.hip.cu:196-254, 357-470): LJ 12-6 plus the
 * short-range SOG Coulomb inside cut_off.  sigma / eps per type (host);
 * energy (host, may be NULL) receives {E_LJ, E_coul}, half-counted;
 * flat_virial (device, may be NULL) the per-atom virial flat_virial[c*n + i]
 * (xx, yy, zz, xy, xz, yz) of ComputeVirial (lj_op.hip.cu:76-88). */
int rbx_pair_force_verlet_sog(const rbx_box* box, int level, double cut_off, double qqr2e,
                              int num_atoms, int ntypes, const double* sigma, const double* eps,
                              const int* type, const double* charge, const double* px,
                              const double* py, const double* pz, int cap, const int* cand_count,
                              const int* cand, double* fx, double* fy, double* fz,
                              double* energy, double* flat_virial, void* stream);

/* ------------------------------------------------------------------------ */
/* Neighbor-list ops (device pointers)                                       */
/* ------------------------------------------------------------------------ */

/* Cell grid of edge >= neighbor_cutoff: dims[d] = floor(L_d / neighbor_cutoff).
 * Returns RBX_ERR_INVALID if a dimension has fewer than 3 cells. */
int rbx_cell_grid(const rbx_box* box, double neighbor_cutoff, int dims[3]);

/* Bin atoms into cells, stable-sort by cell and give cell ranges.  Replaces
 * LinkedCell::AssignAtomsToCell + SortAtomsByCellKey + ComputeCellRangesIndices
 * (src/neighbor_list/src/linked_cell/linked_cell.cpp:428-670,
 * src/neighbor_list/src/op/rocm/linked_cell_op.hip.cu:57-164).
 * perm[new] = old index (caller gathers its arrays); cell_start has
 * ncell + 1 entries.  scratch needs rbx_cells_scratch_bytes(n, ncell) bytes. */
size_t rbx_cells_scratch_bytes(int n, int ncell);
int rbx_cells_sort(const rbx_box* box, double neighbor_cutoff, int n,
                   const double* px, const double* py, const double* pz,
                   int* perm, int* cell_of_sorted, int* cell_start,
                   void* scratch, void* stream);

/* Skin test of a cached list: *reuse = 1 when every atom moved at most
 * skin / 2 (minimum image) since the positions cached at the last build,
 * else 0; *max_disp_sq (may be null) receives the largest squared
 * displacement.  The displacement test of
 * BaseNeighborListBuilder::ShouldReuseNeighborList
 * (base_neighbor_list_builder.cpp:219-319); the cache-validity bookkeeping
 * (atom count, order, box) stays with the caller.  Synchronises the stream. */
int rbx_nlist_should_reuse(const rbx_box* box, int n, const double* px, const double* py,
                           const double* pz, const double* cached_px, const double* cached_py,
                           const double* cached_pz, double skin, int* reuse,
                           double* max_disp_sq, void* stream);

/* Full (i->j and j->i) list of sorted atoms within neighbor_cutoff, j != i,
 * row-major with a fixed row capacity: nbrs[i*cap + t], count[i] = true count.
 * *overflow (device int) is set to 1 when some count exceeds cap.  Replaces
 * Estimate/GenerateFullNeighborListOp (full_neighbor_list_op.hip.cu:177-288)
 * for cells of edge >= neighbor_cutoff. */
int rbx_full_list(const rbx_box* box, double neighbor_cutoff, int n,
                  const double* px, const double* py, const double* pz,
                  const int* cell_start, int cap, int* count, int* nbrs,
                  int* overflow, void* stream);

/* Split candidates into the RBL core list (r^2 < core_cutoff_2) and the hashed
 * shell sample (r^2 < force_cutoff_2, SplitMix64 pair hash % freq == 0).
 * Same arguments as FilterRblNeighborCandidatesOp
 * (src/neighbor_list/src/op/rocm/rbl_full_neighbor_list_op.hip.cu:237-334):
 * candidate CSR [start,end), core rows at core_start[i] with capacity
 * max_core_neighbor_num[i], shell sample-major random_neighbors[s*n + i]. */
int rbx_rbl_filter(double core_cutoff_2, double force_cutoff_2, int total_atom_num,
                   const int* atoms_id, const double* px, const double* py,
                   const double* pz, const int* candidate_start,
                   const int* candidate_end, const int* candidate_neighbors,
                   const int* max_core_neighbor_num, const int* core_start,
                   int* core_end, int* core_neighbors,
                   int random_neighbor_capacity, int* random_neighbors,
                   int* random_neighbors_num,
                   int* required_random_neighbor_capacity, const rbx_box* box,
                   int* should_realloc, int selection_frequency,
                   int sample_epoch, void* stream);

/* ------------------------------------------------------------------------ */
/* Pair-force ops (device pointers)                                          */
/* ------------------------------------------------------------------------ */

/* RBL real-space force: core CSR [start_id, end_id) + sample-major shell list.
 * Same arguments as LJCutCoulRBLForceOp (lj_cut_coul_kspace_op.h:155-181,
 * kernel lj_cut_coul_kspace_op.hip.cu:569-683). */
int rbx_pair_force_rbl(const rbx_box* box, double rs, double rc, int num_atoms,
                       int neighbor_sample_num, int pice_num, double alpha,
                       double qqr2e, const int* atoms_type, const double* sigma,
                       const double* eps, const int* start_id, const int* end_id,
                       const int* id_verletlist, const int* id_random_neighbor,
                       const int* random_neighbor_num, const double* charge,
                       const double* px, const double* py, const double* pz,
                       double* fx, double* fy, double* fz, void* stream);

/* Subtract the mean force over all atoms, computed on the device (FP64,
 * deterministic).  Replaces the three thrust::reduce host round trips +
 * FixRBLForceOp (lj_cut_coul_kspace.cpp:537-563, force_op.hip.cu:9-45).
 * mean_out (device, 3 doubles) may be NULL. */
int rbx_fix_rbl_force(int num_atoms, double* fx, double* fy, double* fz,
                      double* mean_out, void* stream);

/* Verlet real-space force + per-atom virial flat_virial[c*n + i] + energies.
 * Same arguments as LJCutCoulForceOp (lj_cut_coul_kspace_op.h:117-140, kernel
 * lj_cut_coul_kspace_op.hip.cu:256-356); total_evdwl / total_ecoul (device)
 * are overwritten with deterministic sums (the reference accumulates). */
int rbx_pair_force_verlet(const rbx_box* box, double cut_off, int num_atoms,
                          double alpha, double qqr2e, const int* atoms_type,
                          const double* sigma, const double* eps,
                          const int* start_id, const int* end_id,
                          const int* id_verletlist, const double* charge,
                          const double* px, const double* py, const double* pz,
                          double* fx, double* fy, double* fz,
                          double* flat_virial, double* total_evdwl,
                          double* total_ecoul, void* stream);

/* ------------------------------------------------------------------------ */
/* FP32 twins for the reference's default build: rbmd::Real is float unless  */
/* ENABLE_DOUBLE (cmake/option.cmake:1, src/common/types.h:4-8).  Argument   */
/* order and meaning as the FP64 entries above and the functors they cite;   */
/* every Real buffer and scalar is float, ids stay int (rbmd::Id without      */
/* ENABLE_64BIT_IDS).  Membership tests (list predicates, force windows) are */
/* evaluated in float as the float build evaluates them, so lists and kept   */
/* pairs are that build's; values are computed in FP64 (real space, energy)  */
/* or in the mixed form (structure factor and RBE force: exact integer phase */
/* on fixed-point coordinates, FP32 sincos, FP64 reductions) and stored in   */
/* float.                                                                    */
/* ------------------------------------------------------------------------ */

/* ComputePnumberChargeStructureFactorOp, float build (kspace_calculator_op.h:106-121). */
int rbx_rbe_structure_factor_f32(const rbx_box* box, int num_atoms, int p_number,
                                 const float* charge, const float* p_sample_x,
                                 const float* p_sample_y, const float* p_sample_z,
                                 const float* px, const float* py, const float* pz,
                                 float* density_real, float* density_imag, void* stream);

/* ComputeRBEForceOp, float build (kspace_calculator_op.h:123-135). */
int rbx_rbe_force_f32(const rbx_box* box, int num_atoms, int p_number, float alpha,
                      float rbe_sum_gauss, float qqr2e, const float* real_array,
                      const float* imag_array, const float* charge, const float* p_sample_x,
                      const float* p_sample_y, const float* p_sample_z, const float* px,
                      const float* py, const float* pz, float* fx, float* fy, float* fz,
                      void* stream);

/* ComputeRBEForceVirialOp, float build (kspace_calculator_op.hip.cu:573-674). */
int rbx_rbe_energy_virial_f32(const rbx_box* box, int p, float alpha, float rbe_sum_gauss,
                              float qqrd2e, float qsqsum, float qsum, const float* real_array,
                              const float* imag_array, const float* p_sample_x,
                              const float* p_sample_y, const float* p_sample_z,
                              float* virial_tensor, float* energy, void* stream);

/* FilterRblNeighborCandidatesOp, float build
 * (rbl_full_neighbor_list_op.hip.cu:237-334): CaculateDistance in float
 * (POW = powf), thresholds r_core^2 - EPSILON and cut_off^2 - EPSILON as the
 * float build forms them. */
int rbx_rbl_filter_f32(float core_cutoff_2, float force_cutoff_2, int total_atom_num,
                       const int* atoms_id, const float* px, const float* py, const float* pz,
                       const int* candidate_start, const int* candidate_end,
                       const int* candidate_neighbors, const int* max_core_neighbor_num,
                       const int* core_start, int* core_end, int* core_neighbors,
                       int random_neighbor_capacity, int* random_neighbors,
                       int* random_neighbors_num, int* required_random_neighbor_capacity,
                       const rbx_box* box, int* should_realloc, int selection_frequency,
                       int sample_epoch, void* stream);

/* LJCutCoulRBLForceOp, float build (lj_cut_coul_kspace_op.hip.cu:569-683). */
int rbx_pair_force_rbl_f32(const rbx_box* box, float rs, float rc, int num_atoms,
                           int neighbor_sample_num, int pice_num, float alpha, float qqr2e,
                           const int* atoms_type, const float* sigma, const float* eps,
                           const int* start_id, const int* end_id, const int* id_verletlist,
                           const int* id_random_neighbor, const int* random_neighbor_num,
                           const float* charge, const float* px, const float* py,
                           const float* pz, float* fx, float* fy, float* fz, void* stream);

/* Mean-force removal, float build (lj_cut_coul_kspace.cpp:537-563,
 * force_op.hip.cu:9-45): the mean is summed in FP64; mean_out (device, 3
 * floats) may be NULL. */
int rbx_fix_rbl_force_f32(int num_atoms, float* fx, float* fy, float* fz, float* mean_out,
                          void* stream);

/* LJCutCoulForceOp, float build (lj_cut_coul_kspace_op.hip.cu:256-356):
 * flat_virial[c*n + i] in float; total_evdwl / total_ecoul (device floats,
 * may be NULL) are overwritten with FP64 sums. */
int rbx_pair_force_verlet_f32(const rbx_box* box, float cut_off, int num_atoms, float alpha,
                              float qqr2e, const int* atoms_type, const float* sigma,
                              const float* eps, const int* start_id, const int* end_id,
                              const int* id_verletlist, const float* charge, const float* px,
                              const float* py, const float* pz, float* fx, float* fy, float* fz,
                              float* flat_virial, float* total_evdwl, float* total_ecoul,
                              void* stream);

/* ------------------------------------------------------------------------ */
/* Engine: LJCutCoulKspace (src/force/src/lj_cut_coul_kspace.cpp) with its   */
/* KSpaceCalculator and neighbor builders, plus the NVE velocity-Verlet step */
/* (NVEensemble::Solve, src/simulate_pipeline/src/nve_ensemble.cpp:59-91).   */
/* ------------------------------------------------------------------------ */

typedef struct rbx_engine rbx_engine;

/* Largest number of atom types an engine takes: the per-type-pair LJ tables
 * (2 x ntypes^2 doubles, and floats in the mixed form) live in each pair
 * kernel block's shared memory.  The force adjoint takes at most 16 types. */
#define RBX_MAX_TYPES 64

typedef enum { RBX_PLAIN_FP64 = 0, RBX_MIXED = 1 } rbx_precision;
/* neighbor.type: "Verlet-List", "RBL", "VERLET-SOG" (Verlet list with the
 * short-range SOG Coulomb of RBSOG in place of erfc) */
typedef enum {
  RBX_NEIGHBOR_VERLET = 0,
  RBX_NEIGHBOR_RBL = 1,
  RBX_NEIGHBOR_VERLET_SOG = 2
} rbx_neighbor_type;
/* coulomb.type: RBE, EWALD (op level only), RBSOG */
typedef enum {
  RBX_COULOMB_NONE = 0,
  RBX_COULOMB_RBE = 1,
  RBX_COULOMB_EWALD = 2,
  RBX_COULOMB_RBSOG = 3
} rbx_coulomb_type;

typedef struct {
  int neighbor_type;        /* hyper_parameters.neighbor.type */
  double cut_off;           /* hyper_parameters.neighbor.cut_off */
  double r_core;            /* hyper_parameters.neighbor.r_core (RBL) */
  double skin;              /* hyper_parameters.neighbor.skin */
  int neighbor_sample_num;  /* hyper_parameters.neighbor.neighbor_sample_num */
  int coulomb_type;         /* hyper_parameters.coulomb.type */
  double alpha;             /* hyper_parameters.coulomb.alpha (= g_ewald^2) */
  int coulomb_sample_num;   /* hyper_parameters.coulomb.coulomb_sample_num (P) */
  int kmax[3];              /* hyper_parameters.coulomb.kmax (EWALD) */
  uint64_t random_seed;     /* hyper_parameters.coulomb.random_seed */
  double qqr2e;             /* from init_configuration.read_data.unit */
  double dt;                /* execution.timestep */
  int precision;            /* rbx_precision */
  int ntypes;               /* 1 .. RBX_MAX_TYPES */
  const double* sigma;      /* host, ntypes */
  const double* eps;        /* host, ntypes */
  const double* mass;       /* host, ntypes */
  double fmt2v;             /* force/mass*time -> velocity of the unit style
                               (UnitFactor::_fmt2v; 0 is read as 1, LJ units) */
  int rbsog_level;          /* hyper_parameters.coulomb.rbsog_level (RBSOG,
                               VERLET-SOG) */
  double rbsog_S;           /* RBSOG sampling normalisation: 0 = RBSOGSetup's S
                               (the reference's forces), < 0 = the full S_full
                               (see rbx_rbsog_info), > 0 = this value */
} rbx_params;

/* Engine statistics (host copy). */
typedef struct {
  int64_t steps;            /* velocity-Verlet steps taken */
  int64_t force_calls;      /* force evaluations */
  int64_t rebuilds;         /* neighbor-list rebuilds */
  int epoch;                /* RBL hash epoch / k-sample step of the last evaluation */
  int selection_frequency;  /* RBL pice_num */
  int candidate_capacity;   /* row capacity of the candidate list */
  int64_t candidates;       /* candidate pairs in the list at the last rebuild */
  double e_kspace;          /* last RBE energy (only if requested) */
  double virial_kspace[6];  /* last k-space virial (xx, yy, zz, xy, xz, yz); RBSOG:
                               sampled + direct with the NPT gather chain */
} rbx_stats;

rbx_engine* rbx_engine_create(const rbx_params* params, const rbx_box* box,
                              int num_atoms, int device);
/* Build from the reference's JSON keys (hyper_parameters.force_field/neighbor/
 * coulomb, init_configuration.read_data.unit, execution.timestep) the way
 * LJCutCoulKspace::Init + KSpaceCalculator::Init do
 * (src/force/src/lj_cut_coul_kspace.cpp:424-462, kspace_calculator.cpp:159-355),
 * with the same required-key errors; per-type sigma/eps/mass from host arrays.
 * charges (host, num_atoms) may be NULL unless alpha is derived from
 * coulomb.accuracy. precision: rbx_precision. Returns NULL on error. */
rbx_engine* rbx_engine_create_json(const char* json_text, const rbx_box* box,
                                   int num_atoms, int ntypes, const double* sigma,
                                   const double* eps, const double* mass,
                                   const double* charges, int precision, int device);

/* The force plugin itself: LJCutCoulKspace behind RBMD's Force interface
 * (Init / Execute / EvaluatePotentialEnergy, src/force/include/force.h:10-48),
 * built from the same JSON as rbx_engine_create_json.  rbx_force_engine gives
 * the engine it drives (set positions and k-samples through the engine
 * functions).  rbx_force_execute runs one force evaluation at sample epoch
 * `epoch` and then EvaluatePotentialEnergy; thermo_step stands for
 * ThermoStats::ShouldOutput() (with energy_rbe_flag "yes" the RBE energy of a
 * thermo step is the exact Ewald energy over kmax plus the self energy).
 * rbx_force_energies: {e_vdwl, e_coul, e_kspace, e_pe} of the last
 * evaluation, per atom in LJ units as RBMD reports them (totals in other
 * units); the pair energies only for a Verlet list, or RBL with
 * energy_rbl_flag "yes" (lj_cut_coul_kspace.cpp:570-572, 867-878). */
typedef struct rbx_force rbx_force;
rbx_force* rbx_force_create_json(const char* json_text, const rbx_box* box, int num_atoms,
                                 int ntypes, const double* sigma, const double* eps,
                                 const double* mass, const double* charges, int precision,
                                 int device);
void rbx_force_destroy(rbx_force* f);
rbx_engine* rbx_force_engine(rbx_force* f);
int rbx_force_execute(rbx_force* f, int epoch, int thermo_step);
int rbx_force_energies(rbx_force* f, double out[4]);
void rbx_engine_destroy(rbx_engine* e);
/* Build and load an engine from RBMD's input files the way MDApplication
 * starts (md_application.cpp:175-195, LammpsFullReader::Load,
 * lammps_full_reader.cpp:455-632): the JSON config at json_path ('//' and
 * block comments allowed) names init_configuration.read_data.file (resolved
 * next to the config, else from the working directory), atom_style, unit,
 * replicate and velocity_type GAUSS (execution.temperature[0], velocity_seed);
 * Masses and Pair Coeffs (eps, sigma per type) come from the data file; the
 * plugin parameters as rbx_engine_create_json.  Atoms keep file order (host
 * order), gid = file id - 1, positions wrapped into the box with the wraps
 * added to the file's image flags.  Returns NULL on error. */
rbx_engine* rbx_engine_create_from_files(const char* json_path, int precision, int device);
/* Size, types and box of an engine; per-atom gid / type / charge in host
 * order and per-type sigma / eps / mass.  Any pointer may be NULL. */
int rbx_engine_get_system(rbx_engine* e, int* num_atoms, int* ntypes, rbx_box* box);
int rbx_engine_get_atoms(rbx_engine* e, int* gid, int* type, double* charge);
int rbx_engine_get_type_params(rbx_engine* e, double* sigma, double* eps, double* mass);


/* Host arrays in any atom order; the engine keeps its own (cell-sorted) order. */
int rbx_engine_set_state(rbx_engine* e, const int* gid, const int* type,
                         const double* charge, const double* px, const double* py,
                         const double* pz, const double* vx, const double* vy,
                         const double* vz);
/* Inject the k-samples used by subsequent evaluations (host, p doubles each);
 * pass NULL to return to on-device Philox sampling. */
int rbx_engine_set_k_samples(rbx_engine* e, int p, const double* mx,
                             const double* my, const double* mz);
/* Force evaluation at the current positions with the given epoch (RBL hash
 * epoch and k-sample step), as LJCutCoulKspace::Execute. */
int rbx_engine_compute_forces(rbx_engine* e, int epoch);
/* nsteps velocity-Verlet steps, state resident on the device. */
int rbx_engine_step(rbx_engine* e, int nsteps);
/* One step end to end from host buffers laid out [3][n] (x row, y row, z row),
 * in the atom order given to rbx_engine_set_state: copies x, v in (pinned or
 * pageable), steps once and copies x, v, f out; the copy of x out overlaps the
 * force computation.  Returns when the outputs are on the host. */
int rbx_engine_step_host(rbx_engine* e, const double* x_in, const double* v_in,
                         double* x_out, double* v_out, double* f_out);
/* Copy the state to host arrays, in the atom order of the arrays given to
 * rbx_engine_set_state. Any pointer may be NULL. f is the last total force
 * (real space + k-space). */
int rbx_engine_get_state(rbx_engine* e, double* px, double* py, double* pz,
                         double* vx, double* vy, double* vz, double* fx,
                         double* fy, double* fz);
/* Autotuner (no counterpart in the reference): times the engine's kernels on
 * its current state for each candidate launch shape -- rho(k): k-vectors per
 * thread 1/2/4/8 (32 per warp each) x atom blocks (1, 2, 4, 8 per SM); force
 * scatter: 128/256/512 atoms per block; RBL kernel: 2/4/8/16 waves of
 * resident blocks -- keeps the fastest, and caches the choice per size bin
 * (atom count and k count on a half-octave grid, precision, neighbor and
 * coulomb type), so engines of the same bin reuse it without timing
 * (force = 0).  The choice of atom blocks and waves changes the order of the
 * fixed-order sums (results stay deterministic for a given choice).  Forces
 * are recomputed with the chosen shapes. */
typedef struct {
  int rho_kpt, rho_blocks, force_block, rbl_waves;
  int cache_hit;            /* 1: taken from the cache, nothing timed */
  float rho_ms, force_ms, rbl_ms;      /* best times per launch */
  float rho_ms_default, force_ms_default, rbl_ms_default;  /* built-in shapes */
} rbx_tuning;
int rbx_engine_autotune(rbx_engine* e, int force, rbx_tuning* out);

/* NVT: Nose-Hoover chain thermostat of RBMD's NVT ensemble with
 * temp_ctrl_type NOSE_HOOVER (NVTensemble::Solve, nvt_ensemble.cpp:128-160;
 * NoseHooverController, nose_hoover_controller.cpp): chain length 3, one
 * sub-cycle, temperature ramped t_start -> t_stop over num_steps, damping
 * t_damp (execution.temperature = [t_start, t_stop, t_damp]); kb and mvv2e of
 * the unit style; tdof <= 0 means 3N - 3.  Each step scales the velocities
 * before the first half kick and after the second, as InitialIntegrate /
 * FinalIntegrate do, all on the device (inside the step graph).  Call after
 * rbx_engine_set_state: the chain starts from the current temperature.
 * t_damp <= 0 switches the thermostat off (NVE). */
int rbx_engine_set_nose_hoover(rbx_engine* e, double t_start, double t_stop, double t_damp,
                               int64_t num_steps, double kb, double mvv2e, double tdof);
/* Current thermostat state: temperature (after the last step's scaling),
 * eta[3], eta_dot[3]; any pointer may be NULL. */
int rbx_engine_get_thermostat(rbx_engine* e, double* temperature, double* eta, double* eta_dot);
/* CVFF special bonds on the RBL pair force (ComputeSpecialLJCutCoulRBLForce,
 * src/force/src/cvff_op/rocm/cvff_op.hip.cu:401-533): row h of special
 * ([n][maxspecial], atom indices in the order given to rbx_engine_set_state)
 * lists atom h's 1-2, then 1-3, then 1-4 partners, nspecial[h] ([n][3]) the
 * cumulative counts; a listed pair's LJ is scaled by its weight w and its
 * Coulomb loses (1 - w) times the bare Coulomb, so w = 0 excludes it from
 * real space and cancels its k-space part.  Weights of
 * hyper_parameters.extend.special_bonds.  maxspecial = 0 switches it off.
 * The bonded CVFF terms (bond, angle, dihedral, improper) are not computed. */
int rbx_engine_set_special(rbx_engine* e, int maxspecial, const int* nspecial,
                           const int* special, double w12, double w13, double w14);
/* Special rows from the topology as LammpsFullReader builds them
 * (lammps_full_reader.cpp:2101-2230): bonds [nbonds][2] give 1-2 pairs,
 * angles [nangles][3] their end atoms (1-3), dihedrals [ndihedrals][4] their
 * end atoms (1-4), 0-based atom indices; a repeated pair keeps its first
 * band.  Writes *maxspecial; fills nspecial [n][3] and special
 * [n][*maxspecial] when both are non-NULL (call once for the size). */
int rbx_special_build(int n, int nbonds, const int64_t* bonds, int nangles,
                      const int64_t* angles, int ndihedrals, const int64_t* dihedrals,
                      int* maxspecial, int* nspecial, int* special);
/* SHAKE / RATTLE of rigid three-atom clusters (RBMD's ShakeA / ShakeB,
 * shake_controller_op.hip.cu:19-660, serial path shake_controller.cpp:2130-2220):
 * clusters [nclusters][3] are atom indices in the order given to
 * rbx_engine_set_state with the centre atom second (the angle's atoms, H O H
 * for water); distances held at bond (0-1, 1-2) and
 * sqrt(2 bond^2 (1 - cos angle_deg)) (0-2); RBMD hard-codes bond 1.0 and
 * 109.47 degrees.  Position constraints after the drift, velocity constraints
 * after the second half kick, on the device inside the step.  With the
 * Nose-Hoover thermostat pass tdof = 3N - 3 - N as RBMD's Computedof does.
 * nclusters = 0 switches it off. */
int rbx_engine_set_shake(rbx_engine* e, int nclusters, const int* clusters, double bond,
                         double angle_deg);
/* Clusters in use and the number of cluster solves that did not converge
 * (5000 iterations, 1e-5 on the multipliers) or had a near-singular matrix. */
int rbx_engine_get_shake(rbx_engine* e, int* nclusters, int* failures);
/* Periodic image counters, [n][3] ints in the atom order given to
 * rbx_engine_set_state: how many times each atom has wrapped through each face
 * (+1 leaving through hi).  rbx_engine_set_state zeroes them; the drift of
 * every step counts the wraps (UpdatePositionFlagOp, default_position_controller.cpp:111-121
 * and update_position_op.hip.cu:22, replaces; unwrapped x = x + image * L as
 * UnwarpPositionOp). */
int rbx_engine_set_images(rbx_engine* e, const int* image);
int rbx_engine_get_images(rbx_engine* e, int* image);
/* Append (append != 0) or write one frame in RBMD's trajectory format
 * (TrajectoryOutput::Execute, src/output/src/TrajectoryOutput.cpp:467-500):
 * "ITEM: TIMESTEP", "ITEM: NUMBER OF ATOMS", "ITEM: BOX BOUNDS pp pp pp" with
 * lo hi per axis, then "ITEM: ATOMS id type q x y z xu yu zu vx vy vz" sorted
 * by id, ids and types 1-based, reals in shortest round-trip form. */
int rbx_engine_write_trajectory(rbx_engine* e, const char* path, int64_t timestep, int append);
/* Last real-space (after mean removal for RBL) and k-space forces, [n][3] each,
 * in the atom order given to rbx_engine_set_state. */
int rbx_engine_get_force_parts(rbx_engine* e, double* f_pair, double* f_kspace);
/* LJ and Coulomb (erfc) pair energies and the pair virial (xx, yy, zz, xy,
 * xz, yz) of the current positions over every pair within cut_off, each pair
 * counted from both sides: LJCutCoulKspace::ComputeLJCoulEnergy with
 * LJCutCoulEnergyOp (src/force/src/lj_cut_coul_kspace.cpp:821-865,
 * lj_cut_coul_kspace_op.hip.cu:475-568), which RBMD runs after the RBL force
 * when neighbor.energy_rbl_flag is "yes" and inside the force op for a Verlet
 * list.  FP64 in both precision forms.  Totals: RBMD divides them by the atom
 * count in LJ units.  Any pointer may be NULL.  RBL and Verlet-list engines
 * (VERLET-SOG reports its energies through rbx_pair_force_verlet_sog).  As in
 * RBMD's LJCutCoulEnergyOp, no CVFF special-bond weights are applied: with
 * rbx_engine_set_special the energies and virial still include the excluded
 * and scaled pairs that the force weights. */
int rbx_engine_pair_energy(rbx_engine* e, double* e_vdwl, double* e_coul, double* virial);
/* Exact Ewald reciprocal energy over the kmax box plus the self energy
 * (-qqr2e sqrt(alpha / pi) sum q^2) of the current positions, on the host:
 * KSpaceCalculator::ComputeKspaceEnergy + ComputeSelfEnergy
 * (src/force/src/kspace_calculator.cpp:816-907), which RBMD reports as the RBE
 * k-space energy on thermo steps when coulomb.energy_rbe_flag is "yes"
 * (:630-645).  FP64 in both precision forms. */
int rbx_engine_kspace_energy_exact(rbx_engine* e, const int kmax[3], double* energy);
/* Last RBL lists as (gid_i, gid_j) pairs; sizes in/out. */
int rbx_engine_get_rbl_pairs(rbx_engine* e, int* core_pairs, int64_t* n_core,
                             int* shell_pairs, int64_t* n_shell);
int rbx_engine_get_stats(rbx_engine* e, rbx_stats* out);
/* RBSOG engines: *p = P, and with idx_npt (host int[P], may be NULL) the NPT
 * gather map (see rbx_rbsog_npt_chain) of the last force evaluation's samples. */
int rbx_engine_rbsog_npt_map(rbx_engine* e, int* p, int* idx_npt);
/* Stream the engine launches on (cudaStream_t as void*). */
void* rbx_engine_stream(rbx_engine* e);
/* Mean device time per step since profiling was switched on, per phase, in
 * ms: [0] kick + drift, [1] skin check / rebuild, [2] real space, [3] k-space
 * (sample, rho, finalize, force + combine + kick). */
int rbx_engine_phase_ms(rbx_engine* e, float out[4]);
/* Enable/disable CUDA events around the phases (off by default); resets the
 * accumulated phase times. */
int rbx_engine_set_profiling(rbx_engine* e, int on);
/* Run rbx_engine_step as a CUDA graph per MD step (on, the default) or as
 * individual launches with the host deciding each rebuild (off).  The graph
 * holds kick, drift, the skin check, the neighbour rebuild under a conditional
 * node, the forces and the second kick, with no host synchronisation inside a
 * call of rbx_engine_step; both give identical results.  Profiled steps always
 * run as individual launches.  No counterpart in the reference (its
 * NVEensemble::Solve launches and synchronises step by step). */
int rbx_engine_set_step_graph(rbx_engine* e, int on);

/* Force-field parameters of a live engine (for fitting): per-type LJ sigma
 * and eps ([ntypes]), per-atom charges ([n], host atom order), the RBE/Ewald
 * alpha (JSON alpha = g_ewald^2).  Forces must be computed again afterwards.
 * RBMD reads these once at Init (LJCutCoulKspace::Init, KSpaceCalculator::Init);
 * no counterpart for changing them later. */
int rbx_engine_set_lj_params(rbx_engine* e, const double* sigma, const double* eps);
int rbx_engine_set_charges(rbx_engine* e, const double* charge);
int rbx_engine_set_alpha(rbx_engine* e, double alpha);

/* Adjoint of the last force evaluation (rbx_engine_compute_forces or the last
 * step), for force-field fitting: given g = dL/dF ([n][3], host atom order)
 * it returns dL/d(eps_t) and dL/d(sigma_t) per type ([ntypes]; mixing
 * eps_ij = sqrt(eps_i eps_j), sigma_ij = (sigma_i + sigma_j)/2), dL/dq_i
 * ([n], host order), dL/dalpha ([1]) and dL/dr_i ([n][3], host order, the
 * Hessian-vector product), with the same RBL lists, batch selection and
 * k-samples held fixed.  Computed in FP64 in both forms (the mixed form's
 * rho(k) is recomputed in FP64); any output may be null.  RBL engines only.
 * No counterpart in the reference (RBMD has no adjoint). */
int rbx_engine_force_vjp(rbx_engine* e, const double* g, double* d_eps, double* d_sigma,
                         double* d_charge, double* d_alpha, double* d_pos);

/* ---- LAMMPS data files --------------------------------------------------
 * The reader of RBMD's read_data (LammpsFullReader,
 * src/reader/src/format/lammps/lammps_full_reader.cpp): header counts and
 * orthogonal box, Masses, Pair Coeffs (eps sigma per type), Atoms in the
 * atomic / charge / full style with optional image flags, Velocities, Bonds,
 * Angles, Dihedrals, Impropers.  Ids, types and molecules are returned 0-based
 * as RBMD stores them (its atom id is the RBL batch-hash id); atoms stay in
 * file order.  atom_style may be null (taken from the "Atoms # <style>"
 * comment); replicate (may be null) tiles the box like
 * init_configuration.read_data.replicate. */
typedef struct rbx_lammps_data rbx_lammps_data;
typedef struct rbx_lammps_info {
  int64_t n_atoms, n_bonds, n_angles, n_dihedrals, n_impropers;
  int n_atom_types, n_bond_types, n_angle_types, n_dihedral_types, n_improper_types;
  int atom_style; /* 0 atomic, 1 charge, 2 full */
  int has_masses, has_pair_coeffs, has_velocities, has_images;
  rbx_box box;
} rbx_lammps_info;
rbx_lammps_data* rbx_lammps_read(const char* path, const char* atom_style, const int* replicate);
void rbx_lammps_free(rbx_lammps_data* d);
/* velocity_type GAUSS on a data set read by rbx_lammps_read
 * (LammpsFullReader::ApplyGaussianVelocitiesIfRequested,
 * lammps_full_reader.cpp:710-864): per atom a std::mt19937_64 seeded from
 * (seed, file id), three std::normal_distribution<double> draws / sqrt(mass),
 * centre-of-mass velocity removed, scaled to temperature with 3N - 3 degrees
 * of freedom (kb, mvv2e of unit "LJ" / "REAL" / "METAL").  Needs Masses. */
int rbx_lammps_gauss_velocities(rbx_lammps_data* h, double temperature, const char* unit,
                                int seed);
int rbx_lammps_get_info(const rbx_lammps_data* d, rbx_lammps_info* out);
/* Per-atom arrays of n_atoms entries (image: [n][3]); any may be null. */
int rbx_lammps_get_atoms(const rbx_lammps_data* d, int64_t* id, int* type, int* molecule,
                         double* charge, double* x, double* y, double* z, double* vx,
                         double* vy, double* vz, int* image);
/* Per-type mass, Pair Coeffs eps and sigma ([n_atom_types]); any may be null. */
int rbx_lammps_get_types(const rbx_lammps_data* d, double* mass, double* eps, double* sigma);
/* kind 2 bonds, 3 angles, 4 dihedrals, 5 impropers: types [count] and 0-based
 * atom ids [count][kind == 2 ? 2 : kind == 3 ? 3 : 4]. */
int rbx_lammps_get_topology(const rbx_lammps_data* d, int kind, int* type, int64_t* atoms);
/* Writes an atom_style charge data file with ids id[i] + 1 and types
 * type[i] + 1 (so a reader that makes them 0-based sees id[i], type[i]);
 * velocities may be null. */
int rbx_lammps_write_charge(const char* path, const rbx_box* box, int n, int ntypes,
                            const double* mass, const double* eps, const double* sigma,
                            const int64_t* id, const int* type, const double* charge,
                            const double* x, const double* y, const double* z, const double* vx,
                            const double* vy, const double* vz);

/* ---- Batches of replicas ------------------------------------------------
 * Independent engines on one device advanced together: each rbx_batch_step
 * MD step is one CUDA graph launch.  Two designs of that graph:
 *   RBX_BATCH_PHASED: one kernel launch per phase of the step over the blocks
 *     of every replica (drift with the first half kick and the rebuild
 *     decision; fused RBL force; structure factor with the k-sampling;
 *     finalize; RBE force with the second half kick), each replica's rebuild
 *     under its own conditional node between the drift and the RBL phase.
 *     For RBL engines in the mixed form with RBE k-space, NVE, no SHAKE and
 *     no special bonds;
 *   RBX_BATCH_BRANCHES: every replica's own step graph as a parallel branch.
 * RBX_BATCH_AUTO (the default) takes the phased design for replicas of fewer
 * than 5,000 atoms on average when every replica allows it, else the
 * branches.  The engines stay owned by the caller and
 * must outlive the batch; each must have skin > 0 and profiling off.  Results
 * equal stepping each engine alone, in either design.  No counterpart in the
 * reference (one system per process). */
#define RBX_BATCH_AUTO 0
#define RBX_BATCH_PHASED 1
#define RBX_BATCH_BRANCHES 2
typedef struct rbx_batch rbx_batch;
rbx_batch* rbx_batch_create(rbx_engine* const* engines, int count);
/* Autotune every engine of a batch (rbx_engine_autotune without forcing:
 * replicas of one size bin share one timing); before the first rbx_batch_step.
 * In the phased design replicas whose tuned launch shapes differ take
 * separate launches of a phase. */
int rbx_batch_autotune(rbx_batch* b);
void rbx_batch_destroy(rbx_batch* b);
int rbx_batch_step(rbx_batch* b, int nsteps);
/* The stream the batch graph runs on (cudaStream_t). */
void* rbx_batch_stream(rbx_batch* b);
/* Request a design (RBX_BATCH_AUTO, _PHASED or _BRANCHES; the graph is
 * captured again at the next step).  With RBX_BATCH_PHASED a batch whose
 * replicas do not all allow it fails at rbx_batch_step. */
int rbx_batch_set_mode(rbx_batch* b, int mode);
/* The design of the captured graph (RBX_BATCH_PHASED or RBX_BATCH_BRANCHES),
 * -1 before the first step after creation or a change of mode. */
int rbx_batch_design(const rbx_batch* b);

#ifdef __cplusplus
}
#endif
#endif /* RBX_H */
