/*
 * rbx_oracle.h -- FP64 host restatement of RBMD's RBE + LJ/erfc-Coulomb force
 * path.  TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check and the
 * bench's CPU-baseline leg call it as the checker.  The product (librbx) never
 * links or calls it.
 *
 * Every function names the reference file:line it restates (paths relative to
 * the RBMD 2.0 source tree).  Parity pin: the restatement is checked against
 * the reference's own kernels compiled from their sources and run on B200
 * (fixtures under tests/golden/, generating script tests/golden/make_golden.py).
 */
#ifndef RBX_ORACLE_H
#define RBX_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Orthogonal, fully periodic box (src/data_manager/include/model/box.h:5-49). */
typedef struct {
  double lo[3];
  double hi[3];
} orc_box;

/* ---- k-space (RBE / Ewald) ---------------------------------------------- */
double orc_rbe_gauss_sum(const orc_box* box, double alpha);
void orc_rbe_structure_factor(int n, int p, const orc_box* box, const double* q,
                              const double* x, const double* y, const double* z,
                              const double* mx, const double* my,
                              const double* mz, double* re, double* im);
void orc_rbe_force(int n, int p, const orc_box* box, double S, double qqr2e,
                   const double* re, const double* im, const double* q,
                   const double* mx, const double* my, const double* mz,
                   const double* x, const double* y, const double* z,
                   double* fx, double* fy, double* fz);
void orc_rbe_energy_virial(int p, const orc_box* box, double alpha, double S,
                           double qqr2e, double qsq, double qsum,
                           const double* re, const double* im,
                           const double* mx, const double* my,
                           const double* mz, double* virial6, double* energy);
int orc_ewald_num_k(const int kmax[3]);
void orc_ewald_kvectors(const int kmax[3], const orc_box* box, double* kx,
                        double* ky, double* kz);
void orc_ewald_structure_factor(int n, int nk, const double* q,
                                const double* x, const double* y,
                                const double* z, const double* kx,
                                const double* ky, const double* kz, double* re,
                                double* im);
void orc_ewald_force(int n, int nk, const orc_box* box, double alpha,
                     double qqr2e, const double* kx, const double* ky,
                     const double* kz, const double* re, const double* im,
                     const double* q, const double* x, const double* y,
                     const double* z, double* fx, double* fy, double* fz);
double orc_ewald_energy(int nk, const orc_box* box, double alpha, double qqr2e,
                        double qsq, const double* kx, const double* ky,
                        const double* kz, const double* re, const double* im);

/* ---- k-vector samplers ---------------------------------------------------- */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2],
                       uint32_t out[4]);
int orc_rbe_sample_philox(int p, const orc_box* box, double alpha,
                          uint64_t seed, int64_t step, double* mx, double* my,
                          double* mz);
void orc_rbe_sample_mh(int p, const orc_box* box, double alpha, uint64_t seed,
                       double* mx, double* my, double* mz);

/* ---- geometry, cells, lists ---------------------------------------------- */
double orc_dist2(const orc_box* box, double xi, double yi, double zi, double xj,
                 double yj, double zj);
int orc_cell_grid(const orc_box* box, double neighbor_cutoff, int dims[3]);
int orc_cells_sort(int n, const orc_box* box, double neighbor_cutoff,
                   const double* x, const double* y, const double* z,
                   int* perm, int* cell_of_sorted, int* cell_start,
                   int* cell_end);
int64_t orc_full_list(int n, const orc_box* box, double neighbor_cutoff,
                      const double* x, const double* y, const double* z,
                      const int* cell_of, const int* cell_start,
                      const int* cell_end, int cap, int* count, int* nbrs);
int orc_rbl_params(int n_global, const orc_box* box, double r_core,
                   double cut_off, int sample_num, int* rs_num, int* rc_num);
uint64_t orc_rbl_mix(uint64_t v);
int orc_rbl_selected(int freq, int epoch, int gid_i, int gid_j);
void orc_rbl_filter(int n, const orc_box* box, double r_core, double cut_off,
                    int freq, int epoch, const int* gid, const double* x,
                    const double* y, const double* z, int cap,
                    const int* cand_count, const int* cand, int* core_count,
                    int* core, int* shell_count, int* shell);

/* ---- pair forces ----------------------------------------------------------- */
void orc_pair_force_rbl(int n, const orc_box* box, double r_core, double cut_off,
                        int freq, double alpha, double qqr2e, const int* type,
                        const double* sigma, const double* eps, const double* q,
                        const double* x, const double* y, const double* z,
                        int cap, const int* core_count, const int* core,
                        const int* shell_count, const int* shell, double* fx,
                        double* fy, double* fz);
/* CVFF RBL pair force with special-bond weights (specials indexed by atom
 * index i, partners as gids; special may be NULL). */
void orc_pair_force_rbl_special(int n, const orc_box* box, double r_core, double cut_off,
                                int freq, double alpha, double qqr2e, const int* type,
                                int ntypes, const double* lj12, const double* lj6,
                                const int* gid, const double* q, const double* x,
                                const double* y, const double* z, int cap,
                                const int* core_count, const int* core, const int* shell_count,
                                const int* shell, const int* nspecial, const int* special,
                                int maxs, double w12, double w13, double w14, double* fx,
                                double* fy, double* fz);
void orc_fix_rbl(int n, double* fx, double* fy, double* fz, double mean_out[3]);
void orc_pair_force_verlet(int n, const orc_box* box, double cut_off,
                           double alpha, double qqr2e, const int* type,
                           const double* sigma, const double* eps,
                           const double* q, const double* x, const double* y,
                           const double* z, int cap, const int* count,
                           const int* nbrs, double* fx, double* fy, double* fz,
                           double* virial6, double* evdwl, double* ecoul);
double orc_max_disp2(int n, const orc_box* box, const double* x,
                     const double* y, const double* z, const double* x0,
                     const double* y0, const double* z0);

/* ---- whole MD step (CPU baseline) ----------------------------------------- */
typedef struct orc_engine orc_engine;
orc_engine* orc_engine_create(int n, const orc_box* box, int ntypes,
                              const double* sigma, const double* eps,
                              const double* mass, double cut_off, double r_core,
                              double skin, int neighbor_sample_num,
                              double alpha, int kspace_p, double qqr2e,
                              double dt, uint64_t seed, int use_rbl);
void orc_engine_destroy(orc_engine* e);
int orc_engine_set_state(orc_engine* e, const int* gid, const int* type,
                         const double* q, const double* x, const double* y,
                         const double* z, const double* vx, const double* vy,
                         const double* vz);
int orc_engine_compute_forces(orc_engine* e, int epoch);
int orc_engine_step(orc_engine* e, int nsteps);
int orc_engine_get(orc_engine* e, int* gid, double* x, double* y, double* z,
                   double* vx, double* vy, double* vz, double* fx, double* fy,
                   double* fz);
int orc_engine_rebuilds(const orc_engine* e);
/* NVT with the Nose-Hoover chain (t_damp <= 0: off; tdof <= 0: 3N - 3). */
int orc_engine_set_nose_hoover(orc_engine* e, double t_start, double t_stop, double t_damp,
                               long long num_steps, double kb, double mvv2e, double tdof);
void orc_engine_get_thermostat(const orc_engine* e, double* temperature, double* eta,
                               double* eta_dot);
/* Unit style's force/mass*time -> velocity factor (1 for LJ). */
void orc_engine_set_fmt2v(orc_engine* e, double fmt2v);
/* SHAKE / RATTLE clusters given by gid, centre second (nc = 0: off). */
int orc_engine_set_shake(orc_engine* e, int nc, const int* cluster_gids, double bond,
                         double angle_deg);
int orc_engine_shake_failures(const orc_engine* e);
int orc_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
