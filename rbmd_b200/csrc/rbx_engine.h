// rbx_engine.h -- engine state behind the opaque rbx_engine handle (internal).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "rbx.h"
#include "rbx_kernels.h"

struct rbx_engine {
  // configuration
  rbx_params prm{};
  std::vector<double> sigma, eps, mass;
  rbx_box box{};
  rbx::DBox dbox{};
  int n = 0;
  int device = 0;
  cudaStream_t st = nullptr;
  int dims[3] = {0, 0, 0};
  int ncell = 0;
  int freq = 1;
  rbx::DivTest div{};
  int P = 0;
  // RBSOG: Pk = P + 6 k entries (samples, then the |m| = 1 vectors), per-k
  // weights, the mixture sampler's tables; VERLET-SOG pair parameters
  bool sog = false, sog_pair = false;
  int Pk = 0;
  double sog_self = 0.0;  // self_coeff (E_self = -self_coeff qsq qqr2e)
  double4* sog_w = nullptr;
  double *sog_cdf = nullptr, *sog_tab = nullptr, *sog_tot = nullptr;
  int *sog_off = nullptr, *sog_cnt = nullptr;
  rbx::RbsogTables sog_tables{};
  // k-space virial: the NPT gather chain over the samples (map, multiplicities),
  // per-k NPT weights, the Gaussian weights the chain reads
  double *sog_coef = nullptr, *sog_coef_npt = nullptr, *sog_wv = nullptr;
  int *sog_idx = nullptr, *sog_mult = nullptr;
  rbx::SogGauss sog_gauss{};
  rbx::SogPairParams sogp{};
  int init_rbsog();
  double S = 0.0, qsq = 0.0, qsum = 0.0;
  rbx::PairParams pp{};

  // per-atom device arrays, cell-sorted order
  double *x = nullptr, *y = nullptr, *z = nullptr;
  double *vx = nullptr, *vy = nullptr, *vz = nullptr;
  double *fx = nullptr, *fy = nullptr, *fz = nullptr;     // total force
  double *fpx = nullptr, *fpy = nullptr, *fpz = nullptr;  // real space (before mean removal)
  double *fkx = nullptr, *fky = nullptr, *fkz = nullptr;  // k-space (kept on request)
  double *q = nullptr, *x0 = nullptr, *y0 = nullptr, *z0 = nullptr;
  int *type = nullptr, *gid = nullptr, *orig = nullptr;
  unsigned long long *key_a = nullptr, *key_b = nullptr;
  int* img[3] = {};  // periodic image counters per atom (x, y, z)
  // host-order copies of what set_state received (trajectory output)
  std::vector<int> h_gid, h_type;
  std::vector<double> h_q;
  uint4* atoms = nullptr;  // mixed form: {ux, uy, uz, q_f32}
  double* tmpd = nullptr;
  int* tmpi = nullptr;
  unsigned long long* tmpu = nullptr;
  double* stage = nullptr;  // 9 n doubles for host transfers

  // cells and candidate list
  int *perm = nullptr, *cell_of_sorted = nullptr, *cell_start = nullptr;
  char* cell_scratch = nullptr;
  char* list_scratch = nullptr;
  int cap = 0;
  int *cand_count = nullptr, *cand = nullptr;
  int* cand_far = nullptr;  // RBL engines: far-segment size of each candidate row
  rbx::Rows rows() const {
    rbx::Rows r;
    r.count = cand_count;
    r.far = cand_far;
    r.idx = cand;
    r.cap = cap;
    return r;
  }
  // RBL engines split the candidate rows at r_core + skin (near / far segments)
  const rbx::FarSplit* far_split() {
    if (!cand_far) return nullptr;
    split.r_near = prm.r_core + prm.skin;
    split.far = cand_far;
    return &split;
  }
  rbx::FarSplit split{};
  // blocks of the Verlet pair kernel (its energy partials live in epart)
  int verlet_blocks() const { return std::min(nfpart, rbx::sm_count() * 32); }

  // reductions, flags
  int nfpart = 0;  // capacity of fpart / epart (blocks)
  int nrbl = 0;    // blocks of the fused RBL launch (depends on cap)
  double *fpart = nullptr, *epart = nullptr, *mean = nullptr;
  // [0] cell sort, [1] list overflow, [2] sampler, [3] real-space kernel,
  // [4] device epoch (step graphs), [5] rebuilds inside step graphs,
  // [6] SHAKE solves that failed
  int* dflags = nullptr;
  unsigned long long* max_d2 = nullptr;
  double* inv_mass = nullptr;
  double* mass_d = nullptr;  // per type, for the kinetic energy and SHAKE
  // Nose-Hoover chain thermostat (NVT): device state, its snapshot for graph
  // replays, and the kinetic-energy partial sums
  bool nh_on = false;
  rbx::NHParams nhp{};
  double* nh_state = nullptr;
  double* nh_snap = nullptr;
  double* ke_part = nullptr;
  // SHAKE / RATTLE clusters (host indices, centre second), the host index ->
  // cell slot map, positions before the drift, failure counter (dflags[6])
  int shake_nc = 0, shake_cap = 0;
  rbx::ShakeParams shp{};
  int* shake_cl = nullptr;
  int* where = nullptr;
  double* xs = nullptr;
  double* ys = nullptr;
  double* zs = nullptr;
  int shake_a(cudaStream_t s);
  int shake_b(cudaStream_t s);
  int set_shake(int nclusters, const int* clusters, double bond, double angle_deg);
  // launch shapes picked by the autotuner: k-vectors per thread and atom
  // blocks of rho(k), atoms per block of the force scatter, waves of the RBL
  // kernel (defaults = the built-in heuristics)
  struct Tuning {
    int rho_kpt = 4, rho_parts = 0, frc_block = 256, rbl_waves = 8;
  };
  Tuning tun;
  int nparts_cap = 0;
  int autotune(bool force, rbx_tuning* out);
  int apply_tuning(const Tuning& t);
  // CVFF special bonds (host order): cumulative 1-2/1-3/1-4 counts [n][3],
  // partner host indices [n][spec_max], the atoms that have any, weights
  int spec_max = 0, spec_cap = 0, spec_natoms = 0;
  int* spec_cnt = nullptr;
  int* spec_part = nullptr;
  int* spec_atoms = nullptr;
  double spec_w[3] = {1, 1, 1};
  int set_special(int maxspecial, const int* nspecial, const int* special, double w12,
                  double w13, double w14);
  double *lj_eps = nullptr, *lj_s6 = nullptr;
  unsigned long long* h_pinned = nullptr;

  // RBE
  int nparts = 0;
  double *mx = nullptr, *my = nullptr, *mz = nullptr;
  int* mi = nullptr;
  double *part_re = nullptr, *part_im = nullptr, *rho_re = nullptr, *rho_im = nullptr;
  rbx::KTab* tab = nullptr;
  double* kterm = nullptr;  // per-k energy/virial terms [P][8]
  double *ek = nullptr, *virk = nullptr;
  double* sample_tables = nullptr;
  int tcnt[3] = {0, 0, 0};
  double ttot[3] = {0, 0, 0};

  // arrays a rebuild permutes move through shadow copies and back, so every
  // device array keeps its address (a captured step graph stays valid)
  double* shd[13] = {};
  int* shi[6] = {};
  unsigned long long* shu[2] = {};
  // state saved before a run of graph steps (restored if a rebuild inside
  // the graph ran out of capacity): x y z vx vy vz fx fy fz q, type gid orig,
  // images, keys
  double* snapd[10] = {};
  int* snapi[6] = {};
  unsigned long long* snapu[2] = {};

  // CUDA graph of one MD step, the rebuild under a conditional (IF) node
  bool use_graph = true;
  bool graph_dirty = true;   // addresses, capacity or modes changed: capture again
  unsigned graph_version = 0;  // bumped on each such change (batch graphs compare it)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  cudaStream_t st_body = nullptr;  // captures the rebuild body
  unsigned long long graph_step_launches = 0, graph_rebuild_launches = 0;
  // the same step as two graphs for rbx_engine_step_host: [0] up to the drift
  // (+ SHAKE) and the positions in host order, [1] the rest; the copy of the
  // positions to the host runs on st_side while [1] computes the forces
  bool host_graph_dirty = true;
  cudaGraph_t hgraph[2] = {nullptr, nullptr};
  cudaGraphExec_t hexec[2] = {nullptr, nullptr};
  cudaStream_t st_side = nullptr;
  cudaEvent_t ev_side = nullptr;
  // inside a step graph the k-sampling and the structure factor run on a
  // branch of their own (st_ks), beside the real-space force
  cudaStream_t st_ks = nullptr;
  cudaEvent_t ev_ks[2] = {nullptr, nullptr};
  unsigned long long host_step_launches = 0;
  int* run_init = nullptr;   // pinned: device epoch / counter seeds of a graph run
  int* run_flags = nullptr;  // pinned: dflags[0..5] after a graph run

  // adjoint scratch (allocated on first use)
  double* adj_buf = nullptr;
  size_t adj_len = 0;

  // bookkeeping
  bool have_cache = false, have_forces = false, k_injected = false, keep_parts = false;
  bool profiling = false;
  int epoch = 0;
  long long steps = 0, force_calls = 0, rebuilds = 0;
  cudaEvent_t ev[8] = {};
  // accumulated device time per phase while profiling is on
  std::vector<cudaEvent_t> pev;  // 5 events per profiled step
  int pev_used = 0;
  double phase_total[4] = {0, 0, 0, 0};
  long long phase_steps = 0;
  long long* cand_total = nullptr;  // device: sum of candidate counts at the last rebuild
  std::vector<void*> allocs;

  ~rbx_engine();
  int init();
  int set_state(const int* gid, const int* type, const double* q, const double* x,
                const double* y, const double* z, const double* vx, const double* vy,
                const double* vz);
  int set_k_samples(int p, const double* mx, const double* my, const double* mz);
  int rebuild();
  int rebuild_launches(cudaStream_t s, bool in_graph);  // the device work of a rebuild
  rbx::ArraySet permute_set(bool to_shadow) const;
  rbx::ArraySet state_set(bool save) const;
  int capture_step_graph();
  int capture_step_into(cudaGraph_t g, bool fork_kspace = true);
  // kick, drift (+ SHAKE) on st; with cond (same graph as the tail) the drift
  // kernel takes the rebuild decision itself, and *decided says whether it does
  int capture_step_head(const cudaGraphConditionalHandle* cond = nullptr, bool* decided = nullptr);
  // the rebuild, captured on st_body into the body graph of an IF node
  int capture_rebuild_body(cudaGraph_t body);
  // a graph step without its rebuild, recorded for a phase-batched graph
  // (rbx_batch.cu); RBX_ERR_INVALID when a kernel of the step has no batched form
  int record_phased_step(rbx::BatchRecorder* rec, cudaGraphConditionalHandle cond);
  // decide (unless decided), rebuild (IF node on cond, or a new handle), forces, ... on st
  // fork_kspace: the k-sampling and structure factor on a branch beside the
  // real-space force (off inside a batch graph of one branch per replica,
  // where the replicas' branches already run side by side)
  int capture_step_tail(cudaGraph_t g, const cudaGraphConditionalHandle* cond = nullptr,
                        bool decided = false, bool fork_kspace = true);
  int capture_host_graphs();
  void release_host_graphs();
  int graph_run_begin(cudaStream_t s);
  int graph_run_end(int nsteps, unsigned long long step_launches);
  int step_graph(int nsteps);
  int step_plain(int nsteps);
  void release_graph();
  int check_rebuild(bool disp_from_drift);
  int real_space(const int* epoch_dev = nullptr);
  int kspace_and_combine(bool kick, const int* epoch_dev = nullptr);
  // its two parts: the k-sampling and structure-factor partial sums on stream
  // s, then the finalize and the force scatter (+ combine, kick) on st
  int kspace_rho(cudaStream_t s, const int* epoch_dev);
  int kspace_finish(bool kick, const int* epoch_dev);
  int compute_forces(int epoch);
  int check_sampler();
  int step(int nsteps);
  int step_host(const double* xin, const double* vin, double* xout, double* vout, double* fout);
  int get_state(double* px, double* py, double* pz, double* vx, double* vy, double* vz,
                double* fx, double* fy, double* fz);
  int get_force_parts(double* f_pair, double* f_kspace);
  int pair_energy(double* e_vdwl, double* e_coul, double* virial);
  int kspace_energy_exact(const int kmax[3], double* energy);
  int get_rbl_pairs(int* core_pairs, int64_t* n_core, int* shell_pairs, int64_t* n_shell);
  int get_stats(rbx_stats* s);
  int set_images(const int* image);
  int set_nose_hoover(double t_start, double t_stop, double t_damp, long long num_steps,
                      double kb, double mvv2e, double tdof);
  int get_thermostat(double* temperature, double* eta, double* eta_dot);
  int nh_initial(const int* step_dev, long long step_add, cudaStream_t s);
  int nh_final(cudaStream_t s);
  int get_images(int* image);
  int write_trajectory(const char* path, int64_t timestep, bool append);
  int upload_type_tables();
  int build_sampler_tables();
  int set_lj_params(const double* sigma, const double* eps);
  int set_charges(const double* q);
  int set_alpha(double alpha);
  int force_vjp(const double* g, double* d_eps, double* d_sigma, double* d_q, double* d_alpha,
                double* d_r);
  int phase_ms(float out[4]);
  int flush_profile();

  template <typename T>
  int alloc(T** p, size_t count);
  template <typename T>
  void release(T*& p);
};
