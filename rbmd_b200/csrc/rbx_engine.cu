// rbx_engine.cu -- the engine behind rbx_engine_*: the force evaluation of
// LJCutCoulKspace::Execute (src/force/src/lj_cut_coul_kspace.cpp:464-471:
// real space, then KSpaceCalculator::Execute, then SumForces) and the NVE
// velocity-Verlet step of NVEensemble::Solve
// (src/simulate_pipeline/src/nve_ensemble.cpp:59-91), with all state resident
// on one GPU in cell-sorted order.
//
// Per step (RBL + RBE): kick, drift(+wrap, +skin check, +fixed point),
// [rebuild if max displacement > skin/2], fused RBL filter+pair force, Philox
// k-sample, rho(k) partials, finalize (rho, energy/virial, force table, RBL
// mean force), k-space force fused with SumForces, the mean removal and the
// second half kick.  Host syncs per step: one 8-byte read of the displacement
// maximum.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <cmath>
#include <charconv>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "rbx.h"
#include "rbx_common.cuh"
#include "rbx_engine.h"
#include "rbx_kernels.h"
#include "host/rbsog.h"

namespace rbx {
int require_device();
double gauss_sum(const rbx_box& b, double alpha);
double gauss_sum_dalpha(const rbx_box& b, double alpha);
int rbl_freq(int n_global, const rbx_box& b, double r_core, double cut_off, int sample_num);
}  // namespace rbx

using namespace rbx;

#define ETRY(expr)          \
  do {                      \
    const int _rc = (expr); \
    if (_rc) return _rc;    \
  } while (0)

static int cuda_ok(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error("%s: %s", what, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? RBX_ERR_NOMEM : RBX_ERR_CUDA;
  }
  return RBX_OK;
}

template <typename T>
static int dalloc(T** p, size_t count) {
  if (count == 0) count = 1;
  return cuda_ok(cudaMalloc((void**)p, sizeof(T) * count), "cudaMalloc");
}

rbx_engine::~rbx_engine() {
  if (device >= 0) cudaSetDevice(device);
  for (void* ptr : allocs) cudaFree(ptr);
  if (h_pinned) cudaFreeHost(h_pinned);
  for (int i = 0; i < 8; ++i)
    if (ev[i]) cudaEventDestroy(ev[i]);
  for (cudaEvent_t e : pev) cudaEventDestroy(e);
  release_graph();
  release_host_graphs();
  if (ev_side) cudaEventDestroy(ev_side);
  if (st_side) cudaStreamDestroy(st_side);
  for (cudaEvent_t e : ev_ks)
    if (e) cudaEventDestroy(e);
  if (st_ks) cudaStreamDestroy(st_ks);
  if (st_body) cudaStreamDestroy(st_body);
  if (st) cudaStreamDestroy(st);
}

void rbx_engine::release_host_graphs() {
  for (int k = 0; k < 2; ++k) {
    if (hexec[k]) cudaGraphExecDestroy(hexec[k]);
    if (hgraph[k]) cudaGraphDestroy(hgraph[k]);
    hexec[k] = nullptr;
    hgraph[k] = nullptr;
  }
  host_graph_dirty = true;
}

void rbx_engine::release_graph() {
  if (graph_exec) cudaGraphExecDestroy(graph_exec);
  if (graph) cudaGraphDestroy(graph);
  graph_exec = nullptr;
  graph = nullptr;
  graph_dirty = true;
}

template <typename T>
int rbx_engine::alloc(T** p, size_t count) {
  ETRY(dalloc(p, count));
  allocs.push_back((void*)*p);
  return RBX_OK;
}

template <typename T>
void rbx_engine::release(T*& p) {
  if (!p) return;
  auto it = std::find(allocs.begin(), allocs.end(), (void*)p);
  if (it != allocs.end()) allocs.erase(it);
  cudaFree(p);
  p = nullptr;
}

int rbx_engine::init() {
  ETRY(cuda_ok(cudaSetDevice(device), "cudaSetDevice"));
  ETRY(require_device());
  ETRY(cuda_ok(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate"));
  ETRY(cuda_ok(cudaStreamCreateWithFlags(&st_body, cudaStreamNonBlocking), "cudaStreamCreate"));
  ETRY(cuda_ok(cudaStreamCreateWithFlags(&st_side, cudaStreamNonBlocking), "cudaStreamCreate"));
  ETRY(cuda_ok(cudaEventCreateWithFlags(&ev_side, cudaEventDisableTiming), "cudaEventCreate"));
  ETRY(cuda_ok(cudaStreamCreateWithFlags(&st_ks, cudaStreamNonBlocking), "cudaStreamCreate"));
  for (cudaEvent_t& e : ev_ks)
    ETRY(cuda_ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate"));
  dbox = make_dbox(box);
  const bool rbl = prm.neighbor_type == RBX_NEIGHBOR_RBL;
  if (!(prm.cut_off > 0.0) || prm.skin < 0.0 || (rbl && !(prm.r_core > 0.0)) ||
      (rbl && prm.neighbor_sample_num <= 0)) {
    set_error("invalid neighbor parameters (cut_off > 0, skin >= 0, r_core > 0, "
              "neighbor_sample_num > 0 for RBL)");
    return RBX_ERR_CONFIG;
  }
  if (prm.coulomb_type == RBX_COULOMB_RBE && (prm.coulomb_sample_num <= 0 || !(prm.alpha > 0))) {
    set_error("RBE needs coulomb_sample_num > 0 and alpha > 0");
    return RBX_ERR_CONFIG;
  }
  if (prm.coulomb_type == RBX_COULOMB_RBSOG && prm.coulomb_sample_num <= 0) {
    set_error("RBSOG needs coulomb_sample_num > 0");
    return RBX_ERR_CONFIG;
  }
  if (prm.coulomb_type != RBX_COULOMB_NONE && prm.coulomb_type != RBX_COULOMB_RBE &&
      prm.coulomb_type != RBX_COULOMB_RBSOG) {
    set_error("the engine runs coulomb types NONE, RBE and RBSOG");
    return RBX_ERR_CONFIG;
  }
  if (prm.neighbor_type != RBX_NEIGHBOR_VERLET && prm.neighbor_type != RBX_NEIGHBOR_RBL &&
      prm.neighbor_type != RBX_NEIGHBOR_VERLET_SOG) {
    set_error("neighbor type must be Verlet-List, RBL or VERLET-SOG");
    return RBX_ERR_CONFIG;
  }
  if (prm.ntypes <= 0 || prm.ntypes > RBX_MAX_TYPES) {
    set_error("ntypes must be in [1, %d]", RBX_MAX_TYPES);
    return RBX_ERR_CONFIG;
  }
  for (int d = 0; d < 3; ++d)
    if (prm.cut_off + prm.skin > 0.5 * dbox.len[d]) {
      set_error("cut_off + skin (%g) exceeds half the box length (%g) along dimension %d",
                prm.cut_off + prm.skin, 0.5 * dbox.len[d], d);
      return RBX_ERR_CONFIG;
    }
  // cells of edge >= cut_off + skin, floor(L / (cut_off + skin)) per axis (at
  // least two, by the check above); with fewer than three along an axis the
  // candidate rows come from the all-pairs builder instead of the stencil
  for (int d = 0; d < 3; ++d) dims[d] = (int)floor(dbox.len[d] / (prm.cut_off + prm.skin));
  ncell = dims[0] * dims[1] * dims[2];
  freq = rbl ? rbl_freq(n, box, prm.r_core, prm.cut_off, prm.neighbor_sample_num) : 1;
  div = make_divtest(freq);
  sog = prm.coulomb_type == RBX_COULOMB_RBSOG;
  sog_pair = prm.neighbor_type == RBX_NEIGHBOR_VERLET_SOG;
  P = (prm.coulomb_type == RBX_COULOMB_RBE || sog) ? prm.coulomb_sample_num : 0;
  Pk = sog ? P + 6 : P;
  S = (P > 0 && !sog) ? gauss_sum(box, prm.alpha) : 0.0;

  const size_t N = (size_t)n;
  double** dptrs[] = {&x, &y, &z, &vx, &vy, &vz, &fx, &fy, &fz, &q, &x0, &y0, &z0,
                      &fpx, &fpy, &fpz, &fkx, &fky, &fkz, &tmpd};
  for (double** p : dptrs) ETRY(alloc(p, N));
  ETRY(alloc(&stage, 9 * N));  // host transfer staging (x,v in; x,v,f out)
  for (double*& p : shd) ETRY(alloc(&p, N));
  for (int*& p : shi) ETRY(alloc(&p, N));
  for (int*& p : img) ETRY(alloc(&p, N));
  for (unsigned long long*& p : shu) ETRY(alloc(&p, N));
  for (double*& p : snapd) ETRY(alloc(&p, N));
  for (int*& p : snapi) ETRY(alloc(&p, N));
  for (unsigned long long*& p : snapu) ETRY(alloc(&p, N));
  int** iptrs[] = {&type, &gid, &orig, &tmpi, &perm, &cell_of_sorted, &cand_count};
  for (int** p : iptrs) ETRY(alloc(p, N));
  // RBL rows of the mixed form are split at r_core + skin (far pairs take the
  // batch hash before any gather).  The plain FP64 form keeps one segment:
  // its split kernel queues the selected far pairs before their window test,
  // and those beyond cut_off at the step pay the FP64 pair math for nothing,
  // while the unsplit list builds faster
  if (prm.neighbor_type == RBX_NEIGHBOR_RBL && prm.precision == RBX_MIXED)
    ETRY(alloc(&cand_far, N));
  ETRY(alloc(&key_a, N));
  ETRY(alloc(&key_b, N));
  ETRY(alloc(&tmpu, N));
  ETRY(alloc(&atoms, N));
  ETRY(alloc(&cell_start, (size_t)ncell + 1));
  ETRY(alloc(&cell_scratch, cells_scratch_bytes(n, ncell)));
  ETRY(alloc(&list_scratch, full_list_scratch_bytes(n, ncell)));
  ETRY(alloc(&dflags, 12));  // [8], [9]: block counters of the drift and the RBE finalize
  ETRY(cuda_ok(cudaMemsetAsync(dflags, 0, sizeof(int) * 12, st), "memset"));
  ETRY(alloc(&max_d2, 1));
  ETRY(alloc(&cand_total, 1));
  nfpart = rbl_fused_blocks(n);
  ETRY(alloc(&fpart, (size_t)(nfpart + SPEC_PARTS) * 3));
  ETRY(alloc(&epart, (size_t)nfpart * 8));
  ETRY(alloc(&mean, 3));
  ETRY(alloc(&ek, 1));
  ETRY(alloc(&virk, 6));
  ETRY(alloc(&inv_mass, (size_t)prm.ntypes));
  ETRY(alloc(&mass_d, (size_t)prm.ntypes));
  ETRY(alloc(&nh_state, (size_t)NH_SLOTS));
  ETRY(alloc(&nh_snap, (size_t)NH_SLOTS));
  ETRY(alloc(&ke_part, (size_t)KE_PARTS));
  ETRY(cuda_ok(cudaMemsetAsync(nh_state, 0, sizeof(double) * NH_SLOTS, st), "memset"));
  ETRY(alloc(&lj_eps, (size_t)prm.ntypes * prm.ntypes));
  ETRY(alloc(&lj_s6, (size_t)prm.ntypes * prm.ntypes));
  // LJ mixing of ComputeLJCutCoulRBLForce (lj_cut_coul_kspace_op.hip.cu:582-600):
  ETRY(upload_type_tables());
  if (P > 0) {
    nparts = rbe_partial_blocks(n);
    nparts_cap = std::max(nparts, 8 * sm_count());
    ETRY(alloc(&mx, (size_t)Pk));
    ETRY(alloc(&my, (size_t)Pk));
    ETRY(alloc(&mz, (size_t)Pk));
    ETRY(alloc(&mi, (size_t)3 * Pk));
    ETRY(alloc(&part_re, (size_t)nparts_cap * Pk));
    ETRY(alloc(&part_im, (size_t)nparts_cap * Pk));
    ETRY(alloc(&rho_re, (size_t)Pk));
    ETRY(alloc(&rho_im, (size_t)Pk));
    ETRY(alloc(&tab, (size_t)Pk));
    ETRY(alloc(&kterm, (size_t)8 * Pk));
    if (!sog) ETRY(build_sampler_tables());
  } else {
    ETRY(alloc(&tab, 1));
    ETRY(alloc(&mx, 1));
    ETRY(alloc(&my, 1));
    ETRY(alloc(&mz, 1));
  }
  if (sog || sog_pair) ETRY(init_rbsog());
  // candidate capacity from the number density, with headroom (a row that
  // overflows triggers a regrow and rebuild)
  const double V = dbox.len[0] * dbox.len[1] * dbox.len[2];
  const double rcs = prm.cut_off + prm.skin;
  const double expect = (double)n / V * 4.0 / 3.0 * M_PI * rcs * rcs * rcs;
  cap = ((int)(1.3 * expect + 64) + 31) / 32 * 32;
  ETRY(alloc(&cand, N * (size_t)cap));
  ETRY(cuda_ok(cudaHostAlloc((void**)&h_pinned, 128, cudaHostAllocDefault), "cudaHostAlloc"));
  run_init = (int*)(h_pinned + 2);   // 2 ints
  run_flags = (int*)(h_pinned + 4);  // 6 ints
  for (int i = 0; i < 8; ++i) ETRY(cuda_ok(cudaEventCreate(&ev[i]), "cudaEventCreate"));
  pp.box = dbox;
  pp.rs2 = prm.r_core * prm.r_core;
  pp.rc2 = prm.cut_off * prm.cut_off;
  pp.core2_list = prm.r_core * prm.r_core - RBX_EPSILON;
  pp.force2_list = prm.cut_off * prm.cut_off - RBX_EPSILON;
  pp.alpha = prm.alpha;
  pp.sqrt_alpha = sqrt(prm.alpha);
  pp.qqr2e = prm.qqr2e;
  pp.freq = freq;
  nrbl = rbl_fused_grid(prm.precision == RBX_MIXED, freq, n, cap, nfpart, tun.rbl_waves,
                        prm.ntypes);
  pp.div = div;
  pp.ntypes = prm.ntypes;
  pp.lj_eps = lj_eps;
  pp.lj_s6 = lj_s6;
  for (int d = 0; d < 3; ++d) pp.sf[d] = (float)(dbox.len[d] / 4294967296.0);
  // fixed-point screens: the guard band covers the fixed-point quantisation
  // (< 3 units of L_d/2^32 per coordinate, at most 3 units of L_max/2^32 once
  // weighted by L_d/L_max) with a wide margin
  pp.cubic = dbox.len[0] == dbox.len[1] && dbox.len[1] == dbox.len[2];
  {
    const double L = std::max(dbox.len[0], std::max(dbox.len[1], dbox.len[2]));
    for (int d = 0; d < 3; ++d) pp.sw[d] = (float)(dbox.len[d] / L);
    // FP32 |d|^2 carries < 1e-6 relative rounding (the weights add two
    // roundings per coordinate, < 2e-7 more) plus < 6 s |d| of quantisation
    // error; the band is several times both
    const double qerr = 64.0 * (L / 4294967296.0) * (rcs + 1.0);
    auto band = [&](double C) { return 1e-4 + 8e-6 * C + qerr; };
    pp.sc_eps = make_screen(RBX_EPSILON, L, std::min(band(RBX_EPSILON), 0.5 * RBX_EPSILON));
    pp.sc_core = make_screen(pp.core2_list, L, band(pp.core2_list));
    pp.sc_rs = make_screen(pp.rs2, L, band(pp.rs2));
    pp.sc_force = make_screen(pp.force2_list, L, band(pp.force2_list));
    pp.sc_rc = make_screen(pp.rc2, L, band(pp.rc2));
  }
  return RBX_OK;
}

int rbx_engine::set_state(const int* hgid, const int* htype, const double* hq, const double* hx,
                          const double* hy, const double* hz, const double* hvx,
                          const double* hvy, const double* hvz) {
  cudaSetDevice(device);
  const size_t N = (size_t)n;
  for (int i = 0; i < n; ++i)
    if (htype[i] < 0 || htype[i] >= prm.ntypes) {
      set_error("atom %d has type %d outside [0, %d)", i, htype[i], prm.ntypes);
      return RBX_ERR_INVALID;
    }
  std::vector<int> horig(N);
  for (int i = 0; i < n; ++i) horig[i] = i;
  qsq = 0;
  qsum = 0;
  for (int i = 0; i < n; ++i) {
    qsq += hq[i] * hq[i];
    qsum += hq[i];
  }
  const double* hsrc[] = {hx, hy, hz, hvx, hvy, hvz, hq};
  double* ddst[] = {x, y, z, vx, vy, vz, q};
  for (int a = 0; a < 7; ++a)
    ETRY(cuda_ok(cudaMemcpyAsync(ddst[a], hsrc[a], sizeof(double) * N, cudaMemcpyHostToDevice, st),
                 "H2D state"));
  ETRY(cuda_ok(cudaMemcpyAsync(type, htype, sizeof(int) * N, cudaMemcpyHostToDevice, st), "H2D"));
  ETRY(cuda_ok(cudaMemcpyAsync(gid, hgid, sizeof(int) * N, cudaMemcpyHostToDevice, st), "H2D"));
  ETRY(cuda_ok(cudaMemcpyAsync(orig, horig.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st),
               "H2D"));
  if (where) ETRY(launch_inverse_perm(n, orig, where, st));
  ETRY(cuda_ok(cudaMemsetAsync(fx, 0, sizeof(double) * N, st), "memset"));
  ETRY(cuda_ok(cudaMemsetAsync(fy, 0, sizeof(double) * N, st), "memset"));
  ETRY(cuda_ok(cudaMemsetAsync(fz, 0, sizeof(double) * N, st), "memset"));
  ETRY(launch_rbl_keys(n, gid, key_a, key_b, st));
  for (int d = 0; d < 3; ++d)
    ETRY(cuda_ok(cudaMemsetAsync(img[d], 0, sizeof(int) * N, st), "memset"));
  h_gid.assign(hgid, hgid + n);
  h_type.assign(htype, htype + n);
  h_q.assign(hq, hq + n);
  ETRY(cuda_ok(cudaStreamSynchronize(st), "set_state sync"));
  have_cache = false;
  have_forces = false;
  epoch = 0;
  graph_dirty = host_graph_dirty = true;
  ++graph_version;
  return RBX_OK;
}

// The per-atom arrays a rebuild permutes, moved into their shadows
// (to_shadow, through perm) or copied back (with x0 = x for the skin check).
ArraySet rbx_engine::permute_set(bool to_shadow) const {
  ArraySet a{};
  double* const pd[13] = {x, y, z, vx, vy, vz, fx, fy, fz, q, fpx, fpy, fpz};
  int* const pi[6] = {type, gid, orig, img[0], img[1], img[2]};
  unsigned long long* const pu[2] = {key_a, key_b};
  for (int k = 0; k < 13; ++k) {
    a.src_f64[k] = to_shadow ? pd[k] : shd[k];
    a.dst_f64[k] = to_shadow ? shd[k] : pd[k];
  }
  a.nf64 = 13;
  if (!to_shadow) {  // positions at the rebuild, for the skin check
    double* const p0[3] = {x0, y0, z0};
    for (int k = 0; k < 3; ++k) {
      a.src_f64[13 + k] = shd[k];
      a.dst_f64[13 + k] = p0[k];
    }
    a.nf64 = 16;
  }
  for (int k = 0; k < 6; ++k) {
    a.src_i32[k] = to_shadow ? pi[k] : shi[k];
    a.dst_i32[k] = to_shadow ? shi[k] : pi[k];
  }
  a.ni32 = 6;
  for (int k = 0; k < 2; ++k) {
    a.src_u64[k] = to_shadow ? pu[k] : shu[k];
    a.dst_u64[k] = to_shadow ? shu[k] : pu[k];
  }
  a.nu64 = 2;
  return a;
}

// The integration state and the arrays a rebuild permutes, copied to the
// saved set (save) or back from it.
ArraySet rbx_engine::state_set(bool save) const {
  ArraySet a{};
  double* const pd[10] = {x, y, z, vx, vy, vz, fx, fy, fz, q};
  int* const pi[6] = {type, gid, orig, img[0], img[1], img[2]};
  unsigned long long* const pu[2] = {key_a, key_b};
  for (int k = 0; k < 10; ++k) {
    a.src_f64[k] = save ? pd[k] : snapd[k];
    a.dst_f64[k] = save ? snapd[k] : pd[k];
  }
  for (int k = 0; k < 6; ++k) {
    a.src_i32[k] = save ? pi[k] : snapi[k];
    a.dst_i32[k] = save ? snapi[k] : pi[k];
  }
  for (int k = 0; k < 2; ++k) {
    a.src_u64[k] = save ? pu[k] : snapu[k];
    a.dst_u64[k] = save ? snapu[k] : pu[k];
  }
  a.nf64 = 10;
  a.ni32 = 6;
  a.nu64 = 2;
  return a;
}

// The device work of a rebuild on stream s: cell sort, permutation of every
// per-atom array (addresses unchanged), fixed-point records, candidate list.
// in_graph: also the candidate total and the device rebuild counter, with no
// host decision (the host checks the flags after the graph has run).
int rbx_engine::rebuild_launches(cudaStream_t s, bool in_graph) {
  // the cell sort's first kernel clears the cell-sort status, the list
  // overflow and the candidate total (and counts a rebuild inside a graph);
  // the list builder sums the candidates
  const RebuildBook book{dflags, (long long*)cand_total, in_graph ? dflags + 5 : nullptr};
  ETRY(launch_cells_sort(dbox, dims, n, x, y, z, perm, cell_of_sorted, cell_start, cell_scratch,
                         dflags, s, &book));
  ETRY(launch_move_set(n, perm, permute_set(true), s));
  ETRY(launch_move_set(n, nullptr, permute_set(false), s));
  if (where) ETRY(launch_inverse_perm(n, orig, where, s));  // SHAKE / special rows
  ETRY(launch_to_fixed(dbox, n, x, y, z, q, atoms, s));
  ETRY(launch_full_list(dbox, dims, prm.cut_off + prm.skin, n, x, y, z, cell_start, cap,
                        cand_count, cand, dflags + 1, list_scratch, s, far_split(),
                        (long long*)cand_total));
  return RBX_OK;
}

// Rebuild: cell sort, permute every per-atom array, candidate list; the row
// capacity grows (and the list is built again) until no row overflows.
int rbx_engine::rebuild() {
  ETRY(rebuild_launches(st, false));
  for (int attempt = 0; attempt < 4; ++attempt) {
    int h[2] = {0, 0};
    ETRY(cuda_ok(cudaMemcpyAsync(h, dflags, sizeof(int) * 2, cudaMemcpyDeviceToHost, st), "D2H"));
    ETRY(cuda_ok(cudaStreamSynchronize(st), "rebuild sync"));
    if (h[0]) {
      set_error("cell sort: a cell holds more than 2048 atoms");
      return RBX_ERR_CAPACITY;
    }
    if (!(h[1] & 1)) {
      have_cache = true;
      ++rebuilds;
      return RBX_OK;
    }
    // grow the row capacity and build the list again
    int maxc = 0;
    {
      std::vector<int> hc(n);
      ETRY(cuda_ok(cudaMemcpy(hc.data(), cand_count, sizeof(int) * n, cudaMemcpyDeviceToHost),
                   "D2H"));
      for (int v : hc) maxc = std::max(maxc, v);
    }
    release(cand);
    cap = ((int)(maxc * 1.2) + 31) / 32 * 32;
    ETRY(alloc(&cand, (size_t)n * cap));
    nrbl = rbl_fused_grid(prm.precision == RBX_MIXED, pp.freq, n, cap, nfpart, tun.rbl_waves,
                          prm.ntypes);
    graph_dirty = host_graph_dirty = true;  // the list moved
    ++graph_version;
    ETRY(launch_fill_i32(1, dflags + 1, 0, st));
    ETRY(launch_zero_u64((unsigned long long*)cand_total, st));
    ETRY(launch_full_list(dbox, dims, prm.cut_off + prm.skin, n, x, y, z, cell_start, cap,
                          cand_count, cand, dflags + 1, list_scratch, st, far_split(),
                          (long long*)cand_total));
  }
  set_error("candidate list capacity did not converge");
  return RBX_ERR_CAPACITY;
}

int rbx_engine::check_rebuild(bool disp_from_drift) {
  if (!have_cache || prm.skin <= 0.0) return rebuild();
  if (!disp_from_drift) {
    ETRY(cuda_ok(cudaMemsetAsync(max_d2, 0, sizeof(unsigned long long), st), "memset"));
    ETRY(launch_max_disp(dbox, n, x, y, z, x0, y0, z0, max_d2, st));
  }
  ETRY(cuda_ok(cudaMemcpyAsync(h_pinned, max_d2, sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, st),
               "D2H"));
  ETRY(cuda_ok(cudaStreamSynchronize(st), "skin check sync"));
  double d2;
  memcpy(&d2, h_pinned, sizeof(double));
  const double thr = prm.skin * 0.5;
  if (d2 > thr * thr) return rebuild();
  return RBX_OK;
}

int rbx_engine::real_space(const int* epoch_dev) {
  const bool mixed = prm.precision == RBX_MIXED;
  if (prm.neighbor_type == RBX_NEIGHBOR_RBL) {
    ETRY(launch_rbl_fused(mixed, pp, n, atoms, x, y, z, q, type, key_a, key_b, epoch, epoch_dev,
                          rows(), fpx, fpy, fpz, fpart, nrbl, st));
    if (!spec_natoms) return RBX_OK;
    return launch_special_rbl(pp, spec_natoms, spec_atoms, spec_cnt, spec_part, spec_max,
                              spec_w[0], spec_w[1], spec_w[2], where, x, y, z, q, type, key_a,
                              key_b, epoch, epoch_dev, fpx, fpy, fpz, fpart + (size_t)nrbl * 3, st);
  }
  if (sog_pair) {
    if (mixed)
      return launch_verlet_sog_mixed(sogp, pp.sf, n, atoms, type, cand_count, cand, cap, fpx, fpy,
                                     fpz, st);
    return launch_verlet_sog(sogp, n, x, y, z, q, type, cand_count, cand, cap, fpx, fpy, fpz,
                             nullptr, st);
  }
  return launch_verlet_fused_f64(pp, n, atoms, x, y, z, q, type, rows(), fpx, fpy,
                                 fpz, nullptr, epart, verlet_blocks(), st);
}

int rbx_engine::kspace_and_combine(bool kick, const int* epoch_dev) {
  ETRY(kspace_rho(st, epoch_dev));
  return kspace_finish(kick, epoch_dev);
}

int rbx_engine::kspace_rho(cudaStream_t s, const int* epoch_dev) {
  const bool mixed = prm.precision == RBX_MIXED;
  if (P > 0) {
    // a failed draw raises dflags[2] until check_sampler reads it; RBE samples
    // are drawn inside the structure-factor kernel (no launch of their own)
    const SampleArgs sa = make_sample_args(sample_tables, tcnt, ttot, prm.random_seed, epoch,
                                           epoch_dev, mx, my, mz, mixed ? mi : nullptr,
                                           dflags + 2);
    const bool draw_in_rho = !k_injected && !sog && n > 0;
    if (!k_injected && sog)
      ETRY(launch_rbsog_sample(P, sog_tables, prm.random_seed, (uint64_t)(int64_t)epoch,
                               epoch_dev, mx, my, mz, mixed ? mi : nullptr, dflags + 2, s));
    else if (!k_injected && !draw_in_rho)
      ETRY(launch_rbe_sample(P, sample_tables, tcnt, ttot, prm.random_seed, epoch, epoch_dev,
                             mx, my, mz, mixed ? mi : nullptr, dflags + 2, s));
    if (mixed)
      ETRY(launch_rbe_rho_partial_mixed(n, Pk, mi, atoms, part_re, part_im, nparts, s,
                                        tun.rho_kpt, draw_in_rho ? &sa : nullptr));
    else
      ETRY(launch_rbe_rho_partial_f64(dbox, n, Pk, mx, my, mz, q, x, y, z, part_re, part_im,
                                      nparts, s, tun.rho_kpt, draw_in_rho ? &sa : nullptr));
    // the RBSOG virial's gather chain reads only the samples
    if (sog)
      ETRY(launch_rbsog_npt_chain(dbox, P, mx, my, mz, sog_gauss, prm.random_seed,
                                  (uint64_t)(int64_t)epoch, epoch_dev, sog_idx, sog_mult, s));
  }
  return RBX_OK;
}

int rbx_engine::kspace_finish(bool kick, const int* epoch_dev) {
  const bool mixed = prm.precision == RBX_MIXED;
  const bool rbl = prm.neighbor_type == RBX_NEIGHBOR_RBL;
  const int mean_parts = rbl ? nrbl + (spec_natoms ? SPEC_PARTS : 0) : 0;
  if (sog) {
    const SogVirial sv{P, sog_mult, sog_wv, kterm + 2 * (size_t)Pk, virk};
    ETRY(launch_rbsog_finalize(dbox, Pk, nparts, part_re, part_im, mx, my, mz, sog_w, rho_re,
                               rho_im, tab, kterm, -sog_self * qsq * prm.qqr2e, ek, mean_parts,
                               fpart, n, rbl ? mean : nullptr, st, &sv));
  } else
    ETRY(launch_rbe_finalize(dbox, P, P > 0 ? nparts : 0, part_re, part_im, mx, my, mz,
                             prm.alpha, S, prm.qqr2e, qsq, qsum, P > 0 ? rho_re : nullptr,
                             rho_im, P > 0 ? ek : nullptr, virk, P > 0 ? tab : nullptr,
                             mean_parts, fpart, n, rbl ? mean : nullptr, kterm, st,
                             (unsigned*)(dflags + 9)));
  RbeForceOut o;
  o.f_pair_x = fpx;
  o.f_pair_y = fpy;
  o.f_pair_z = fpz;
  o.mean = rbl ? mean : nullptr;
  o.f_out_x = fx;
  o.f_out_y = fy;
  o.f_out_z = fz;
  if (keep_parts) {
    o.fk_x = fkx;
    o.fk_y = fky;
    o.fk_z = fkz;
  }
  if (kick) {
    o.vx = vx;
    o.vy = vy;
    o.vz = vz;
    o.type = type;
    o.inv_mass = inv_mass;
    o.half_dt = 0.5 * prm.dt;
  }
  if (mixed)
    ETRY(launch_rbe_force_mixed(n, Pk, tab, atoms, o, st, tun.frc_block));
  else
    ETRY(launch_rbe_force_f64(n, Pk, tab, q, x, y, z, o, st, tun.frc_block));
  return RBX_OK;
}

// ---------------------------------------------------------------------------
// Autotuner: candidate launch shapes timed on the current state with CUDA
// events on the engine's stream; the choice is cached per size bin.
// ---------------------------------------------------------------------------
namespace {
struct TuneKey {
  int nbin, kbin, precision, neighbor, coulomb, sms;
  bool operator<(const TuneKey& o) const {
    return std::tie(nbin, kbin, precision, neighbor, coulomb, sms) <
           std::tie(o.nbin, o.kbin, o.precision, o.neighbor, o.coulomb, o.sms);
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, rbx_engine::Tuning> g_tune_cache;

int half_octave(int v) { return v > 0 ? (int)std::lround(2.0 * std::log2((double)v)) : -1; }
}  // namespace

int rbx_engine::apply_tuning(const Tuning& t) {
  tun = t;
  if (P > 0) nparts = t.rho_parts > 0 ? std::min(t.rho_parts, nparts_cap) : rbe_partial_blocks(n);
  if (prm.neighbor_type == RBX_NEIGHBOR_RBL)
    nrbl = rbl_fused_grid(prm.precision == RBX_MIXED, pp.freq, n, cap, nfpart, tun.rbl_waves,
                          prm.ntypes);
  graph_dirty = host_graph_dirty = true;
  ++graph_version;
  return RBX_OK;
}

int rbx_engine::autotune(bool force, rbx_tuning* out) {
  cudaSetDevice(device);
  const TuneKey key{half_octave(n), half_octave(Pk), prm.precision, prm.neighbor_type,
                    prm.coulomb_type, sm_count()};
  rbx_tuning info{};
  if (!force) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      ETRY(apply_tuning(it->second));
      info.cache_hit = 1;
    }
  }
  if (!info.cache_hit) {
    if (!have_cache) ETRY(compute_forces(epoch));
    const bool mixed = prm.precision == RBX_MIXED;
    cudaEvent_t e0, e1;
    ETRY(cuda_ok(cudaEventCreate(&e0), "cudaEventCreate"));
    ETRY(cuda_ok(cudaEventCreate(&e1), "cudaEventCreate"));
    constexpr int kReps = 10;
    constexpr float kMargin = 0.97f;  // a candidate must beat the default by 3 %
    // mean device time per launch of fn (2 untimed launches first)
    auto time_it = [&](auto&& fn, float* ms) -> int {
      for (int r = 0; r < 2; ++r) ETRY(fn());
      ETRY(cuda_ok(cudaEventRecord(e0, st), "cudaEventRecord"));
      for (int r = 0; r < kReps; ++r) ETRY(fn());
      ETRY(cuda_ok(cudaEventRecord(e1, st), "cudaEventRecord"));
      ETRY(cuda_ok(cudaEventSynchronize(e1), "cudaEventSynchronize"));
      float t = 0.f;
      ETRY(cuda_ok(cudaEventElapsedTime(&t, e0, e1), "cudaEventElapsedTime"));
      *ms = t / kReps;
      return RBX_OK;
    };
    Tuning best = tun;
    int rc = RBX_OK;
    // the fastest candidate, unless the built-in shape is within the margin
    struct Cand {
      int a, b;
      float ms;
    };
    auto pick = [&](const std::vector<Cand>& c, int def_a, int def_b, float* def_ms) {
      Cand best_c = c.front();
      *def_ms = 0.f;
      for (const Cand& k : c) {
        if (k.ms < best_c.ms) best_c = k;
        if (k.a == def_a && k.b == def_b) *def_ms = k.ms;
      }
      if (*def_ms > 0.f && !(best_c.ms < kMargin * *def_ms)) return Cand{def_a, def_b, *def_ms};
      return best_c;
    };
    if (P > 0) {
      // rho(k): k-vectors per thread x atom blocks
      std::vector<Cand> c;
      const int sm = sm_count(), def_parts = rbe_partial_blocks(n);
      std::vector<int> parts_list = {def_parts};
      for (int mult : {1, 2, 4, 8}) {
        const int parts = std::min(std::min(mult * sm, nparts_cap), std::max(1, (n + 31) / 32));
        if (std::find(parts_list.begin(), parts_list.end(), parts) == parts_list.end())
          parts_list.push_back(parts);
      }
      for (int parts : parts_list)
        for (int kpt : {1, 2, 4, 8}) {
          float ms = 0.f;
          rc = time_it(
              [&]() {
                return mixed ? launch_rbe_rho_partial_mixed(n, Pk, mi, atoms, part_re, part_im,
                                                            parts, st, kpt)
                             : launch_rbe_rho_partial_f64(dbox, n, Pk, mx, my, mz, q, x, y, z,
                                                          part_re, part_im, parts, st, kpt);
              },
              &ms);
          if (rc) break;
          c.push_back({kpt, parts, ms});
        }
      if (!rc) {
        const Cand r = pick(c, 4, def_parts, &info.rho_ms_default);
        best.rho_kpt = r.a;
        best.rho_parts = r.b;
        info.rho_ms = r.ms;
      }
      // force scatter (the table of the last evaluation; output to the k-space scratch)
      RbeForceOut o;
      o.f_out_x = fkx;
      o.f_out_y = fky;
      o.f_out_z = fkz;
      c.clear();
      for (int blk : {128, 256, 512}) {
        if (rc) break;
        float ms = 0.f;
        rc = time_it(
            [&]() {
              return mixed ? launch_rbe_force_mixed(n, Pk, tab, atoms, o, st, blk)
                           : launch_rbe_force_f64(n, Pk, tab, q, x, y, z, o, st, blk);
            },
            &ms);
        c.push_back({blk, 0, ms});
      }
      if (!rc) {
        const Cand r = pick(c, 256, 0, &info.force_ms_default);
        best.frc_block = r.a;
        info.force_ms = r.ms;
      }
    }
    if (!rc && prm.neighbor_type == RBX_NEIGHBOR_RBL) {
      std::vector<Cand> c;
      for (int waves : {2, 4, 8, 16}) {
        const int nb = rbl_fused_grid(mixed, pp.freq, n, cap, nfpart, waves, prm.ntypes);
        float ms = 0.f;
        rc = time_it(
            [&]() {
              return launch_rbl_fused(mixed, pp, n, atoms, x, y, z, q, type, key_a, key_b, epoch,
                                      nullptr, rows(), fpx, fpy, fpz, fpart, nb, st);
            },
            &ms);
        if (rc) break;
        c.push_back({waves, 0, ms});
      }
      if (!rc) {
        const Cand r = pick(c, 8, 0, &info.rbl_ms_default);
        best.rbl_waves = r.a;
        info.rbl_ms = r.ms;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ETRY(rc);
    ETRY(apply_tuning(best));
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      g_tune_cache[key] = best;
    }
    ETRY(compute_forces(epoch));  // forces of the current state with the chosen shapes
  }
  if (out) {
    out->rho_kpt = tun.rho_kpt;
    out->rho_blocks = nparts;
    out->force_block = tun.frc_block;
    out->rbl_waves = tun.rbl_waves;
    out->cache_hit = info.cache_hit;
    out->rho_ms = info.rho_ms;
    out->force_ms = info.force_ms;
    out->rbl_ms = info.rbl_ms;
    out->rho_ms_default = info.rho_ms_default;
    out->force_ms_default = info.force_ms_default;
    out->rbl_ms_default = info.rbl_ms_default;
  }
  return RBX_OK;
}

// RBSOG k-space (per-k weights, the |m| = 1 vectors after the P samples, the
// mixture sampler's tables) and the VERLET-SOG pair parameters; see rbx_rbsog.cu.
int rbx_engine::init_rbsog() {
  rbx_host::RbsogSetup s;
  try {
    s = rbx_host::rbsog_setup(prm.rbsog_level, prm.cut_off, box);
  } catch (const std::exception& ex) {
    set_error("%s", ex.what());
    return RBX_ERR_CONFIG;
  }
  if (sog_pair) {
    sogp.box = dbox;
    sogp.cut_off = prm.cut_off;
    sogp.qqr2e = prm.qqr2e;
    sogp.ntypes = prm.ntypes;
    sogp.lj_eps = lj_eps;
    sogp.lj_s6 = lj_s6;
    for (int i = 0; i < 6; ++i) sogp.taylor[i] = s.taylor[i];
    sogp.sigma = s.sigma;
    sogp.b = s.b;
    sogp.w0 = s.w0;
    sogp.norm = 2.0 * log(s.b) / sqrt(2.0 * M_PI * s.sigma * s.sigma);
    sogp.mmax = s.mmax;
  }
  if (!sog) return RBX_OK;
  S = prm.rbsog_S > 0 ? prm.rbsog_S : (prm.rbsog_S < 0 ? s.S_full : s.S);
  sog_self = s.self_coeff;
  const double V = dbox.len[0] * dbox.len[1] * dbox.len[2], qe = prm.qqr2e;
  std::vector<double4> w(Pk);
  for (int k = 0; k < P; ++k) w[k] = make_double4(-S * qe / P, 0.0, S * qe / (2.0 * P * V), 0.0);
  std::vector<double> dm[3];
  std::vector<int> dmi;
  for (int k = 0; k < 6; ++k) {
    w[P + k] = make_double4(0.0, -qe * s.direct_fb[k], 0.0, qe * s.direct_fb[k] / (2.0 * V));
    for (int d = 0; d < 3; ++d) {
      dm[d].push_back(s.direct_m[3 * k + d]);
      dmi.push_back(s.direct_m[3 * k + d]);
    }
  }
  // NPT weights of the virial: sampled -S_npt qqr2e / (4 P V) (times the
  // chain's multiplicity / |k|^4), direct -qqr2e G_npt(k) / (4 V)
  std::vector<double> wv(Pk);
  for (int k = 0; k < P; ++k) wv[k] = -s.S_npt * qe / (4.0 * P * V);
  for (int k = 0; k < 6; ++k) wv[P + k] = -qe * s.direct_fb_npt[k] / (4.0 * V);
  ETRY(alloc(&sog_wv, (size_t)Pk));
  ETRY(alloc(&sog_coef, (size_t)s.mmax));
  ETRY(alloc(&sog_coef_npt, (size_t)s.mmax));
  ETRY(alloc(&sog_idx, (size_t)(P > 0 ? P : 1)));
  ETRY(alloc(&sog_mult, (size_t)(P > 0 ? P : 1)));
  ETRY(alloc(&sog_w, (size_t)Pk));
  ETRY(alloc(&sog_cdf, s.comp_cdf.size()));
  ETRY(alloc(&sog_tab, s.tables.size()));
  ETRY(alloc(&sog_tot, s.tab_tot.size()));
  ETRY(alloc(&sog_off, s.tab_off.size()));
  ETRY(alloc(&sog_cnt, s.tab_cnt.size()));
  auto up = [&](void* dst, const void* src, size_t bytes) {
    return cuda_ok(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice), "H2D");
  };
  ETRY(up(sog_w, w.data(), sizeof(double4) * Pk));
  ETRY(up(sog_wv, wv.data(), sizeof(double) * Pk));
  ETRY(up(sog_coef, s.coef.data(), sizeof(double) * s.mmax));
  ETRY(up(sog_coef_npt, s.coef_npt.data(), sizeof(double) * s.mmax));
  sog_gauss = SogGauss{sog_coef, sog_coef_npt, s.mmax, s.b * s.b, s.sigma * s.sigma};
  ETRY(up(sog_cdf, s.comp_cdf.data(), sizeof(double) * s.comp_cdf.size()));
  ETRY(up(sog_tab, s.tables.data(), sizeof(double) * s.tables.size()));
  ETRY(up(sog_tot, s.tab_tot.data(), sizeof(double) * s.tab_tot.size()));
  ETRY(up(sog_off, s.tab_off.data(), sizeof(int) * s.tab_off.size()));
  ETRY(up(sog_cnt, s.tab_cnt.data(), sizeof(int) * s.tab_cnt.size()));
  ETRY(up(mx + P, dm[0].data(), sizeof(double) * 6));
  ETRY(up(my + P, dm[1].data(), sizeof(double) * 6));
  ETRY(up(mz + P, dm[2].data(), sizeof(double) * 6));
  ETRY(up(mi + 3 * P, dmi.data(), sizeof(int) * 18));
  ETRY(cuda_ok(cudaMemset(virk, 0, sizeof(double) * 6), "memset"));
  sog_tables = RbsogTables{sog_cdf, (int)s.comp_cdf.size(), s.comp_cdf.back(), sog_tab, sog_off,
                           sog_cnt, sog_tot};
  return RBX_OK;
}

int rbx_engine::compute_forces(int ep) {
  cudaSetDevice(device);
  epoch = ep;
  ETRY(check_rebuild(false));
  ETRY(launch_to_fixed(dbox, n, x, y, z, q, atoms, st));
  ETRY(real_space());
  ETRY(kspace_and_combine(false));
  ETRY(cuda_ok(cudaStreamSynchronize(st), "compute_forces sync"));
  ETRY(check_sampler());
  have_forces = true;
  ++force_calls;
  return RBX_OK;
}

// Device status words raised during the last steps: [2] k-sampler, [3] real-space kernel.
int rbx_engine::check_sampler() {
  int h[2] = {0, 0};
  ETRY(cuda_ok(cudaMemcpy(h, dflags + 2, sizeof(int) * 2, cudaMemcpyDeviceToHost), "D2H"));
  if (h[1]) {
    set_error("real-space kernel: a candidate-row copy did not complete (status %d)", h[1]);
    return RBX_ERR_CUDA;
  }
  if (h[0]) {
    ETRY(cuda_ok(cudaMemset(dflags + 2, 0, sizeof(int)), "memset"));  // reported once
    if (P > 0 && !k_injected) {
      set_error("k-sampler: a sample needed more than 64 draws to avoid m = 0");
      return RBX_ERR_SAMPLER;
    }
  }
  return RBX_OK;
}

int rbx_engine::step(int nsteps) {
  cudaSetDevice(device);
  if (!have_forces) ETRY(compute_forces(epoch));
  if (nsteps <= 0) return RBX_OK;
  // profiled steps time their phases with events between launches: no graph
  if (use_graph && !profiling && have_cache && prm.skin > 0.0) return step_graph(nsteps);
  return step_plain(nsteps);
}

// One velocity-Verlet step after another, the host deciding each rebuild.
int rbx_engine::step_plain(int nsteps) {
  for (int s = 0; s < nsteps; ++s) {
    cudaEvent_t* e = nullptr;
    if (profiling) {
      if ((size_t)pev_used + 5 > pev.size()) ETRY(flush_profile());
      while ((size_t)pev_used + 5 > pev.size()) {
        cudaEvent_t t;
        ETRY(cuda_ok(cudaEventCreate(&t), "cudaEventCreate"));
        pev.push_back(t);
      }
      e = &pev[pev_used];
      pev_used += 5;
      cudaEventRecord(e[0], st);
    }
    if (nh_on) ETRY(nh_initial(nullptr, epoch + 1, st));
    ETRY(cuda_ok(cudaMemsetAsync(max_d2, 0, sizeof(unsigned long long), st), "memset"));
    const KickArgs kick{fx, fy, fz, type, inv_mass, 0.5 * prm.dt};
    ETRY(launch_drift(dbox, n, prm.dt, x, y, z, vx, vy, vz, x0, y0, z0, max_d2, atoms, q,
                     ImageRefs{{img[0], img[1], img[2]}}, Pos3{shake_nc ? xs : nullptr, ys, zs},
                     st, &kick));
    if (shake_nc) ETRY(shake_a(st));
    if (e) cudaEventRecord(e[1], st);
    ++epoch;
    ETRY(check_rebuild(true));
    if (e) cudaEventRecord(e[2], st);
    ETRY(real_space());
    if (e) cudaEventRecord(e[3], st);
    ETRY(kspace_and_combine(true));
    if (shake_nc) ETRY(shake_b(st));
    if (nh_on) ETRY(nh_final(st));
    if (e) cudaEventRecord(e[4], st);
    ++steps;
    ++force_calls;
  }
  ETRY(cuda_ok(cudaStreamSynchronize(st), "step sync"));
  if (profiling) ETRY(flush_profile());
  ETRY(check_sampler());
  return RBX_OK;
}

// Capture one MD step as a CUDA graph: kick, drift, the rebuild decision (a
// one-thread kernel that advances the device epoch and sets the condition),
// an IF node whose body is the rebuild, then the real-space force, k-space and
// the second half kick.  Nothing in it waits for the host.
int rbx_engine::capture_step_graph() {
  release_graph();
  ETRY(cuda_ok(cudaGraphCreate(&graph, 0), "cudaGraphCreate"));
  ETRY(cuda_ok(cudaStreamBeginCaptureToGraph(st, graph, nullptr, nullptr, 0,
                                             cudaStreamCaptureModeThreadLocal),
               "cudaStreamBeginCaptureToGraph"));
  const int rc = capture_step_into(graph);
  cudaGraph_t g = graph;
  const cudaError_t e = cudaStreamEndCapture(st, &g);
  if (rc) {
    release_graph();
    return rc;
  }
  ETRY(cuda_ok(e, "cudaStreamEndCapture"));
  ETRY(cuda_ok(cudaGraphInstantiate(&graph_exec, graph, 0), "cudaGraphInstantiate"));
  graph_dirty = false;
  return RBX_OK;
}

// Record one MD step on st, which must be capturing into g (its own graph or
// a batch graph): the conditional handle is created on g, the IF node goes
// after what st has captured so far, its body is captured on st_body.
int rbx_engine::capture_step_into(cudaGraph_t g, bool fork_kspace) {
  const unsigned long long l0 = rbx_launch_count();
  cudaGraphConditionalHandle cond;
  ETRY(cuda_ok(cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault),
               "cudaGraphConditionalHandleCreate"));
  bool decided = false;
  ETRY(capture_step_head(&cond, &decided));
  ETRY(capture_step_tail(g, &cond, decided, fork_kspace));
  graph_step_launches = rbx_launch_count() - l0 - graph_rebuild_launches;
  return RBX_OK;
}

// First part of a step: half kick, drift with the skin check (+ SHAKE).
// Without SHAKE (which moves atoms after the drift) the drift kernel takes the
// rebuild decision when given the step's conditional handle; max_d2 and its
// block counter are then cleared by the kernel itself after each decision
// (and by graph_run_begin before the first step).
int rbx_engine::capture_step_head(const cudaGraphConditionalHandle* cond, bool* decided) {
  if (nh_on) ETRY(nh_initial(dflags + 4, 1, st));  // the device epoch is still the last step's
  const bool fold = cond && !shake_nc && n > 0;
  if (!fold) ETRY(launch_zero_u64(max_d2, st));
  const KickArgs kick{fx, fy, fz, type, inv_mass, 0.5 * prm.dt};
  const double thr = prm.skin * 0.5;
  const DecideArgs dec{(unsigned*)(dflags + 8), thr * thr, dflags + 4, fold ? *cond : 0};
  ETRY(launch_drift(dbox, n, prm.dt, x, y, z, vx, vy, vz, x0, y0, z0, max_d2, atoms, q,
                     ImageRefs{{img[0], img[1], img[2]}}, Pos3{shake_nc ? xs : nullptr, ys, zs},
                     st, &kick, fold ? &dec : nullptr));
  if (shake_nc) ETRY(shake_a(st));
  if (decided) *decided = fold;
  return RBX_OK;
}

// Rest of a step, captured on st into g: rebuild decision and the rebuild
// under an IF node, forces, second half kick (+ RATTLE, thermostat).
int rbx_engine::capture_step_tail(cudaGraph_t g, const cudaGraphConditionalHandle* cond_in,
                                  bool decided, bool fork_kspace) {
  cudaGraphConditionalHandle cond;
  if (cond_in) {
    cond = *cond_in;
  } else {
    ETRY(cuda_ok(cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault),
                 "cudaGraphConditionalHandleCreate"));
  }
  const double thr = prm.skin * 0.5;
  if (!decided) ETRY(launch_step_decide(max_d2, thr * thr, dflags + 4, cond, st));
  // the conditional node after everything captured so far on st
  cudaStreamCaptureStatus cs;
  cudaGraph_t capg = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  ETRY(cuda_ok(cudaStreamGetCaptureInfo(st, &cs, nullptr, &capg, &deps, &ndeps),
               "cudaStreamGetCaptureInfo"));
  cudaGraphNodeParams np{};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = cond;
  np.conditional.type = cudaGraphCondTypeIf;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  ETRY(cuda_ok(cudaGraphAddNode(&node, capg, deps, ndeps, &np), "cudaGraphAddNode"));
  cudaGraph_t body = np.conditional.phGraph_out[0];
  ETRY(cuda_ok(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies),
               "cudaStreamUpdateCaptureDependencies"));
  ETRY(capture_rebuild_body(body));
  if (fork_kspace) {
    // the k-sampling and the structure factor read only the positions (after
    // the rebuild's reordering): a branch beside the real-space force, joined
    // before the finalize, which needs both
    ETRY(cuda_ok(cudaEventRecord(ev_ks[0], st), "cudaEventRecord"));
    ETRY(cuda_ok(cudaStreamWaitEvent(st_ks, ev_ks[0], 0), "cudaStreamWaitEvent"));
    ETRY(kspace_rho(st_ks, dflags + 4));
    ETRY(cuda_ok(cudaEventRecord(ev_ks[1], st_ks), "cudaEventRecord"));
    ETRY(real_space(dflags + 4));
    ETRY(cuda_ok(cudaStreamWaitEvent(st, ev_ks[1], 0), "cudaStreamWaitEvent"));
    ETRY(kspace_finish(true, dflags + 4));
  } else {
    ETRY(real_space(dflags + 4));
    ETRY(kspace_and_combine(true, dflags + 4));
  }
  if (shake_nc) ETRY(shake_b(st));
  if (nh_on) ETRY(nh_final(st));
  return RBX_OK;
}

int rbx_engine::capture_rebuild_body(cudaGraph_t body) {
  const unsigned long long b0 = rbx_launch_count();
  ETRY(cuda_ok(cudaStreamBeginCaptureToGraph(st_body, body, nullptr, nullptr, 0,
                                             cudaStreamCaptureModeThreadLocal),
               "cudaStreamBeginCaptureToGraph"));
  const int brc = rebuild_launches(st_body, true);
  cudaGraph_t body_out = body;
  const cudaError_t be = cudaStreamEndCapture(st_body, &body_out);
  ETRY(brc);
  ETRY(cuda_ok(be, "cudaStreamEndCapture (rebuild body)"));
  graph_rebuild_launches = rbx_launch_count() - b0;
  return RBX_OK;
}

// The launchers record instead of launching while rec is installed; the
// recording runs inside a capture of st into a graph that is thrown away, so
// a launch without a batched form (counted by rbx_launch_count) never runs.
int rbx_engine::record_phased_step(BatchRecorder* rec, cudaGraphConditionalHandle cond) {
  const bool ok = prm.neighbor_type == RBX_NEIGHBOR_RBL && prm.precision == RBX_MIXED && !sog &&
                  !sog_pair && !shake_nc && !nh_on && !spec_natoms && n > 0 && P > 0 &&
                  !profiling;
  if (!ok) {
    set_error("phase-batched step: needs an RBL engine in the mixed form with RBE k-space, "
              "NVE, no SHAKE and no special bonds");
    return RBX_ERR_INVALID;
  }
  ETRY(cuda_ok(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal),
               "cudaStreamBeginCapture"));
  batch_recorder() = rec;
  const unsigned long long l0 = rbx_launch_count();
  bool decided = false;
  int rc = capture_step_head(&cond, &decided);
  if (!rc) rc = real_space(dflags + 4);
  if (!rc) rc = kspace_and_combine(true, dflags + 4);
  batch_recorder() = nullptr;
  const bool foreign = rbx_launch_count() != l0;
  cudaGraph_t scratch = nullptr;
  const cudaError_t e = cudaStreamEndCapture(st, &scratch);
  if (scratch) cudaGraphDestroy(scratch);
  ETRY(rc);
  ETRY(cuda_ok(e, "cudaStreamEndCapture (phase recording)"));
  if (foreign || !decided) {
    set_error("phase-batched step: a kernel of the step has no batched form");
    return RBX_ERR_INVALID;
  }
  return RBX_OK;
}

// The two graphs of a host-buffer step (see hgraph).
int rbx_engine::capture_host_graphs() {
  release_host_graphs();
  const unsigned long long l0 = rbx_launch_count();
  for (int k = 0; k < 2; ++k) {
    ETRY(cuda_ok(cudaGraphCreate(&hgraph[k], 0), "cudaGraphCreate"));
    ETRY(cuda_ok(cudaStreamBeginCaptureToGraph(st, hgraph[k], nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal),
                 "cudaStreamBeginCaptureToGraph"));
    int rc;
    if (k == 0) {
      rc = capture_step_head();
      if (!rc) {  // positions, cell order -> host order, into stage[0, 3n)
        ArraySet out{};
        const double* src[] = {x, y, z};
        for (int a = 0; a < 3; ++a) {
          out.src_f64[a] = src[a];
          out.dst_f64[a] = stage + (size_t)a * n;
        }
        out.nf64 = 3;
        rc = launch_scatter_set(n, orig, out, st);
      }
    } else {
      rc = capture_step_tail(hgraph[k]);
    }
    cudaGraph_t gk = hgraph[k];
    const cudaError_t e = cudaStreamEndCapture(st, &gk);
    if (rc) {
      release_host_graphs();
      return rc;
    }
    ETRY(cuda_ok(e, "cudaStreamEndCapture"));
    ETRY(cuda_ok(cudaGraphInstantiate(&hexec[k], hgraph[k], 0), "cudaGraphInstantiate"));
  }
  host_step_launches = rbx_launch_count() - l0 - graph_rebuild_launches;
  host_graph_dirty = false;
  return RBX_OK;
}

// Before a run of graph steps: save the state, seed the device epoch and the
// in-graph rebuild counter (all on stream s).
int rbx_engine::graph_run_begin(cudaStream_t s) {
  ETRY(launch_move_set(n, nullptr, state_set(true), s));
  if (nh_on)
    ETRY(cuda_ok(cudaMemcpyAsync(nh_snap, nh_state, sizeof(double) * NH_SLOTS,
                                 cudaMemcpyDeviceToDevice, s),
                 "D2D"));
  run_init[0] = epoch;  // [4] epoch, [5] rebuilds inside the graph
  run_init[1] = 0;
  // the maximum displacement and the drift's block counter start from zero
  ETRY(cuda_ok(cudaMemsetAsync(max_d2, 0, sizeof(unsigned long long), s), "memset"));
  ETRY(cuda_ok(cudaMemsetAsync(dflags + 8, 0, sizeof(int), s), "memset"));
  return cuda_ok(cudaMemcpyAsync(dflags + 4, run_init, sizeof(int) * 2, cudaMemcpyHostToDevice, s),
                 "H2D");
}

// After the graph steps (flags copied to run_flags and the stream synchronised):
// account for the steps, or restore the saved state and replay them launch by
// launch when a rebuild inside the graph overflowed.
int rbx_engine::graph_run_end(int nsteps, unsigned long long step_launches) {
  const int* h = run_flags;
  if (h[0] || (h[1] & 1)) {
    ETRY(launch_move_set(n, nullptr, state_set(false), st));
    if (where) ETRY(launch_inverse_perm(n, orig, where, st));
    if (nh_on)
      ETRY(cuda_ok(cudaMemcpyAsync(nh_state, nh_snap, sizeof(double) * NH_SLOTS,
                                   cudaMemcpyDeviceToDevice, st),
                   "D2D"));
    have_cache = false;
    return step_plain(nsteps);
  }
  count_launch((int)(step_launches * nsteps + graph_rebuild_launches * h[5]));
  epoch += nsteps;
  steps += nsteps;
  force_calls += nsteps;
  rebuilds += h[5];
  return check_sampler();
}

// nsteps launches of the step graph with one host synchronisation at the
// end.  The state is saved first: if a rebuild inside the graph ran out of
// row capacity (or a cell overflowed the sort), the saved state comes back
// and the same steps run again with the host deciding each rebuild (which
// grows the capacity).
int rbx_engine::step_graph(int nsteps) {
  if (graph_dirty || !graph_exec) ETRY(capture_step_graph());
  ETRY(graph_run_begin(st));
  for (int k = 0; k < nsteps; ++k)
    ETRY(cuda_ok(cudaGraphLaunch(graph_exec, st), "cudaGraphLaunch"));
  ETRY(cuda_ok(cudaMemcpyAsync(run_flags, dflags, sizeof(int) * 6, cudaMemcpyDeviceToHost, st),
               "D2H"));
  ETRY(cuda_ok(cudaStreamSynchronize(st), "step graph sync"));
  return graph_run_end(nsteps, graph_step_launches);
}

// Fold the recorded per-step phase events into the running totals.
int rbx_engine::flush_profile() {
  ETRY(cuda_ok(cudaStreamSynchronize(st), "profile sync"));
  for (int b = 0; b + 5 <= pev_used; b += 5) {
    for (int k = 0; k < 4; ++k) {
      float v = 0.f;
      ETRY(cuda_ok(cudaEventElapsedTime(&v, pev[b + k], pev[b + k + 1]), "cudaEventElapsedTime"));
      phase_total[k] += v;
    }
    ++phase_steps;
  }
  pev_used = 0;
  return RBX_OK;
}

// Mean device time per profiled step and phase, in ms.
int rbx_engine::phase_ms(float out[4]) {
  if (phase_steps == 0) {
    set_error("no profiled steps (enable rbx_engine_set_profiling, then step)");
    return RBX_ERR_INVALID;
  }
  for (int k = 0; k < 4; ++k) out[k] = (float)(phase_total[k] / (double)phase_steps);
  return RBX_OK;
}

int rbx_engine::get_state(double* hx, double* hy, double* hz, double* hvx, double* hvy,
                          double* hvz, double* hfx, double* hfy, double* hfz) {
  cudaSetDevice(device);
  const double* src[] = {x, y, z, vx, vy, vz, fx, fy, fz};
  double* dst[] = {hx, hy, hz, hvx, hvy, hvz, hfx, hfy, hfz};
  for (int a = 0; a < 9; ++a) {
    if (!dst[a]) continue;
    ETRY(launch_scatter_f64(n, orig, src[a], stage + (size_t)a * n, st));
  }
  for (int a = 0; a < 9; ++a) {
    if (!dst[a]) continue;
    ETRY(cuda_ok(cudaMemcpyAsync(dst[a], stage + (size_t)a * n, sizeof(double) * n,
                                 cudaMemcpyDeviceToHost, st),
                 "D2H"));
  }
  return cuda_ok(cudaStreamSynchronize(st), "get_state sync");
}

int rbx_engine::step_host(const double* xin, const double* vin, double* xout, double* vout,
                          double* fout) {
  cudaSetDevice(device);
  const size_t N = (size_t)n;
  // x_in / v_in are [3][n] blocks (x,y,z then vx,vy,vz) in host order
  ETRY(cuda_ok(cudaMemcpyAsync(stage, xin, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, st),
               "H2D"));
  ETRY(cuda_ok(cudaMemcpyAsync(stage + 3 * N, vin, sizeof(double) * 3 * N, cudaMemcpyHostToDevice,
                               st),
               "H2D"));
  ArraySet in{};
  double* dst[] = {x, y, z, vx, vy, vz};
  for (int a = 0; a < 6; ++a) {
    in.src_f64[a] = stage + a * N;
    in.dst_f64[a] = dst[a];
  }
  in.nf64 = 6;
  ETRY(launch_move_set(n, orig, in, st));  // host order -> cell order
  // outputs from array `first` on (x y z vx vy vz fx fy fz): cell order ->
  // host order into stage, then the copies out, all queued on st
  double* const outs[3] = {xout, vout, fout};
  auto queue_out = [&](int first) -> int {
    ArraySet out{};
    const double* src[] = {x, y, z, vx, vy, vz, fx, fy, fz};
    for (int a = first; a < 9; ++a) {
      out.src_f64[a - first] = src[a];
      out.dst_f64[a - first] = stage + a * N;
    }
    out.nf64 = 9 - first;
    ETRY(launch_scatter_set(n, orig, out, st));
    for (int b = first / 3; b < 3; ++b)
      ETRY(cuda_ok(cudaMemcpyAsync(outs[b], stage + 3 * b * N, sizeof(double) * 3 * N,
                                   cudaMemcpyDeviceToHost, st),
                   "D2H"));
    return RBX_OK;
  };
  if (!have_forces) ETRY(compute_forces(epoch));
  if (use_graph && !profiling && have_cache && prm.skin > 0.0) {
    // two graph launches; the positions go out on st_side while the second
    // computes the forces; one host synchronisation
    if (host_graph_dirty || !hexec[0] || !hexec[1]) ETRY(capture_host_graphs());
    ETRY(graph_run_begin(st));
    int rc = cuda_ok(cudaGraphLaunch(hexec[0], st), "cudaGraphLaunch");
    if (!rc) rc = cuda_ok(cudaEventRecord(ev_side, st), "cudaEventRecord");
    if (!rc) rc = cuda_ok(cudaStreamWaitEvent(st_side, ev_side, 0), "cudaStreamWaitEvent");
    if (!rc)
      rc = cuda_ok(cudaMemcpyAsync(xout, stage, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost,
                                   st_side),
                   "D2H");
    if (!rc) rc = cuda_ok(cudaGraphLaunch(hexec[1], st), "cudaGraphLaunch");
    if (!rc)
      rc = cuda_ok(cudaMemcpyAsync(run_flags, dflags, sizeof(int) * 6, cudaMemcpyDeviceToHost, st),
                   "D2H");
    if (!rc) rc = queue_out(3);
    if (rc) {  // no copy into the caller's buffers may be left in flight
      cudaStreamSynchronize(st_side);
      cudaStreamSynchronize(st);
      return rc;
    }
    ETRY(cuda_ok(cudaStreamSynchronize(st_side), "step_host sync"));
    ETRY(cuda_ok(cudaStreamSynchronize(st), "step_host sync"));
    const bool replay = run_flags[0] || (run_flags[1] & 1);
    ETRY(graph_run_end(1, host_step_launches));  // on overflow: state restored, step replayed
    if (!replay) return RBX_OK;
  } else {
    ETRY(step(1));
  }
  const int rc = queue_out(0);
  if (rc) {
    cudaStreamSynchronize(st);
    return rc;
  }
  return cuda_ok(cudaStreamSynchronize(st), "step_host sync");
}

int rbx_engine::get_force_parts(double* f_pair, double* f_kspace) {
  cudaSetDevice(device);
  if (!keep_parts) {
    set_error("force parts are not kept; enable with rbx_engine_set_k_samples or a parity run");
    return RBX_ERR_INVALID;
  }
  const size_t N = (size_t)n;
  // pair part after mean removal: f_total - f_k
  const double* src[] = {fx, fy, fz, fkx, fky, fkz};
  for (int a = 0; a < 6; ++a) ETRY(launch_scatter_f64(n, orig, src[a], stage + a * N, st));
  std::vector<double> h(6 * N);
  ETRY(cuda_ok(cudaMemcpyAsync(h.data(), stage, sizeof(double) * 6 * N, cudaMemcpyDeviceToHost, st),
               "D2H"));
  ETRY(cuda_ok(cudaStreamSynchronize(st), "sync"));
  for (size_t i = 0; i < N; ++i)
    for (int d = 0; d < 3; ++d) {
      const double fk = h[(3 + d) * N + i];
      if (f_kspace) f_kspace[i * 3 + d] = fk;
      if (f_pair) f_pair[i * 3 + d] = h[d * N + i] - fk;
    }
  return RBX_OK;
}

// LJ and erfc-Coulomb energies and the virial over every pair within cut_off
// of the current positions: the Verlet kernel over the candidate rows (their
// forces go to scratch), per-block partials summed here in block order.  A
// Verlet-list engine whose forces are those of the current positions already
// holds the partials of that same kernel from its last force evaluation.
int rbx_engine::pair_energy(double* e_vdwl, double* e_coul, double* virial) {
  cudaSetDevice(device);
  if (prm.neighbor_type == RBX_NEIGHBOR_VERLET_SOG) {
    set_error("pair energy: the VERLET-SOG energies come from rbx_pair_force_verlet_sog");
    return RBX_ERR_INVALID;
  }
  const int nvb = verlet_blocks();
  if (!(prm.neighbor_type == RBX_NEIGHBOR_VERLET && have_forces)) {
    ETRY(check_rebuild(false));  // rows that hold every pair within cut_off
    ETRY(launch_to_fixed(dbox, n, x, y, z, q, atoms, st));
    const size_t N = (size_t)n;
    ETRY(launch_verlet_fused_f64(pp, n, atoms, x, y, z, q, type, rows(), stage,
                                 stage + N, stage + 2 * N, nullptr, epart, nvb, st));
  }
  std::vector<double> h((size_t)nvb * 8);
  ETRY(cuda_ok(cudaMemcpyAsync(h.data(), epart, sizeof(double) * h.size(), cudaMemcpyDeviceToHost,
                               st),
               "D2H"));
  ETRY(cuda_ok(cudaStreamSynchronize(st), "pair energy sync"));
  double t[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int b = 0; b < nvb; ++b)
    for (int k = 0; k < 8; ++k) t[k] += h[(size_t)b * 8 + k];
  if (e_vdwl) *e_vdwl = t[0];
  if (e_coul) *e_coul = t[1];
  if (virial)
    for (int k = 0; k < 6; ++k) virial[k] = t[2 + k];
  return RBX_OK;
}

// Exact Ewald reciprocal energy over the kmax box plus the self energy of the
// current positions (ComputeKspaceEnergy + ComputeSelfEnergy,
// kspace_calculator.cpp:630-645, 816-907): what RBMD reports on thermo steps
// when energy_rbe_flag is "yes".
int rbx_engine::kspace_energy_exact(const int kmax[3], double* energy) {
  cudaSetDevice(device);
  if (!kmax || kmax[0] < 0 || kmax[1] < 0 || kmax[2] < 0 || !energy) {
    set_error("kspace_energy_exact: invalid kmax or output");
    return RBX_ERR_INVALID;
  }
  const int nk = (2 * kmax[0] + 1) * (2 * kmax[1] + 1) * (2 * kmax[2] + 1) - 1;
  if (nk <= 0) {
    *energy = -prm.qqr2e * sqrt(prm.alpha / RBX_PI) * qsq;
    return RBX_OK;
  }
  double* buf = nullptr;  // re, im, k vectors, one energy
  if (cudaMallocAsync((void**)&buf, sizeof(double) * (5 * (size_t)nk + 1), st) != cudaSuccess) {
    cudaGetLastError();
    set_error("kspace_energy_exact: cudaMallocAsync failed");
    return RBX_ERR_NOMEM;
  }
  const size_t N = (size_t)n;
  int rc = launch_ewald(dbox, n, kmax, prm.alpha, prm.qqr2e, qsq, q, x, y, z, buf, buf + nk,
                        buf + 2 * (size_t)nk, stage, stage + N, stage + 2 * N,
                        buf + 5 * (size_t)nk, st);
  if (!rc)
    rc = cuda_ok(cudaMemcpyAsync(energy, buf + 5 * (size_t)nk, sizeof(double),
                                 cudaMemcpyDeviceToHost, st),
                 "D2H");
  cudaFreeAsync(buf, st);
  if (!rc) rc = cuda_ok(cudaStreamSynchronize(st), "kspace energy sync");
  return rc;
}

int rbx_engine::get_rbl_pairs(int* core_pairs, int64_t* n_core, int* shell_pairs,
                              int64_t* n_shell) {
  cudaSetDevice(device);
  if (prm.neighbor_type != RBX_NEIGHBOR_RBL || !have_cache) {
    set_error("no RBL lists: engine is not RBL or has not built its lists");
    return RBX_ERR_INVALID;
  }
  int *cc = nullptr, *core = nullptr, *sc = nullptr, *shell = nullptr;
  const size_t N = (size_t)n;
  ETRY(dalloc(&cc, N));
  ETRY(dalloc(&sc, N));
  ETRY(dalloc(&core, N * cap));
  ETRY(dalloc(&shell, N * cap));
  int rc = launch_to_fixed(dbox, n, x, y, z, q, atoms, st);
  if (!rc)
    rc = launch_rbl_lists(pp, n, atoms, x, y, z, key_a, key_b, epoch, rows(), cc,
                          core, sc, shell, st);
  std::vector<int> hcc(N), hsc(N), hcore(N * cap), hshell(N * cap), hgid(N);
  if (!rc) {
    cudaMemcpyAsync(hcc.data(), cc, sizeof(int) * N, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hsc.data(), sc, sizeof(int) * N, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hcore.data(), core, sizeof(int) * N * cap, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hshell.data(), shell, sizeof(int) * N * cap, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hgid.data(), gid, sizeof(int) * N, cudaMemcpyDeviceToHost, st);
    rc = cuda_ok(cudaStreamSynchronize(st), "sync");
  }
  cudaFree(cc);
  cudaFree(sc);
  cudaFree(core);
  cudaFree(shell);
  if (rc) return rc;
  int64_t tc = 0, ts = 0;
  for (size_t i = 0; i < N; ++i) {
    tc += hcc[i];
    ts += hsc[i];
  }
  const int64_t capc = *n_core, caps = *n_shell;
  *n_core = tc;
  *n_shell = ts;
  if (!core_pairs || !shell_pairs) return RBX_OK;  // size query
  if (capc < tc || caps < ts) {
    set_error("output arrays too small: need %lld core and %lld shell pairs", (long long)tc,
              (long long)ts);
    return RBX_ERR_INVALID;
  }
  int64_t a = 0, b = 0;
  for (size_t i = 0; i < N; ++i) {
    for (int t = 0; t < hcc[i]; ++t) {
      core_pairs[2 * a] = hgid[i];
      core_pairs[2 * a + 1] = hgid[hcore[i * cap + t]];
      ++a;
    }
    for (int t = 0; t < hsc[i]; ++t) {
      shell_pairs[2 * b] = hgid[i];
      shell_pairs[2 * b + 1] = hgid[hshell[i * cap + t]];
      ++b;
    }
  }
  return RBX_OK;
}

int rbx_engine::set_k_samples(int p, const double* hmx, const double* hmy, const double* hmz) {
  cudaSetDevice(device);
  graph_dirty = host_graph_dirty = true;
  ++graph_version;
  if (!hmx) {
    k_injected = false;
    return RBX_OK;
  }
  if (p != P) {
    set_error("injected sample count %d differs from coulomb_sample_num %d", p, P);
    return RBX_ERR_INVALID;
  }
  ETRY(cuda_ok(cudaMemcpyAsync(mx, hmx, sizeof(double) * p, cudaMemcpyHostToDevice, st), "H2D"));
  ETRY(cuda_ok(cudaMemcpyAsync(my, hmy, sizeof(double) * p, cudaMemcpyHostToDevice, st), "H2D"));
  ETRY(cuda_ok(cudaMemcpyAsync(mz, hmz, sizeof(double) * p, cudaMemcpyHostToDevice, st), "H2D"));
  ETRY(launch_m_to_int(p, mx, my, mz, mi, st));
  ETRY(cuda_ok(cudaStreamSynchronize(st), "sync"));
  k_injected = true;
  keep_parts = true;
  return RBX_OK;
}

// Adjoint of the last force evaluation: upstream g = dL/dF ([n][3], host
// order) -> dL/d(eps_t, sigma_t) per type, dL/dq_i, dL/dalpha, dL/dr_i
// (host order).  Uses the lists, batch selection (epoch) and k-samples of that
// evaluation; nothing may have moved since.
int rbx_engine::force_vjp(const double* g, double* d_eps, double* d_sigma, double* d_q_out,
                          double* d_alpha, double* d_r_out) {
  cudaSetDevice(device);
  if (prm.neighbor_type != RBX_NEIGHBOR_RBL || sog || !have_forces || !have_cache) {
    set_error("force_vjp: needs an RBL + RBE engine whose forces were computed at the current "
              "state");
    return RBX_ERR_INVALID;
  }
  const size_t N = (size_t)n;
  const int nt = prm.ntypes, npar = 2 * nt + 1;
  const int nb_pair = adj_pair_blocks(n), nb_k = adj_k_blocks(n);
  if (!adj_buf) {
    // g (3n), d_r (3n), d_q (n), type tables (2 nt), pair partials, k partials
    adj_len = 7 * N + 2 * (size_t)nt + (size_t)nb_pair * npar + (size_t)nb_k;
    ETRY(alloc(&adj_buf, adj_len));
  }
  double* gx = adj_buf;
  double* gy = gx + N;
  double* gz = gy + N;
  double* rx = gz + N;
  double* ry = rx + N;
  double* rz = ry + N;
  double* dq = rz + N;
  double* sig_t = dq + N;
  double* eps_t = sig_t + nt;
  double* ppart = eps_t + nt;
  double* kpart = ppart + (size_t)nb_pair * npar;
  double mean_g[3] = {0, 0, 0};
  for (size_t i = 0; i < N; ++i)
    for (int d = 0; d < 3; ++d) mean_g[d] += g[3 * i + d];
  for (int d = 0; d < 3; ++d) mean_g[d] /= (double)n;
  ETRY(cuda_ok(cudaMemcpyAsync(stage, g, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, st),
               "H2D"));
  ETRY(cuda_ok(cudaMemcpyAsync(sig_t, sigma.data(), sizeof(double) * nt, cudaMemcpyHostToDevice,
                               st),
               "H2D"));
  ETRY(cuda_ok(cudaMemcpyAsync(eps_t, eps.data(), sizeof(double) * nt, cudaMemcpyHostToDevice, st),
               "H2D"));
  ETRY(launch_gather_vec3(n, orig, stage, gx, gy, gz, st));
  // mixed form: FP32 pair and k-space terms (exact fixed-point phases, the k
  // table of the last force evaluation), FP64 sums; plain FP64 otherwise
  const bool mixed = prm.precision == RBX_MIXED;
  ETRY(launch_adj_pair(pp, n, x, y, z, q, type, sig_t, eps_t, key_a, key_b, epoch, rows(), gx,
                       gy, gz, mean_g, rx, ry, rz, dq, ppart, nb_pair, st, mixed));
  if (P > 0) {
    const double V = dbox.len[0] * dbox.len[1] * dbox.len[2];
    const double cscale = -4.0 * M_PI * prm.qqr2e * S / ((double)P * V);
    if (mixed)
      ETRY(launch_adj_kspace_mixed(n, P, cscale, tab, atoms, gx, gy, gz, part_re, part_im,
                                   nparts, kterm, rx, ry, rz, dq, kpart, st));
    else
      ETRY(launch_adj_kspace(n, P, cscale, tab, q, x, y, z, gx, gy, gz, part_re, part_im, nparts,
                             kterm, rx, ry, rz, dq, kpart, st));
  }
  std::vector<double> hp((size_t)nb_pair * npar), hk(P > 0 ? nb_k : 0);
  ETRY(cuda_ok(cudaMemcpyAsync(hp.data(), ppart, sizeof(double) * hp.size(),
                               cudaMemcpyDeviceToHost, st),
               "D2H"));
  if (P > 0)
    ETRY(cuda_ok(cudaMemcpyAsync(hk.data(), kpart, sizeof(double) * hk.size(),
                                 cudaMemcpyDeviceToHost, st),
                 "D2H"));
  // per-atom outputs back in host order: [n][3] positions, [n] charges
  double* const src[4] = {rx, ry, rz, dq};
  for (int a = 0; a < 4; ++a) ETRY(launch_scatter_f64(n, orig, src[a], stage + (size_t)a * N, st));
  std::vector<double> h(4 * N);
  ETRY(cuda_ok(cudaMemcpyAsync(h.data(), stage, sizeof(double) * 4 * N, cudaMemcpyDeviceToHost,
                               st),
               "D2H"));
  ETRY(cuda_ok(cudaStreamSynchronize(st), "force_vjp sync"));
  std::vector<double> par(npar, 0.0);
  for (int b = 0; b < nb_pair; ++b)  // fixed order
    for (int t = 0; t < npar; ++t) par[t] += hp[(size_t)b * npar + t];
  double gk = 0.0;
  for (double v : hk) gk += v;
  if (d_eps)
    for (int t = 0; t < nt; ++t) d_eps[t] = par[t];
  if (d_sigma)
    for (int t = 0; t < nt; ++t) d_sigma[t] = par[nt + t];
  if (d_alpha)  // k-space: the force scales with S(alpha) for fixed k-samples
    *d_alpha = par[2 * nt] + (P > 0 ? gauss_sum_dalpha(box, prm.alpha) / S * gk : 0.0);
  if (d_q_out)
    for (size_t i = 0; i < N; ++i) d_q_out[i] = h[3 * N + i];
  if (d_r_out)
    for (size_t i = 0; i < N; ++i)
      for (int d = 0; d < 3; ++d) d_r_out[3 * i + d] = h[(size_t)d * N + i];
  return RBX_OK;
}

// Per-type-pair LJ tables, eps_ij = sqrt(eps_i eps_j), sigma_ij^6 with
// sigma_ij = (sigma_i + sigma_j)/2, and fmt2v / mass for the kick (the unit's
// force-to-velocity factor folded in, as UpdateVelocityOp multiplies by it).
int rbx_engine::upload_type_tables() {
  const int nt = prm.ntypes;
  const double fmt2v = prm.fmt2v > 0 ? prm.fmt2v : 1.0;
  std::vector<double> he(nt * nt), hs(nt * nt), im(nt);
  for (int a = 0; a < nt; ++a) {
    im[a] = fmt2v == 1.0 ? 1.0 / mass[a] : fmt2v / mass[a];
    for (int b = 0; b < nt; ++b) {
      he[a * nt + b] = sqrt(eps[a] * eps[b]);
      hs[a * nt + b] = pow((sigma[a] + sigma[b]) / 2, 6.0);
    }
  }
  ETRY(cuda_ok(cudaMemcpy(inv_mass, im.data(), sizeof(double) * nt, cudaMemcpyHostToDevice),
               "H2D"));
  ETRY(cuda_ok(cudaMemcpy(mass_d, mass.data(), sizeof(double) * nt, cudaMemcpyHostToDevice),
               "H2D"));
  ETRY(cuda_ok(cudaMemcpy(lj_eps, he.data(), sizeof(double) * nt * nt, cudaMemcpyHostToDevice),
               "H2D"));
  return cuda_ok(cudaMemcpy(lj_s6, hs.data(), sizeof(double) * nt * nt, cudaMemcpyHostToDevice),
                 "H2D");
}

// Cumulative per-axis k-sampling tables for the current alpha.
int rbx_engine::build_sampler_tables() {
  std::vector<double> w;
  int off = 0;
  for (int d = 0; d < 3; ++d) {
    std::vector<double> t(8192);
    tcnt[d] = rbe_axis_table(dbox.len[d], prm.alpha, t.data(), 8192, &ttot[d]);
    if (tcnt[d] < 0) {
      set_error("k-sampler table too large for this box/alpha");
      return RBX_ERR_SAMPLER;
    }
    w.insert(w.end(), t.begin(), t.begin() + tcnt[d]);
    off += tcnt[d];
  }
  release(sample_tables);
  ETRY(alloc(&sample_tables, (size_t)off));
  return cuda_ok(cudaMemcpy(sample_tables, w.data(), sizeof(double) * off, cudaMemcpyHostToDevice),
                 "H2D");
}

// Force-field parameters (host atom order for charges).  Forces must be
// computed again; a captured step graph is captured again where it holds them.
int rbx_engine::set_lj_params(const double* hsigma, const double* heps) {
  cudaSetDevice(device);
  for (int t = 0; t < prm.ntypes; ++t)
    if (!(hsigma[t] > 0.0) || !(heps[t] >= 0.0)) {
      set_error("type %d: sigma must be > 0 and eps >= 0", t);
      return RBX_ERR_INVALID;
    }
  sigma.assign(hsigma, hsigma + prm.ntypes);
  eps.assign(heps, heps + prm.ntypes);
  have_forces = false;
  return upload_type_tables();
}

int rbx_engine::set_charges(const double* hq) {
  cudaSetDevice(device);
  qsq = 0;
  qsum = 0;
  for (int i = 0; i < n; ++i) {
    if (!std::isfinite(hq[i])) {
      set_error("atom %d has a non-finite charge", i);
      return RBX_ERR_INVALID;
    }
    qsq += hq[i] * hq[i];
    qsum += hq[i];
  }
  ETRY(cuda_ok(cudaMemcpyAsync(stage, hq, sizeof(double) * n, cudaMemcpyHostToDevice, st), "H2D"));
  ETRY(launch_gather_f64(n, orig, stage, q, st));
  h_q.assign(hq, hq + n);
  ETRY(launch_to_fixed(dbox, n, x, y, z, q, atoms, st));
  ETRY(cuda_ok(cudaStreamSynchronize(st), "set_charges sync"));
  have_forces = false;
  graph_dirty = host_graph_dirty = true;  // the energy terms carry the charge sums
  ++graph_version;
  return RBX_OK;
}

int rbx_engine::set_alpha(double a) {
  cudaSetDevice(device);
  if (!(a > 0.0)) {
    set_error("alpha must be > 0");
    return RBX_ERR_INVALID;
  }
  prm.alpha = a;
  pp.alpha = a;
  pp.sqrt_alpha = sqrt(a);
  if (P > 0 && !sog) {
    S = gauss_sum(box, a);
    ETRY(build_sampler_tables());
  }
  have_forces = false;
  graph_dirty = host_graph_dirty = true;
  ++graph_version;
  return RBX_OK;
}

// Nose-Hoover chain thermostat (NoseHooverController, nose_hoover_controller.cpp):
// t_damp <= 0 switches it off; tdof <= 0 means 3N - 3 (Computedof :1013-1025).
// SetUp (:415-471) runs here on the current velocities.
int rbx_engine::set_nose_hoover(double t_start, double t_stop, double t_damp, long long num_steps,
                                double kb, double mvv2e, double tdof) {
  cudaSetDevice(device);
  graph_dirty = host_graph_dirty = true;
  ++graph_version;  // batch graphs holding this engine are captured again
  if (!(t_damp > 0)) {
    nh_on = false;
    return RBX_OK;
  }
  if (!(t_start > 0) || !(t_stop > 0) || !(kb > 0) || !(mvv2e > 0)) {
    set_error("Nose-Hoover: temperatures, kB and mvv2e must be > 0");
    return RBX_ERR_INVALID;
  }
  if (t_stop != t_start && num_steps <= 0) {
    set_error("Nose-Hoover: a temperature ramp needs num_steps > 0");
    return RBX_ERR_INVALID;
  }
  nhp.t_start = t_start;
  nhp.t_stop = t_stop;
  nhp.t_freq = 1.0 / t_damp;
  nhp.dt = prm.dt;
  nhp.kb = kb;
  nhp.mvv2e = mvv2e;
  nhp.tdof = tdof > 0 ? tdof : 3.0 * n - 3.0;
  nhp.num_steps = num_steps;
  nh_on = true;
  ETRY(cuda_ok(cudaMemsetAsync(nh_state, 0, sizeof(double) * NH_SLOTS, st), "memset"));
  ETRY(launch_ke_partials(n, type, mass_d, vx, vy, vz, nhp.mvv2e, ke_part, st));
  ETRY(launch_nh_chain(nhp, nh_state, ke_part, nullptr, 0, 0, st));
  return cuda_ok(cudaStreamSynchronize(st), "set_nose_hoover sync");
}

// InitialIntegrate's thermostat half (nose_hoover_controller.cpp:633-646):
// target at the step being taken, chain half step, velocities scaled.
int rbx_engine::nh_initial(const int* step_dev, long long step_add, cudaStream_t s) {
  ETRY(launch_nh_chain(nhp, nh_state, ke_part, step_dev, step_add, 1, s));
  return launch_scale_v(n, nh_state, vx, vy, vz, s);
}

// FinalIntegratePostShake (:689-711): temperature of the new velocities,
// chain half step, velocities scaled.
int rbx_engine::nh_final(cudaStream_t s) {
  ETRY(launch_ke_partials(n, type, mass_d, vx, vy, vz, nhp.mvv2e, ke_part, s));
  ETRY(launch_nh_chain(nhp, nh_state, ke_part, nullptr, 0, 2, s));
  return launch_scale_v(n, nh_state, vx, vy, vz, s);
}

int rbx_engine::get_thermostat(double* temperature, double* eta, double* eta_dot) {
  cudaSetDevice(device);
  double h[NH_SLOTS];
  ETRY(cuda_ok(cudaMemcpyAsync(h, nh_state, sizeof(h), cudaMemcpyDeviceToHost, st), "D2H"));
  ETRY(cuda_ok(cudaStreamSynchronize(st), "sync"));
  if (temperature) *temperature = h[NH_TEMP];
  for (int c = 0; c < NH_CHAIN; ++c) {
    if (eta) eta[c] = h[NH_ETA + c];
    if (eta_dot) eta_dot[c] = h[NH_ETA_DOT + c];
  }
  return RBX_OK;
}

// SHAKE / RATTLE clusters (ShakeController serial path): clusters[3c..3c+2]
// are host atom indices with the centre second; bond <= 0 or no clusters
// switches it off.  The geometry of all clusters is bond, bond and
// sqrt(2 bond^2 (1 - cos angle)) as the reference's ShakeA hard-codes it.
int rbx_engine::set_shake(int nclusters, const int* clusters, double bond, double angle_deg) {
  cudaSetDevice(device);
  graph_dirty = host_graph_dirty = true;
  ++graph_version;  // batch graphs holding this engine are captured again
  if (nclusters <= 0 || !(bond > 0)) {
    shake_nc = 0;
    return RBX_OK;
  }
  std::vector<int> seen(n, 0);
  for (int c = 0; c < 3 * nclusters; ++c) {
    const int h = clusters[c];
    if (h < 0 || h >= n) {
      set_error("SHAKE cluster %d names atom %d outside [0, %d)", c / 3, h, n);
      return RBX_ERR_INVALID;
    }
    if (seen[h]++) {
      set_error("atom %d is in more than one SHAKE cluster", h);
      return RBX_ERR_INVALID;
    }
  }
  if (nclusters > shake_cap) {
    ETRY(alloc(&shake_cl, (size_t)3 * nclusters));
    shake_cap = nclusters;
  }
  if (!where) {
    ETRY(alloc(&where, (size_t)n));
    ETRY(alloc(&xs, (size_t)n));
    ETRY(alloc(&ys, (size_t)n));
    ETRY(alloc(&zs, (size_t)n));
    ETRY(launch_inverse_perm(n, orig, where, st));
  }
  ETRY(cuda_ok(cudaMemcpyAsync(shake_cl, clusters, sizeof(int) * 3 * nclusters,
                               cudaMemcpyHostToDevice, st),
               "H2D"));
  const double ang = angle_deg / 180.0 * M_PI;
  shp.dt = prm.dt;
  shp.b1sq = bond * bond;
  shp.b2sq = bond * bond;
  const double b12 = sqrt(bond * bond + bond * bond - 2.0 * bond * bond * cos(ang));
  shp.b12sq = b12 * b12;
  shp.tol = 1e-5;
  shp.max_iter = 5000;
  shake_nc = nclusters;
  ETRY(cuda_ok(cudaMemsetAsync(dflags + 6, 0, sizeof(int), st), "memset"));
  return cuda_ok(cudaStreamSynchronize(st), "set_shake sync");
}

// CVFF special bonds (LammpsFullReader's special rows, cvff_op.hip.cu
// LookupSpecialWeight): row h lists partner atoms in host order, 1-2 first,
// nspecial[h] the cumulative counts; maxspecial = 0 switches it off.
int rbx_engine::set_special(int maxspecial, const int* nspecial, const int* special, double w12,
                            double w13, double w14) {
  cudaSetDevice(device);
  graph_dirty = host_graph_dirty = true;
  ++graph_version;  // batch graphs holding this engine are captured again
  spec_natoms = 0;
  if (maxspecial <= 0) return RBX_OK;
  if (prm.neighbor_type != RBX_NEIGHBOR_RBL) {
    set_error("special bonds are applied on the RBL pair force only");
    return RBX_ERR_INVALID;
  }
  std::vector<int> list;
  for (int h = 0; h < n; ++h) {
    const int c = std::min(std::max(nspecial[3 * h + 2], 0), maxspecial);
    bool any = false;
    for (int k = 0; k < c; ++k) {
      const int p = special[(size_t)h * maxspecial + k];
      if (p < 0 || p >= n) {
        set_error("special partner %d of atom %d outside [0, %d)", p, h, n);
        return RBX_ERR_INVALID;
      }
      any = true;
    }
    if (any) list.push_back(h);
  }
  if (maxspecial > spec_cap) {
    ETRY(alloc(&spec_part, (size_t)n * maxspecial));
    spec_cap = maxspecial;
  }
  spec_max = maxspecial;
  if (!spec_cnt) {
    ETRY(alloc(&spec_cnt, (size_t)3 * n));
    ETRY(alloc(&spec_atoms, (size_t)n));
  }
  if (!where) {
    ETRY(alloc(&where, (size_t)n));
    ETRY(launch_inverse_perm(n, orig, where, st));
  }
  ETRY(cuda_ok(cudaMemcpy(spec_cnt, nspecial, sizeof(int) * 3 * n, cudaMemcpyHostToDevice), "H2D"));
  ETRY(cuda_ok(cudaMemcpy(spec_part, special, sizeof(int) * (size_t)n * maxspecial,
                          cudaMemcpyHostToDevice),
               "H2D"));
  if (!list.empty())
    ETRY(cuda_ok(cudaMemcpy(spec_atoms, list.data(), sizeof(int) * list.size(),
                            cudaMemcpyHostToDevice),
                 "H2D"));
  spec_w[0] = w12;
  spec_w[1] = w13;
  spec_w[2] = w14;
  spec_natoms = (int)list.size();
  return RBX_OK;
}

int rbx_engine::shake_a(cudaStream_t s) {
  return launch_shake_a(dbox, shp, shake_nc, shake_cl, where, type, mass_d, Pos3{xs, ys, zs},
                        Pos3{x, y, z}, Pos3{vx, vy, vz}, ImageRefs{{img[0], img[1], img[2]}}, x0,
                        y0, z0, max_d2, atoms, q, dflags + 6, s);
}

int rbx_engine::shake_b(cudaStream_t s) {
  return launch_shake_b(dbox, shake_nc, shake_cl, where, type, mass_d, Pos3{x, y, z},
                        Pos3{vx, vy, vz}, dflags + 6, s);
}

// Periodic image counters, [n][3] in host order.
int rbx_engine::set_images(const int* himg) {
  cudaSetDevice(device);
  const size_t N = (size_t)n;
  std::vector<int> cols(3 * N);
  for (size_t i = 0; i < N; ++i)
    for (int d = 0; d < 3; ++d) cols[d * N + i] = himg[3 * i + d];
  int* s32 = reinterpret_cast<int*>(stage);
  ETRY(cuda_ok(cudaMemcpyAsync(s32, cols.data(), sizeof(int) * 3 * N, cudaMemcpyHostToDevice, st),
               "H2D"));
  for (int d = 0; d < 3; ++d) ETRY(launch_gather_i32(n, orig, s32 + d * N, img[d], st));
  return cuda_ok(cudaStreamSynchronize(st), "set_images sync");
}

int rbx_engine::get_images(int* himg) {
  cudaSetDevice(device);
  const size_t N = (size_t)n;
  std::vector<int> h(3 * N);
  for (int d = 0; d < 3; ++d) {
    ETRY(launch_scatter_i32(n, orig, img[d], reinterpret_cast<int*>(stage) + d * N, st));
  }
  ETRY(cuda_ok(cudaMemcpyAsync(h.data(), stage, sizeof(int) * 3 * N, cudaMemcpyDeviceToHost, st),
               "D2H"));
  ETRY(cuda_ok(cudaStreamSynchronize(st), "get_images sync"));
  for (size_t i = 0; i < N; ++i)
    for (int d = 0; d < 3; ++d) himg[3 * i + d] = h[d * N + i];
  return RBX_OK;
}

namespace {
// Shortest decimal that reads back as the same double (the "{}" format of the
// reference's trajectory writer).
void put_real(std::string& out, double v) {
  char b[32];
  const auto r = std::to_chars(b, b + sizeof b, v);
  out.append(b, r.ptr);
}
}  // namespace

// One frame in the reference's trajectory format (TrajectoryOutput::Execute,
// src/output/src/TrajectoryOutput.cpp:467-500): LAMMPS custom dump with
// id type q x y z xu yu zu vx vy vz, atoms by id, ids and types 1-based,
// xu = x + image * L.
int rbx_engine::write_trajectory(const char* path, int64_t timestep, bool append) {
  cudaSetDevice(device);
  const size_t N = (size_t)n;
  std::vector<double> h(6 * N);
  double* c[6];
  for (int a = 0; a < 6; ++a) c[a] = h.data() + a * N;
  ETRY(get_state(c[0], c[1], c[2], c[3], c[4], c[5], nullptr, nullptr, nullptr));
  std::vector<int> im(3 * N);
  ETRY(get_images(im.data()));
  std::vector<size_t> order(N);
  for (size_t i = 0; i < N; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return h_gid[a] < h_gid[b]; });
  FILE* fp = fopen(path, append ? "a" : "w");
  if (!fp) {
    set_error("cannot write %s", path);
    return RBX_ERR_INVALID;
  }
  std::string s;
  s.reserve(N * 200 + 256);
  s += "ITEM: TIMESTEP\n" + std::to_string(timestep) + "\nITEM: NUMBER OF ATOMS\n" +
       std::to_string(n) + "\nITEM: BOX BOUNDS pp pp pp\n";
  for (int d = 0; d < 3; ++d) {
    put_real(s, box.lo[d]);
    s += ' ';
    put_real(s, box.hi[d]);
    s += '\n';
  }
  s += "ITEM: ATOMS id type q x y z xu yu zu vx vy vz\n";
  const double L[3] = {dbox.len[0], dbox.len[1], dbox.len[2]};
  for (size_t k = 0; k < N; ++k) {
    const size_t i = order[k];
    s += std::to_string((long long)h_gid[i] + 1);
    s += ' ';
    s += std::to_string(h_type[i] + 1);
    s += ' ';
    put_real(s, h_q[i]);
    for (int d = 0; d < 3; ++d) {
      s += ' ';
      put_real(s, c[d][i]);
    }
    for (int d = 0; d < 3; ++d) {
      s += ' ';
      put_real(s, c[d][i] + im[3 * i + d] * L[d]);
    }
    for (int d = 0; d < 3; ++d) {
      s += ' ';
      put_real(s, c[3 + d][i]);
    }
    s += '\n';
  }
  const bool ok = fwrite(s.data(), 1, s.size(), fp) == s.size();
  if (fclose(fp) != 0 || !ok) {
    set_error("write error on %s", path);
    return RBX_ERR_INVALID;
  }
  return RBX_OK;
}

int rbx_engine::get_stats(rbx_stats* s) {
  cudaSetDevice(device);
  memset(s, 0, sizeof(*s));
  s->steps = steps;
  s->force_calls = force_calls;
  s->rebuilds = rebuilds;
  s->epoch = epoch;
  s->selection_frequency = freq;
  s->candidate_capacity = cap;
  if (have_cache)
    ETRY(cuda_ok(cudaMemcpy(&s->candidates, cand_total, sizeof(long long), cudaMemcpyDeviceToHost),
                 "D2H"));
  if (P > 0) {
    ETRY(cuda_ok(cudaMemcpy(&s->e_kspace, ek, sizeof(double), cudaMemcpyDeviceToHost), "D2H"));
    ETRY(cuda_ok(cudaMemcpy(s->virial_kspace, virk, sizeof(double) * 6, cudaMemcpyDeviceToHost),
                 "D2H"));
  }
  return RBX_OK;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

rbx_engine* rbx_engine_create(const rbx_params* params, const rbx_box* box, int num_atoms,
                              int device) {
  if (!params || !box || num_atoms <= 0 || !params->sigma || !params->eps || !params->mass) {
    set_error("rbx_engine_create: null params/box or num_atoms <= 0");
    return nullptr;
  }
  rbx_engine* e = new rbx_engine();
  e->prm = *params;
  e->box = *box;
  e->n = num_atoms;
  e->device = device;
  e->sigma.assign(params->sigma, params->sigma + params->ntypes);
  e->eps.assign(params->eps, params->eps + params->ntypes);
  e->mass.assign(params->mass, params->mass + params->ntypes);
  e->prm.sigma = e->sigma.data();
  e->prm.eps = e->eps.data();
  e->prm.mass = e->mass.data();
  if (e->init() != RBX_OK) {
    delete e;
    return nullptr;
  }
  return e;
}

void rbx_engine_destroy(rbx_engine* e) { delete e; }

int rbx_engine_set_state(rbx_engine* e, const int* gid, const int* type, const double* charge,
                         const double* px, const double* py, const double* pz, const double* vx,
                         const double* vy, const double* vz) {
  if (!e || !gid || !type || !charge || !px || !py || !pz || !vx || !vy || !vz) {
    set_error("rbx_engine_set_state: null argument");
    return RBX_ERR_INVALID;
  }
  return e->set_state(gid, type, charge, px, py, pz, vx, vy, vz);
}

int rbx_engine_set_k_samples(rbx_engine* e, int p, const double* mx, const double* my,
                             const double* mz) {
  if (!e) return RBX_ERR_INVALID;
  return e->set_k_samples(p, mx, my, mz);
}

int rbx_engine_compute_forces(rbx_engine* e, int epoch) {
  if (!e) return RBX_ERR_INVALID;
  e->keep_parts = true;
  return e->compute_forces(epoch);
}

int rbx_engine_step(rbx_engine* e, int nsteps) {
  if (!e || nsteps < 0) return RBX_ERR_INVALID;
  return e->step(nsteps);
}

int rbx_engine_step_host(rbx_engine* e, const double* x_in, const double* v_in, double* x_out,
                         double* v_out, double* f_out) {
  if (!e || !x_in || !v_in || !x_out || !v_out || !f_out) {
    set_error("rbx_engine_step_host: null argument");
    return RBX_ERR_INVALID;
  }
  return e->step_host(x_in, v_in, x_out, v_out, f_out);
}

int rbx_engine_get_state(rbx_engine* e, double* px, double* py, double* pz, double* vx, double* vy,
                         double* vz, double* fx, double* fy, double* fz) {
  if (!e) return RBX_ERR_INVALID;
  return e->get_state(px, py, pz, vx, vy, vz, fx, fy, fz);
}

int rbx_engine_get_force_parts(rbx_engine* e, double* f_pair, double* f_kspace) {
  if (!e) return RBX_ERR_INVALID;
  return e->get_force_parts(f_pair, f_kspace);
}

int rbx_engine_pair_energy(rbx_engine* e, double* e_vdwl, double* e_coul, double* virial) {
  if (!e) return RBX_ERR_INVALID;
  return e->pair_energy(e_vdwl, e_coul, virial);
}

int rbx_engine_kspace_energy_exact(rbx_engine* e, const int kmax[3], double* energy) {
  if (!e) return RBX_ERR_INVALID;
  return e->kspace_energy_exact(kmax, energy);
}

int rbx_engine_get_rbl_pairs(rbx_engine* e, int* core_pairs, int64_t* n_core, int* shell_pairs,
                             int64_t* n_shell) {
  if (!e || !n_core || !n_shell) return RBX_ERR_INVALID;
  return e->get_rbl_pairs(core_pairs, n_core, shell_pairs, n_shell);
}

int rbx_engine_get_stats(rbx_engine* e, rbx_stats* out) {
  if (!e || !out) return RBX_ERR_INVALID;
  return e->get_stats(out);
}

int rbx_engine_rbsog_npt_map(rbx_engine* e, int* p, int* idx_npt) {
  if (!e || !p) return RBX_ERR_INVALID;
  if (!e->sog || e->P <= 0) {
    set_error("rbx_engine_rbsog_npt_map: not an RBSOG engine with samples");
    return RBX_ERR_INVALID;
  }
  *p = e->P;
  if (!idx_npt) return RBX_OK;
  cudaSetDevice(e->device);
  ETRY(cuda_ok(cudaStreamSynchronize(e->st), "rbx_engine_rbsog_npt_map"));
  return cuda_ok(cudaMemcpy(idx_npt, e->sog_idx, sizeof(int) * e->P, cudaMemcpyDeviceToHost),
                 "D2H");
}

void* rbx_engine_stream(rbx_engine* e) { return e ? (void*)e->st : nullptr; }

int rbx_engine_phase_ms(rbx_engine* e, float out[4]) {
  if (!e || !out) return RBX_ERR_INVALID;
  return e->phase_ms(out);
}

int rbx_engine_force_vjp(rbx_engine* e, const double* g, double* d_eps, double* d_sigma,
                         double* d_charge, double* d_alpha, double* d_pos) {
  if (!e || !g) {
    set_error("rbx_engine_force_vjp: null engine or upstream gradient");
    return RBX_ERR_INVALID;
  }
  return e->force_vjp(g, d_eps, d_sigma, d_charge, d_alpha, d_pos);
}

int rbx_engine_set_lj_params(rbx_engine* e, const double* sigma, const double* eps) {
  if (!e || !sigma || !eps) {
    set_error("rbx_engine_set_lj_params: null argument");
    return RBX_ERR_INVALID;
  }
  return e->set_lj_params(sigma, eps);
}

int rbx_engine_set_charges(rbx_engine* e, const double* charge) {
  if (!e || !charge) {
    set_error("rbx_engine_set_charges: null argument");
    return RBX_ERR_INVALID;
  }
  return e->set_charges(charge);
}

int rbx_engine_set_alpha(rbx_engine* e, double alpha) {
  if (!e) return RBX_ERR_INVALID;
  return e->set_alpha(alpha);
}

int rbx_engine_get_system(rbx_engine* e, int* num_atoms, int* ntypes, rbx_box* box) {
  if (!e) return RBX_ERR_INVALID;
  if (num_atoms) *num_atoms = e->n;
  if (ntypes) *ntypes = e->prm.ntypes;
  if (box) *box = e->box;
  return RBX_OK;
}

int rbx_engine_get_atoms(rbx_engine* e, int* gid, int* type, double* charge) {
  if (!e) return RBX_ERR_INVALID;
  if (e->h_gid.size() != (size_t)e->n) {
    set_error("rbx_engine_get_atoms: no state set");
    return RBX_ERR_INVALID;
  }
  if (gid) std::copy(e->h_gid.begin(), e->h_gid.end(), gid);
  if (type) std::copy(e->h_type.begin(), e->h_type.end(), type);
  if (charge) std::copy(e->h_q.begin(), e->h_q.end(), charge);
  return RBX_OK;
}

int rbx_engine_get_type_params(rbx_engine* e, double* sigma, double* eps, double* mass) {
  if (!e) return RBX_ERR_INVALID;
  if (sigma) std::copy(e->sigma.begin(), e->sigma.end(), sigma);
  if (eps) std::copy(e->eps.begin(), e->eps.end(), eps);
  if (mass) std::copy(e->mass.begin(), e->mass.end(), mass);
  return RBX_OK;
}

int rbx_engine_set_nose_hoover(rbx_engine* e, double t_start, double t_stop, double t_damp,
                               int64_t num_steps, double kb, double mvv2e, double tdof) {
  if (!e) return RBX_ERR_INVALID;
  return e->set_nose_hoover(t_start, t_stop, t_damp, (long long)num_steps, kb, mvv2e, tdof);
}

int rbx_engine_get_thermostat(rbx_engine* e, double* temperature, double* eta, double* eta_dot) {
  if (!e) return RBX_ERR_INVALID;
  return e->get_thermostat(temperature, eta, eta_dot);
}

int rbx_engine_set_special(rbx_engine* e, int maxspecial, const int* nspecial,
                           const int* special, double w12, double w13, double w14) {
  if (!e || (maxspecial > 0 && (!nspecial || !special))) return RBX_ERR_INVALID;
  return e->set_special(maxspecial, nspecial, special, w12, w13, w14);
}

int rbx_engine_set_shake(rbx_engine* e, int nclusters, const int* clusters, double bond,
                         double angle_deg) {
  if (!e || (nclusters > 0 && !clusters)) return RBX_ERR_INVALID;
  return e->set_shake(nclusters, clusters, bond, angle_deg);
}

int rbx_engine_get_shake(rbx_engine* e, int* nclusters, int* failures) {
  if (!e) return RBX_ERR_INVALID;
  cudaSetDevice(e->device);
  int f = 0;
  if (cudaMemcpy(&f, e->dflags + 6, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
    set_error("rbx_engine_get_shake: device read failed");
    return RBX_ERR_DEVICE;
  }
  if (nclusters) *nclusters = e->shake_nc;
  if (failures) *failures = f;
  return RBX_OK;
}

int rbx_engine_autotune(rbx_engine* e, int force, rbx_tuning* out) {
  if (!e) return RBX_ERR_INVALID;
  return e->autotune(force != 0, out);
}

int rbx_engine_set_images(rbx_engine* e, const int* image) {
  if (!e || !image) return RBX_ERR_INVALID;
  return e->set_images(image);
}

int rbx_engine_get_images(rbx_engine* e, int* image) {
  if (!e || !image) return RBX_ERR_INVALID;
  return e->get_images(image);
}

int rbx_engine_write_trajectory(rbx_engine* e, const char* path, int64_t timestep, int append) {
  if (!e || !path) return RBX_ERR_INVALID;
  return e->write_trajectory(path, timestep, append != 0);
}

int rbx_engine_set_step_graph(rbx_engine* e, int on) {
  if (!e) return RBX_ERR_INVALID;
  e->use_graph = on != 0;
  return RBX_OK;
}

int rbx_engine_set_profiling(rbx_engine* e, int on) {
  if (!e) return RBX_ERR_INVALID;
  e->profiling = on != 0;
  for (int k = 0; k < 4; ++k) e->phase_total[k] = 0.0;
  e->phase_steps = 0;
  e->pev_used = 0;
  return RBX_OK;
}

}  // extern "C"
