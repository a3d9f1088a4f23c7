// rbx_batch.cu -- many independent engines (replicas) advanced by one CUDA
// graph launch per MD step.  No counterpart in the reference, which runs one
// system per process.
//
// Two graph designs:
//  * phase-batched (the default where every replica allows it): one launch
//    per phase of the step over the blocks of all replicas -- drift with the
//    first half kick and the rebuild decision, fused RBL force, structure
//    factor with the k-sampling, finalize with the energy sum, RBE force with
//    the second half kick -- each block reading its replica's argument block
//    from a device table; between the drift and the RBL phase every replica
//    has its own IF node whose body is that replica's rebuild (replicas
//    rebuild on different steps);
//  * branches: every replica's step graph as a parallel branch (the batch
//    stream forks into each engine's stream and joins back).
#include <map>
#include <tuple>
#include <vector>

#include "rbx_engine.h"

using namespace rbx;

namespace rbx {
void set_error(const char* fmt, ...);

BatchRecorder*& batch_recorder() {
  static thread_local BatchRecorder* rec = nullptr;
  return rec;
}

int record_phase(int kind, int variant, int blocks, int threads, size_t smem, const void* args,
                 size_t bytes) {
  PhaseRecord r;
  r.kind = kind;
  r.variant = variant;
  r.blocks = blocks;
  r.threads = threads;
  r.smem = smem;
  r.args.assign(static_cast<const unsigned char*>(args),
                static_cast<const unsigned char*>(args) + bytes);
  batch_recorder()->recs.push_back(std::move(r));
  return RBX_OK;
}

int launch_phase_batch(int kind, int variant, const void* args, const int* start, int nrep,
                       int total, int threads, size_t smem, cudaStream_t st) {
  (void)threads;
  switch (kind) {
    case PH_DRIFT: return launch_drift_batch(args, start, nrep, total, st);
    case PH_RBL: return launch_rbl_batch(variant, args, start, nrep, total, smem, st);
    case PH_RHO: return launch_rho_mixed_batch(variant, args, start, nrep, total, st);
    case PH_FINALIZE: return launch_finalize_batch(args, start, nrep, total, st);
    case PH_FORCE: return launch_force_mixed_batch(variant, args, start, nrep, total, st);
  }
  set_error("launch_phase_batch: unknown phase %d", kind);
  return RBX_ERR_INVALID;
}
}  // namespace rbx

struct rbx_batch {
  std::vector<rbx_engine*> eng;
  std::vector<unsigned> versions;  // engine graph_version at capture
  std::vector<cudaEvent_t> join;
  cudaEvent_t fork = nullptr;
  cudaStream_t st = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int device = 0;
  int mode = RBX_BATCH_AUTO;   // requested design
  int design = -1;             // captured design (RBX_BATCH_PHASED or RBX_BATCH_BRANCHES)
  void* tables = nullptr;      // device argument tables of the phase launches
  unsigned long long phase_launches = 0;  // kernel launches per step outside the rebuilds

  ~rbx_batch() {
    cudaSetDevice(device);
    release();
    for (cudaEvent_t e : join) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    if (st) cudaStreamDestroy(st);
  }
  void release() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (tables) cudaFree(tables);
    exec = nullptr;
    graph = nullptr;
    tables = nullptr;
    design = -1;
  }
  static int ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return RBX_OK;
    cudaGetLastError();
    set_error("%s: %s", what, cudaGetErrorString(e));
    return RBX_ERR_CUDA;
  }
  // One launch per phase over all replicas (see the file comment).
  int capture_phased() {
    release();
    const int R = (int)eng.size();
    int rc = ok(cudaGraphCreate(&graph, 0), "cudaGraphCreate");
    std::vector<cudaGraphConditionalHandle> cond(R);
    std::vector<BatchRecorder> rec(R);
    for (int r = 0; r < R && !rc; ++r)
      rc = ok(cudaGraphConditionalHandleCreate(&cond[r], graph, 0, cudaGraphCondAssignDefault),
              "cudaGraphConditionalHandleCreate");
    for (int r = 0; r < R && !rc; ++r) rc = eng[r]->record_phased_step(&rec[r], cond[r]);
    const size_t nph = rc ? 0 : rec[0].recs.size();
    if (!rc && (nph < 2 || rec[0].recs[0].kind != PH_DRIFT)) {
      set_error("phase-batched step: the step does not start with the drift");
      rc = RBX_ERR_INVALID;
    }
    for (int r = 1; r < R && !rc; ++r) {
      bool same = rec[r].recs.size() == nph;
      for (size_t k = 0; same && k < nph; ++k) same = rec[r].recs[k].kind == rec[0].recs[k].kind;
      if (!same) {
        set_error("phase-batched step: replica %d runs other phases than replica 0", r);
        rc = RBX_ERR_INVALID;
      }
    }
    if (rc) {
      release();
      return rc;
    }
    // per phase, one launch per (variant, block size): argument blocks back to
    // back, then start[0..nrep] (16-byte aligned pieces of one device table)
    struct Launch {
      int kind, variant, threads, nrep, total;
      size_t smem, args_off, start_off;
    };
    std::vector<Launch> launches;
    std::vector<unsigned char> blob;
    auto align16 = [&blob]() { blob.resize((blob.size() + 15) & ~(size_t)15); };
    for (size_t k = 0; k < nph; ++k) {
      std::map<std::pair<int, int>, std::vector<int>> groups;
      for (int r = 0; r < R; ++r)
        groups[{rec[r].recs[k].variant, rec[r].recs[k].threads}].push_back(r);
      for (auto& g : groups) {
        Launch L{rec[0].recs[k].kind, g.first.first, g.first.second, (int)g.second.size(), 0, 0,
                 0, 0};
        align16();
        L.args_off = blob.size();
        std::vector<int> start(1, 0);
        for (int r : g.second) {
          const PhaseRecord& pr = rec[r].recs[k];
          blob.insert(blob.end(), pr.args.begin(), pr.args.end());
          start.push_back(start.back() + pr.blocks);
          L.smem = std::max(L.smem, pr.smem);
        }
        L.total = start.back();
        align16();
        L.start_off = blob.size();
        const unsigned char* sp = reinterpret_cast<const unsigned char*>(start.data());
        blob.insert(blob.end(), sp, sp + sizeof(int) * start.size());
        launches.push_back(L);
      }
    }
    rc = ok(cudaMalloc(&tables, blob.size()), "cudaMalloc (phase tables)");
    if (!rc)
      rc = ok(cudaMemcpy(tables, blob.data(), blob.size(), cudaMemcpyHostToDevice),
              "H2D (phase tables)");
    if (!rc)
      rc = ok(cudaStreamBeginCaptureToGraph(st, graph, nullptr, nullptr, 0,
                                            cudaStreamCaptureModeThreadLocal),
              "cudaStreamBeginCaptureToGraph");
    if (rc) {
      release();
      return rc;
    }
    const unsigned long long l0 = rbx_launch_count();
    auto run = [&](const Launch& L) {
      const unsigned char* base = static_cast<const unsigned char*>(tables);
      return launch_phase_batch(L.kind, L.variant, base + L.args_off,
                                reinterpret_cast<const int*>(base + L.start_off), L.nrep,
                                L.total, L.threads, L.smem, st);
    };
    size_t li = 0;
    for (; li < launches.size() && launches[li].kind == PH_DRIFT && !rc; ++li)
      rc = run(launches[li]);
    unsigned long long rebuild_launches = 0;
    if (!rc) {  // every replica's rebuild under its own IF node, after the drift
      cudaStreamCaptureStatus cs;
      cudaGraph_t capg = nullptr;
      const cudaGraphNode_t* deps = nullptr;
      size_t ndeps = 0;
      rc = ok(cudaStreamGetCaptureInfo(st, &cs, nullptr, &capg, &deps, &ndeps),
              "cudaStreamGetCaptureInfo");
      const std::vector<cudaGraphNode_t> after(deps, deps + ndeps);
      std::vector<cudaGraphNode_t> nodes(R);
      for (int r = 0; r < R && !rc; ++r) {
        cudaGraphNodeParams np{};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = cond[r];
        np.conditional.type = cudaGraphCondTypeIf;
        np.conditional.size = 1;
        rc = ok(cudaGraphAddNode(&nodes[r], capg, after.data(), after.size(), &np),
                "cudaGraphAddNode");
        if (!rc) rc = eng[r]->capture_rebuild_body(np.conditional.phGraph_out[0]);
        rebuild_launches += eng[r]->graph_rebuild_launches;
      }
      if (!rc)
        rc = ok(cudaStreamUpdateCaptureDependencies(st, nodes.data(), nodes.size(),
                                                    cudaStreamSetCaptureDependencies),
                "cudaStreamUpdateCaptureDependencies");
    }
    for (; li < launches.size() && !rc; ++li) rc = run(launches[li]);
    phase_launches = rbx_launch_count() - l0 - rebuild_launches;
    cudaGraph_t g = graph;
    const cudaError_t ec = cudaStreamEndCapture(st, &g);
    if (!rc) rc = ok(ec, "cudaStreamEndCapture");
    if (!rc) rc = ok(cudaGraphInstantiate(&exec, graph, 0), "cudaGraphInstantiate");
    if (rc) {
      release();
      return rc;
    }
    for (int r = 0; r < R; ++r) versions[r] = eng[r]->graph_version;
    design = RBX_BATCH_PHASED;
    return RBX_OK;
  }

  // AUTO: the phased graph for replicas of fewer than kPhasedMeanAtoms atoms
  // on average, else the branches.  One launch per phase pays off over many
  // small replicas (910 x 2,000 atoms: 5.1x the branches, whose thousand-node
  // graph is bound by node scheduling); at 256 x 7,100 atoms the designs are
  // level, and with larger replicas the branches win (the phased force
  // launches wait for every replica's rebuild).
  static constexpr int kPhasedMeanAtoms = 5000;
  int capture() {
    long long atoms = 0;
    for (rbx_engine* e : eng) atoms += e->n;
    const bool small = atoms < (long long)kPhasedMeanAtoms * (long long)eng.size();
    if (mode == RBX_BATCH_PHASED || (mode == RBX_BATCH_AUTO && small)) {
      const int rc = capture_phased();
      if (rc == RBX_OK || mode == RBX_BATCH_PHASED) return rc;
    }
    return capture_branches();
  }

  int capture_branches() {
    release();
    int rc = ok(cudaGraphCreate(&graph, 0), "cudaGraphCreate");
    if (rc) return rc;
    rc = ok(cudaStreamBeginCaptureToGraph(st, graph, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal),
            "cudaStreamBeginCaptureToGraph");
    if (rc) return rc;
    rc = ok(cudaEventRecord(fork, st), "cudaEventRecord");
    for (size_t r = 0; r < eng.size() && !rc; ++r) {
      rbx_engine* e = eng[r];
      rc = ok(cudaStreamWaitEvent(e->st, fork, 0), "cudaStreamWaitEvent");  // branch r
      if (!rc) rc = e->capture_step_into(graph, false);
      if (!rc) rc = ok(cudaEventRecord(join[r], e->st), "cudaEventRecord");
      if (!rc) rc = ok(cudaStreamWaitEvent(st, join[r], 0), "cudaStreamWaitEvent");  // join
    }
    cudaGraph_t g = graph;
    const cudaError_t ec = cudaStreamEndCapture(st, &g);
    if (!rc) rc = ok(ec, "cudaStreamEndCapture");
    if (!rc) rc = ok(cudaGraphInstantiate(&exec, graph, 0), "cudaGraphInstantiate");
    if (rc) {
      release();
      return rc;
    }
    for (size_t r = 0; r < eng.size(); ++r) versions[r] = eng[r]->graph_version;
    design = RBX_BATCH_BRANCHES;
    return RBX_OK;
  }
};

extern "C" {

rbx_batch* rbx_batch_create(rbx_engine* const* engines, int count) {
  if (!engines || count <= 0) {
    set_error("rbx_batch_create: no engines");
    return nullptr;
  }
  auto* b = new rbx_batch();
  b->device = engines[0]->device;
  for (int r = 0; r < count; ++r) {
    rbx_engine* e = engines[r];
    if (!e || e->device != b->device) {
      set_error("rbx_batch_create: engine %d is null or on another device", r);
      delete b;
      return nullptr;
    }
    for (int q = 0; q < r; ++q)
      if (engines[q] == e) {
        set_error("rbx_batch_create: engine %d appears twice", r);
        delete b;
        return nullptr;
      }
    b->eng.push_back(e);
  }
  cudaSetDevice(b->device);
  b->versions.assign(count, ~0u);
  b->join.assign(count, nullptr);
  bool good = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess;
  for (int r = 0; r < count && good; ++r)
    good = cudaEventCreateWithFlags(&b->join[r], cudaEventDisableTiming) == cudaSuccess;
  if (!good) {
    cudaGetLastError();
    set_error("rbx_batch_create: stream/event creation failed");
    delete b;
    return nullptr;
  }
  return b;
}

void rbx_batch_destroy(rbx_batch* b) { delete b; }

void* rbx_batch_stream(rbx_batch* b) { return b ? (void*)b->st : nullptr; }

int rbx_batch_autotune(rbx_batch* b) {
  if (!b) {
    set_error("rbx_batch_autotune: null batch");
    return RBX_ERR_INVALID;
  }
  for (rbx_engine* e : b->eng) {
    const int rc = e->autotune(false, nullptr);
    if (rc) return rc;
  }
  return RBX_OK;
}

int rbx_batch_step(rbx_batch* b, int nsteps) {
  if (!b || nsteps < 0) {
    set_error("rbx_batch_step: invalid batch or step count");
    return RBX_ERR_INVALID;
  }
  if (nsteps == 0) return RBX_OK;
  cudaSetDevice(b->device);
  bool stale = b->exec == nullptr;
  for (size_t r = 0; r < b->eng.size(); ++r) {
    rbx_engine* e = b->eng[r];
    if (!e->have_forces) {
      const int rc = e->compute_forces(e->epoch);
      if (rc) return rc;
    }
    if (!e->have_cache || e->prm.skin <= 0.0 || e->profiling) {
      set_error("rbx_batch_step: engine %zu needs a neighbour list, skin > 0 and profiling off", r);
      return RBX_ERR_INVALID;
    }
    stale = stale || e->graph_version != b->versions[r];
  }
  if (stale) {
    const int rc = b->capture();
    if (rc) return rc;
  }
  for (rbx_engine* e : b->eng) {
    const int rc = e->graph_run_begin(b->st);
    if (rc) return rc;
  }
  for (int k = 0; k < nsteps; ++k) {
    const int rc = rbx_batch::ok(cudaGraphLaunch(b->exec, b->st), "cudaGraphLaunch");
    if (rc) return rc;
  }
  for (rbx_engine* e : b->eng) {
    const int rc = rbx_batch::ok(cudaMemcpyAsync(e->run_flags, e->dflags, sizeof(int) * 6,
                                                 cudaMemcpyDeviceToHost, b->st),
                                 "D2H");
    if (rc) return rc;
  }
  int rc = rbx_batch::ok(cudaStreamSynchronize(b->st), "batch sync");
  const bool phased = b->design == RBX_BATCH_PHASED;
  for (rbx_engine* e : b->eng)
    if (!rc) rc = e->graph_run_end(nsteps, phased ? 0 : e->graph_step_launches);
  if (!rc && phased) count_launch((int)(b->phase_launches * nsteps));
  return rc;
}

int rbx_batch_set_mode(rbx_batch* b, int mode) {
  if (!b || mode < RBX_BATCH_AUTO || mode > RBX_BATCH_BRANCHES) {
    set_error("rbx_batch_set_mode: invalid batch or mode");
    return RBX_ERR_INVALID;
  }
  if (mode != b->mode) {
    cudaSetDevice(b->device);
    b->release();
    b->mode = mode;
  }
  return RBX_OK;
}

int rbx_batch_design(const rbx_batch* b) { return b ? b->design : -1; }

}  // extern "C"
