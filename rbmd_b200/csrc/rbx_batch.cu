// rbx_batch.cu -- many independent engines (replicas) advanced by one CUDA
// graph launch per MD step.
//
// The batch graph holds every replica's step as a parallel branch: the batch
// stream forks into each engine's stream, each engine records its own step
// (kick, drift, decision kernel, the rebuild under its own conditional node,
// forces, second kick), and the branches join back.  Small systems that
// cannot fill the GPU alone run side by side.  No counterpart in the
// reference, which runs one system per process.
#include <vector>

#include "rbx_engine.h"

using namespace rbx;

namespace rbx {
void set_error(const char* fmt, ...);
}

struct rbx_batch {
  std::vector<rbx_engine*> eng;
  std::vector<unsigned> versions;  // engine graph_version at capture
  std::vector<cudaEvent_t> join;
  cudaEvent_t fork = nullptr;
  cudaStream_t st = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int device = 0;

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
    exec = nullptr;
    graph = nullptr;
  }
  static int ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return RBX_OK;
    cudaGetLastError();
    set_error("%s: %s", what, cudaGetErrorString(e));
    return RBX_ERR_CUDA;
  }
  int capture() {
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
      if (!rc) rc = e->capture_step_into(graph);
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
  for (rbx_engine* e : b->eng)
    if (!rc) rc = e->graph_run_end(nsteps, e->graph_step_launches);
  return rc;
}

}  // extern "C"
