// fz_group.cpp -- several solver handles (rooms) advanced together, one CUDA graph per run of
// graph_steps steps whose parallel branches are the members. Small rooms leave most of the GPU
// idle when stepped one after another; as branches of one graph their kernels share the SMs.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "fz_internal.h"

struct fz_group {
  std::vector<fz_handle*> m;
  int device = 0;
  int graph_steps = 10;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr, done = nullptr;
  std::vector<cudaEvent_t> join;
  // keyed by the members' buffer parities (the field-set rotation repeats every 2 steps)
  std::map<std::vector<int>, cudaGraphExec_t> graphs;
};

namespace {

int gfail(fz_group* g, cudaError_t e, const char* what) {
  return fzi::cuda_fail(g && !g->m.empty() ? g->m[0] : nullptr, e, what);
}

#define FZ_GCUDA(g, call, what)                        \
  do {                                                 \
    cudaError_t e__ = (call);                          \
    if (e__ != cudaSuccess) return gfail(g, e__, what); \
  } while (0)

// every member's stream waits for what is already on the group stream, and vice versa
int order_after(fz_group* g, bool members_wait_for_group) {
  if (members_wait_for_group) {
    FZ_GCUDA(g, cudaEventRecord(g->done, g->stream), "event record");
    for (fz_handle* h : g->m) FZ_GCUDA(g, cudaStreamWaitEvent(h->stream, g->done, 0), "stream wait");
  } else {
    for (size_t i = 0; i < g->m.size(); i++) {
      FZ_GCUDA(g, cudaEventRecord(g->join[i], g->m[i]->stream), "event record");
      FZ_GCUDA(g, cudaStreamWaitEvent(g->stream, g->join[i], 0), "stream wait");
    }
  }
  return FZ_OK;
}

int capture(fz_group* g, cudaGraphExec_t* out) {
  cudaGraph_t graph = nullptr;
  FZ_GCUDA(g, cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
  cudaError_t e = cudaEventRecord(g->fork, g->stream);
  for (size_t i = 0; i < g->m.size() && e == cudaSuccess; i++) {
    fz_handle* h = g->m[i];
    e = cudaStreamWaitEvent(h->stream, g->fork, 0);
    for (int s = 0; s < g->graph_steps && e == cudaSuccess; s++) e = fzi::enqueue(h);
    if (e == cudaSuccess) e = cudaEventRecord(g->join[i], h->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(g->stream, g->join[i], 0);
  }
  const cudaError_t e2 = cudaStreamEndCapture(g->stream, &graph);
  if (e != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return gfail(g, e, "group capture");
  }
  if (e2 != cudaSuccess) return gfail(g, e2, "group end capture");
  e = cudaGraphInstantiate(out, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return gfail(g, e, "group graph instantiate");
  return FZ_OK;
}

}  // namespace

extern "C" {

void fz_group_destroy(fz_group* g) {
  if (!g) return;
  cudaSetDevice(g->device);
  if (g->stream) cudaStreamSynchronize(g->stream);
  for (auto& kv : g->graphs) cudaGraphExecDestroy(kv.second);
  for (cudaEvent_t e : g->join) cudaEventDestroy(e);
  if (g->fork) cudaEventDestroy(g->fork);
  if (g->done) cudaEventDestroy(g->done);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
}

int fz_group_create(fz_handle* const* members, int32_t n, fz_group** out) {
  if (!members || !out || n < 1) return fzi::set_global_error(FZ_EINVAL, "fz_group_create: bad arguments");
  *out = nullptr;
  for (int i = 0; i < n; i++) {
    if (!members[i]) return fzi::set_global_error(FZ_EINVAL, "fz_group_create: NULL member");
    if (members[i]->device != members[0]->device)
      return fzi::set_global_error(FZ_EINVAL, "fz_group_create: members on different devices");
    if (members[i]->profiling)
      return fzi::set_global_error(FZ_EINVAL, "fz_group_create: a member has profiling enabled");
    for (int j = 0; j < i; j++)
      if (members[j] == members[i]) return fzi::set_global_error(FZ_EINVAL, "fz_group_create: repeated member");
  }
  for (int i = 0; i < n; i++) {
    const int rc = fzi::prepare(members[i]);
    if (rc != FZ_OK) return fzi::set_global_error(rc, "fz_group_create: member " + std::to_string(i) + ": " + members[i]->err);
  }
  fz_group* g = new (std::nothrow) fz_group();
  if (!g) return fzi::set_global_error(FZ_ENOMEM, "fz_group_create: out of host memory");
  g->m.assign(members, members + n);
  g->device = members[0]->device;
  cudaSetDevice(g->device);
  cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->done, cudaEventDisableTiming);
  g->join.assign((size_t)n, nullptr);
  for (int i = 0; i < n && e == cudaSuccess; i++) e = cudaEventCreateWithFlags(&g->join[(size_t)i], cudaEventDisableTiming);
  if (e != cudaSuccess) {
    const int rc = fzi::set_global_error(FZ_ECUDA, std::string("fz_group_create: ") + cudaGetErrorString(e));
    fz_group_destroy(g);
    return rc;
  }
  *out = g;
  return FZ_OK;
}

int fz_group_run(fz_group* g, int64_t nsteps) {
  fz_range nvtx_range("fz_group_run");
  if (!g || nsteps < 0) return fzi::set_global_error(FZ_EINVAL, "fz_group_run: bad arguments");
  cudaSetDevice(g->device);
  for (fz_handle* h : g->m)
    if (h->profiling) return fzi::set_global_error(FZ_EINVAL, "fz_group_run: a member has profiling enabled");
  const int G = g->graph_steps;
  int64_t done = 0;
  if (nsteps >= G) {
    int rc = order_after(g, false);  // the group starts after the members' earlier work
    if (rc != FZ_OK) return rc;
    while (nsteps - done >= G) {
      std::vector<int> key;
      for (fz_handle* h : g->m) key.push_back(h->i0);
      auto it = g->graphs.find(key);
      if (it == g->graphs.end()) {
        cudaGraphExec_t ge = nullptr;
        rc = capture(g, &ge);  // G is even: the members' host-side rotation is back where it was
        if (rc != FZ_OK) return rc;
        it = g->graphs.emplace(key, ge).first;
      }
      FZ_GCUDA(g, cudaGraphLaunch(it->second, g->stream), "group graph launch");
      for (fz_handle* h : g->m) h->steps_enqueued += G;
      done += G;
    }
    rc = order_after(g, true);  // later work on a member (fz_sync, fz_get_ir, fz_run) follows
    if (rc != FZ_OK) return rc;
  }
  for (; done < nsteps; done++)
    for (fz_handle* h : g->m) {
      const cudaError_t e = fzi::enqueue(h);
      if (e != cudaSuccess) return fzi::cuda_fail(h, e, "group step launch");
      h->steps_enqueued += 1;
    }
  return FZ_OK;
}

int fz_group_autotune(fz_group* g, int32_t reps, int32_t* kz_chunk, double* ms_per_step) {
  if (!g) return fzi::set_global_error(FZ_EINVAL, "fz_group_autotune: NULL group");
  int rc = fz_group_sync(g, 0);
  if (rc != FZ_OK) return rc;
  cudaSetDevice(g->device);
  // one depth for every member (clamped to each room's planes), or 0: each member's own heuristic
  int nzmax = 1;
  for (fz_handle* h : g->m) nzmax = std::max(nzmax, h->Nz - 2 * fz::GHOST);
  std::vector<fzi::ZPlan> cand{{0, 0}};
  for (int c : {4, 6, 8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256})
    if (c <= nzmax) cand.push_back({c, 0});
  fzi::ZPlan best{0, 0};
  rc = fzi::tune(g->m, g->stream, cand, reps, &best, ms_per_step);
  for (auto& kv : g->graphs) cudaGraphExecDestroy(kv.second);  // captured with the old launch shape
  g->graphs.clear();
  if (rc != FZ_OK) return rc;
  if (kz_chunk) *kz_chunk = best.depth;
  return FZ_OK;
}

int fz_group_sync(fz_group* g, int64_t timeout_ms) {
  if (!g) return fzi::set_global_error(FZ_EINVAL, "fz_group_sync: NULL group");
  if (timeout_ms <= 0) timeout_ms = 600000;
  cudaSetDevice(g->device);
  const auto t0 = std::chrono::steady_clock::now();
  int sleep_us = 20;
  for (;;) {
    const cudaError_t e = cudaStreamQuery(g->stream);
    if (e == cudaSuccess) break;
    if (e != cudaErrorNotReady) return gfail(g, e, "group stream");
    const auto ms =
        std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0).count();
    if (ms > timeout_ms) return fzi::set_global_error(FZ_ETIMEOUT, "fz_group_sync: device work did not finish in time");
    std::this_thread::sleep_for(std::chrono::microseconds(sleep_us));
    sleep_us = std::min(sleep_us * 2, 2000);
  }
  for (fz_handle* h : g->m) {  // each member's own stream and device error word
    const int rc = fz_sync(h, timeout_ms);
    if (rc != FZ_OK) return rc;
  }
  return FZ_OK;
}

int fz_group_run_timed(fz_group* g, int64_t nsteps, double* ms) {
  if (!g || !ms) return fzi::set_global_error(FZ_EINVAL, "fz_group_run_timed: NULL argument");
  int rc = fz_group_sync(g, 0);
  if (rc != FZ_OK) return rc;
  cudaSetDevice(g->device);
  cudaEvent_t a = nullptr, b = nullptr;
  FZ_GCUDA(g, cudaEventCreate(&a), "event");
  cudaError_t e = cudaEventCreate(&b);
  if (e != cudaSuccess) {
    cudaEventDestroy(a);
    return gfail(g, e, "event");
  }
  // the group stream waits for every member before the first event and every member finishes
  // before the second, so the interval covers the whole run even for the ungraphed remainder
  rc = order_after(g, false);
  if (rc == FZ_OK) rc = (cudaEventRecord(a, g->stream) == cudaSuccess) ? FZ_OK : FZ_ECUDA;
  if (rc == FZ_OK) rc = fz_group_run(g, nsteps);
  if (rc == FZ_OK) rc = order_after(g, false);
  if (rc == FZ_OK) rc = (cudaEventRecord(b, g->stream) == cudaSuccess) ? FZ_OK : FZ_ECUDA;
  if (rc == FZ_OK) rc = fz_group_sync(g, 0);
  if (rc == FZ_OK) {
    float x = 0.f;
    e = cudaEventElapsedTime(&x, a, b);
    if (e == cudaSuccess) *ms = x; else rc = gfail(g, e, "event elapsed");
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return rc;
}

}  // extern "C"
