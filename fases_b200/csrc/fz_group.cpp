// fz_group.cpp -- several solver handles (rooms) advanced together. Small rooms leave most of the
// GPU idle when stepped one after another. Rooms of one precision (3D, without animation slices,
// up to FZ_MAX_GROUP) share their launches: per stage one band launch over all members and one
// stage launch per FZ_GROUP_LAUNCH members, their CTAs laid end to end (fz_kernels.cu,
// k_stage_group), from argument tables in device memory, then one receiver launch; runs of
// graph_steps steps are CUDA graphs of these launches. Other groups run each member's own launches as parallel branches of
// one graph per run.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "fz_internal.h"
#include "fz_kernels.h"

// Launch arguments of every member for one buffer-parity key. Device memory holds [3 stages][n]
// stage arguments, [3][n] band arguments and [n] receiver arguments side by side, members ordered
// by branch; each branch's stage launches' kernel parameters (each covering up to FZ_GROUP_LAUNCH
// members, with their TMA descriptors) and its band launches' parameters are kept on the host.
struct FlatBranch {
  std::vector<char> gstage[3];  // GroupStageArgs<R> of each stage launch, one per member chunk
  std::vector<int> chunk_ctas;  // CTAs of each chunk's stage launch
  std::vector<char> gband;      // GroupBandArgs<R> per stage
  int band_blocks = 0;          // band blocks of the branch's members
  int band_fit = 0;             // pole-count form of the band kernel (2, 4 or 0 = general)
  size_t rec_off = 0;           // the branch's receiver arguments in the device buffer
  int n = 0;                    // members in the branch
};

struct FlatTables {
  void* dev = nullptr;
  std::vector<FlatBranch> br;
  std::vector<uint64_t> gen;  // the members' launch_gen when the tables were built
  int nbranch = 0;            // the branch count they were built for
};

struct fz_group {
  std::vector<fz_handle*> m;
  int device = 0;
  int graph_steps = 10;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr, done = nullptr;
  std::vector<cudaEvent_t> join;
  // keyed by the members' buffer parities (the field-set rotation repeats every 2 steps)
  std::map<std::vector<int>, cudaGraphExec_t> graphs;
  // shared launches for all members (3D rooms of one precision, no animation slices, at most
  // FZ_MAX_GROUP); otherwise each member's own launches are branches of the graph
  bool flat = false;
  bool flat_ok = false;  // the members can share launches
  bool fp64 = false;
  std::map<std::vector<int>, FlatTables> tables;
  // shared launches run as `nbranch` concurrent branches (streams), each over a set of members of
  // about equal cells, so one branch's band and receiver launches overlap another's stage launch
  int nbranch = 1;
  std::vector<int> branch_of;  // branch of each member
  std::vector<cudaStream_t> bstream;
  std::vector<cudaEvent_t> bjoin;
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

std::vector<int> parity_key(const fz_group* g) {
  std::vector<int> key;
  for (const fz_handle* h : g->m) key.push_back(h->i0);
  return key;
}

void free_tables(fz_group* g) {
  for (auto& kv : g->tables)
    if (kv.second.dev) cudaFree(kv.second.dev);
  g->tables.clear();
}

void drop_graphs(fz_group* g) {
  for (auto& kv : g->graphs) cudaGraphExecDestroy(kv.second);
  g->graphs.clear();
}

// Branches of a group of n rooms unless set (fz_group_set_branches).
int default_branches(int n) { return n >= 16 ? 4 : n >= 4 ? 2 : 1; }

// Members into branches of about equal cells (largest first into the lightest branch).
void assign_branches(fz_group* g, int nbranch) {
  const int n = (int)g->m.size();
  nbranch = std::max(1, std::min(nbranch, n));
  std::vector<int> idx(n);
  for (int q = 0; q < n; q++) idx[q] = q;
  auto cells = [&](int q) { return (int64_t)g->m[(size_t)q]->ncell_dev * g->m[(size_t)q]->nb; };
  std::sort(idx.begin(), idx.end(), [&](int a, int b) { return cells(a) > cells(b); });
  std::vector<int64_t> load((size_t)nbranch, 0);
  g->branch_of.assign((size_t)n, 0);
  for (int q : idx) {
    const int b = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    g->branch_of[(size_t)q] = b;
    load[(size_t)b] += cells(q);
  }
  g->nbranch = nbranch;
}

// The launch arrangement: -1 each member's own launches as graph branches; 0 the default (shared
// launches in default_branches() branches where the members can share launches); b >= 1 shared
// launches in b branches.
void set_mode(fz_group* g, int mode) {
  const int n = (int)g->m.size();
  if (mode == 0) mode = g->flat_ok ? default_branches(n) : -1;
  g->flat = g->flat_ok && mode > 0;
  assign_branches(g, g->flat ? std::min(mode, std::min(n, 16)) : 1);
}

// Streams and join events of the branches (the group stream is branch 0's).
int ensure_branch_streams(fz_group* g) {
  while ((int)g->bstream.size() < g->nbranch) {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    FZ_GCUDA(g, cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "branch stream");
    const cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) {
      cudaStreamDestroy(st);
      return gfail(g, e, "branch event");
    }
    g->bstream.push_back(st);
    g->bjoin.push_back(ev);
  }
  return FZ_OK;
}

cudaStream_t branch_stream(const fz_group* g, int b) { return b == 0 ? g->stream : g->bstream[(size_t)b]; }

// Builds (or checks) the flat tables of the members' current roles. When a member's launches
// changed since the tables were uploaded (a new launch shape, reallocated or rebound arrays: its
// launch_gen moved) or the branches changed, the tables are built again, and every captured graph
// goes, since graphs hold the old kernel parameters.
template <class R>
int flat_tables(fz_group* g, const std::vector<int>& key) {
  const int n = (int)g->m.size();
  std::vector<uint64_t> gen;
  for (const fz_handle* h : g->m) gen.push_back(h->launch_gen);
  auto it = g->tables.find(key);
  if (it != g->tables.end() && it->second.gen == gen && it->second.nbranch == g->nbranch) return FZ_OK;
  FlatTables t;
  t.gen = gen;
  t.nbranch = g->nbranch;
  // members in branch order: position q of the device arrays holds member order[q]
  std::vector<int> order;
  for (int b = 0; b < g->nbranch; b++)
    for (int q = 0; q < n; q++)
      if (g->branch_of[(size_t)q] == b) order.push_back(q);
  const size_t stage_bytes = sizeof(fz::StageArgs<R>) * n;
  const size_t off_band = ((3 * stage_bytes + 127) / 128) * 128;
  const size_t band_bytes = sizeof(fz::BandArgs<R>) * n;
  const size_t off_rec = off_band + ((3 * band_bytes + 127) / 128) * 128;
  std::vector<char> host(off_rec + sizeof(fz::RecArgs<R>) * n, 0);
  std::vector<fz::StageMaps> maps((size_t)3 * n);
  for (int q = 0; q < n; q++) {
    fz_handle* h = g->m[(size_t)order[(size_t)q]];
    for (int st = 0; st < 3; st++) {
      fzi::stage_desc<R>(h, st, reinterpret_cast<fz::StageArgs<R>*>(host.data() + st * stage_bytes) + q,
                         &maps[(size_t)st * n + q]);
      fzi::band_desc<R>(h, st, reinterpret_cast<fz::BandArgs<R>*>(host.data() + off_band + st * band_bytes) + q);
    }
    fzi::rec_desc<R>(h, reinterpret_cast<fz::RecArgs<R>*>(host.data() + off_rec) + q);
  }
  drop_graphs(g);
  if (it != g->tables.end()) {
    // launches still queued may read the old tables: a new buffer, the old one freed when idle
    FZ_GCUDA(g, cudaDeviceSynchronize(), "group tables");
    cudaFree(it->second.dev);
    g->tables.erase(it);
  }
  FZ_GCUDA(g, cudaMalloc(&t.dev, host.size()), "group tables");
  FZ_GCUDA(g, cudaMemcpy(t.dev, host.data(), host.size(), cudaMemcpyHostToDevice), "group tables upload");
  char* d = (char*)t.dev;
  int q0 = 0;
  for (int b = 0; b < g->nbranch; b++) {
    FlatBranch fb;
    int q1 = q0;
    while (q1 < n && g->branch_of[(size_t)order[(size_t)q1]] == b) q1++;
    fb.n = q1 - q0;
    fb.rec_off = off_rec + sizeof(fz::RecArgs<R>) * q0;
    // band: one launch over the branch's members
    std::vector<fz::GroupBandArgs<R>> gb(3);
    int blocks = 0, kmax = 0, lmax = 0;
    for (int q = q0; q < q1; q++) {
      const fz_handle* h = g->m[(size_t)order[(size_t)q]];
      for (int st = 0; st < 3; st++) gb[st].blk_start[q - q0] = blocks;
      blocks += (int)((h->nB + 255) / 256);
      if (h->nB > 0) {
        kmax = std::max(kmax, h->K);
        lmax = std::max(lmax, h->L);
      }
    }
    for (int st = 0; st < 3; st++) {
      gb[st].n = fb.n;
      gb[st].blk_start[fb.n] = blocks;
      gb[st].args = reinterpret_cast<const fz::BandArgs<R>*>(d + off_band + st * band_bytes) + q0;
    }
    fb.band_blocks = blocks;
    fb.band_fit = (kmax <= 2 && lmax <= 2) ? 2 : (kmax <= 4 && lmax <= 4) ? 4 : 0;
    fb.gband.assign((const char*)gb.data(), (const char*)(gb.data() + 3));
    // stage launches: the branch's members in chunks of at most FZ_GROUP_LAUNCH, as even as possible
    const int nchunk = (fb.n + fz::FZ_GROUP_LAUNCH - 1) / fz::FZ_GROUP_LAUNCH;
    for (int c = 0; c < nchunk; c++) {
      const int m0 = q0 + (int)((int64_t)fb.n * c / nchunk), m1 = q0 + (int)((int64_t)fb.n * (c + 1) / nchunk);
      int ctas = 0;
      for (int st = 0; st < 3; st++) {
        fz::GroupStageArgs<R> ga;
        std::memset(&ga, 0, sizeof(ga));
        ga.args = reinterpret_cast<const fz::StageArgs<R>*>(d + st * stage_bytes) + m0;
        ga.n = m1 - m0;
        ctas = 0;
        for (int q = m0; q < m1; q++) {
          const dim3 gr = g->m[(size_t)order[(size_t)q]]->stage_grid;
          ga.maps[q - m0] = maps[(size_t)st * n + q];
          ga.cta_start[q - m0] = ctas;
          ga.gx[q - m0] = (int)gr.x;
          ga.gy[q - m0] = (int)gr.y;
          ctas += (int)(gr.x * gr.y * gr.z);
        }
        ga.cta_start[m1 - m0] = ctas;
        const char* bp = reinterpret_cast<const char*>(&ga);
        fb.gstage[st].insert(fb.gstage[st].end(), bp, bp + sizeof(ga));
      }
      fb.chunk_ctas.push_back(ctas);
    }
    t.br.push_back(std::move(fb));
    q0 = q1;
  }
  g->tables.emplace(key, std::move(t));
  return FZ_OK;
}

// Tables for the current roles and for the roles one step later (a graph covers both).
int ensure_flat_tables(fz_group* g) {
  int rc = ensure_branch_streams(g);
  if (rc != FZ_OK) return rc;
  for (int flip = 0; flip < 2; flip++) {
    rc = g->fp64 ? flat_tables<double>(g, parity_key(g)) : flat_tables<float>(g, parity_key(g));
    for (fz_handle* h : g->m) fzi::rotate(h);
    if (rc != FZ_OK) {
      if (flip == 0)
        for (fz_handle* h : g->m) fzi::rotate(h);
      return rc;
    }
  }
  return FZ_OK;  // rotated twice: back where it was
}

// Every branch's stream waits for the group stream (fork), and the group stream for every branch
// (join).
cudaError_t branches_fork(fz_group* g) {
  if (g->nbranch <= 1) return cudaSuccess;
  cudaError_t e = cudaEventRecord(g->fork, g->stream);
  for (int b = 1; b < g->nbranch && e == cudaSuccess; b++) e = cudaStreamWaitEvent(g->bstream[(size_t)b], g->fork, 0);
  return e;
}
cudaError_t branches_join(fz_group* g) {
  cudaError_t e = cudaSuccess;
  for (int b = 1; b < g->nbranch && e == cudaSuccess; b++) {
    e = cudaEventRecord(g->bjoin[(size_t)b], g->bstream[(size_t)b]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(g->stream, g->bjoin[(size_t)b], 0);
  }
  return e;
}

template <class R>
cudaError_t flat_stage_launches(fz_group* g, const FlatBranch& fb, int st, cudaStream_t s) {
  const fz::GroupStageArgs<R>* gs = reinterpret_cast<const fz::GroupStageArgs<R>*>(fb.gstage[st].data());
  for (size_t c = 0; c < fb.chunk_ctas.size(); c++) {
    const cudaError_t e = fz::launch_stage_group<R>(st, gs[c], fb.chunk_ctas[c], s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// The stage and band kernels of every member for the current roles, n times, on the branches: the
// autotuner's trial of the shared-launch path. The band kernels write only band cells of the stage
// outputs and the ADE sets the next real step writes before it reads them, so a trial changes
// nothing the solve goes on from (the tuner restores the rest).
template <class R>
cudaError_t flat_trial_kernels(fz_group* g, const FlatTables& t, int n) {
  cudaError_t e = branches_fork(g);
  for (int b = 0; b < g->nbranch && e == cudaSuccess; b++) {
    const FlatBranch& fb = t.br[(size_t)b];
    const fz::GroupBandArgs<R>* gb = reinterpret_cast<const fz::GroupBandArgs<R>*>(fb.gband.data());
    for (int r = 0; r < n && e == cudaSuccess; r++)
      for (int st = 0; st < 3 && e == cudaSuccess; st++) {
        e = flat_stage_launches<R>(g, fb, st, branch_stream(g, b));
        if (e == cudaSuccess) e = fz::launch_band_group<R>(st, gb[st], fb.band_blocks, fb.band_fit, branch_stream(g, b));
      }
  }
  if (e == cudaSuccess) e = branches_join(g);
  return e;
}

// The same trial for each member's own launches, side by side on the members' streams.
cudaError_t member_trial_kernels(fz_group* g, int n) {
  cudaError_t e = cudaEventRecord(g->fork, g->stream);
  for (size_t q = 0; q < g->m.size() && e == cudaSuccess; q++) {
    fz_handle* h = g->m[q];
    e = cudaStreamWaitEvent(h->stream, g->fork, 0);
    for (int r = 0; r < n && e == cudaSuccess; r++)
      for (int st = 0; st < 3 && e == cudaSuccess; st++) e = fzi::enqueue_stage(h, st);
    if (e == cudaSuccess) e = cudaEventRecord(g->join[q], h->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(g->stream, g->join[q], 0);
  }
  return e;
}

// nsteps steps of every member: each branch on its stream runs, per step and stage, its stage
// launches and one band launch, then one receiver launch; the members' roles advance as
// enqueue_finish advances them. Branches depend on nothing of each other within the run.
template <class R>
cudaError_t flat_steps(fz_group* g, int nsteps) {
  cudaError_t e = branches_fork(g);
  for (int s = 0; s < nsteps && e == cudaSuccess; s++) {
    auto it = g->tables.find(parity_key(g));
    if (it == g->tables.end()) return cudaErrorInvalidValue;  // built by ensure_flat_tables first
    const FlatTables& t = it->second;
    for (int b = 0; b < g->nbranch && e == cudaSuccess; b++) {
      const FlatBranch& fb = t.br[(size_t)b];
      const cudaStream_t bs = branch_stream(g, b);
      const fz::GroupBandArgs<R>* gb = reinterpret_cast<const fz::GroupBandArgs<R>*>(fb.gband.data());
      for (int st = 0; st < 3 && e == cudaSuccess; st++) {
        e = flat_stage_launches<R>(g, fb, st, bs);
        if (e == cudaSuccess) e = fz::launch_band_group<R>(st, gb[st], fb.band_blocks, fb.band_fit, bs);
      }
      if (e == cudaSuccess)
        e = fz::launch_receivers_group<R>(reinterpret_cast<const fz::RecArgs<R>*>((const char*)t.dev + fb.rec_off),
                                          fb.n, bs);
    }
    for (fz_handle* h : g->m) fzi::rotate(h);
  }
  if (e == cudaSuccess) e = branches_join(g);
  return e;
}

cudaError_t flat_enqueue(fz_group* g, int nsteps) {
  return g->fp64 ? flat_steps<double>(g, nsteps) : flat_steps<float>(g, nsteps);
}

int capture(fz_group* g, cudaGraphExec_t* out) {
  cudaGraph_t graph = nullptr;
  FZ_GCUDA(g, cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
  cudaError_t e = cudaEventRecord(g->fork, g->stream);
  if (g->flat && e == cudaSuccess) e = flat_enqueue(g, g->graph_steps);
  for (size_t i = 0; i < g->m.size() && e == cudaSuccess && !g->flat; i++) {
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
  free_tables(g);
  for (size_t b = 0; b < g->bstream.size(); b++) {
    if (g->bstream[b]) {
      cudaStreamSynchronize(g->bstream[b]);
      cudaStreamDestroy(g->bstream[b]);
    }
    if (g->bjoin[b]) cudaEventDestroy(g->bjoin[b]);
  }
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
  g->fp64 = members[0]->fp64;
  g->flat_ok = n <= fz::FZ_MAX_GROUP;
  for (fz_handle* h : g->m)
    if (h->fp64 != g->fp64 || h->prm.two_d || h->sl_on) g->flat_ok = false;
  set_mode(g, 0);
  g->bstream.push_back(nullptr);  // branch 0 runs on the group stream
  g->bjoin.push_back(nullptr);
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

int fz_group_info(fz_group* g, int32_t* shared, int32_t* branches) {
  if (!g || !shared) return fzi::set_global_error(FZ_EINVAL, "fz_group_info: NULL argument");
  *shared = g->flat ? 1 : 0;
  if (branches) *branches = g->flat ? g->nbranch : (int32_t)g->m.size();
  return FZ_OK;
}

int fz_group_set_branches(fz_group* g, int32_t branches) {
  if (!g || branches < -1) return fzi::set_global_error(FZ_EINVAL, "fz_group_set_branches: bad arguments");
  if (branches > 0 && !g->flat_ok)
    return fzi::set_global_error(FZ_EINVAL, "fz_group_set_branches: these members cannot share launches "
                                            "(2D rooms, animation slices, mixed precision or more than 64)");
  const int rc = fz_group_sync(g, 0);
  if (rc != FZ_OK) return rc;
  set_mode(g, branches);
  drop_graphs(g);  // tables follow on the next run (they record the branch count)
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
  if (g->flat) {
    if (nsteps == 0) return FZ_OK;
    int rc = ensure_flat_tables(g);
    if (rc == FZ_OK) rc = order_after(g, false);  // the group starts after the members' earlier work
    if (rc != FZ_OK) return rc;
    while (nsteps - done >= G) {
      const std::vector<int> key = parity_key(g);
      auto it = g->graphs.find(key);
      if (it == g->graphs.end()) {
        cudaGraphExec_t ge = nullptr;
        rc = capture(g, &ge);  // G is even: the members' roles are back where they were
        if (rc != FZ_OK) return rc;
        it = g->graphs.emplace(key, ge).first;
      }
      FZ_GCUDA(g, cudaGraphLaunch(it->second, g->stream), "group graph launch");
      for (fz_handle* h : g->m) h->steps_enqueued += G;
      done += G;
    }
    if (done < nsteps) {
      FZ_GCUDA(g, flat_enqueue(g, (int)(nsteps - done)), "group step launch");
      for (fz_handle* h : g->m) h->steps_enqueued += nsteps - done;
      done = nsteps;
    }
    return order_after(g, true);  // later work on a member (fz_sync, fz_get_ir, fz_run) follows
  }
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
  // the launch arrangements worth timing: each member's own launches side by side (-1) and, where
  // the members can share launches, shared launches in 1, 2, 4 or 8 branches
  std::vector<int> modes{-1};
  if (g->flat_ok)
    for (int b : {1, 2, 4, 8})
      if (b <= (int)g->m.size()) modes.push_back(b);
  fzi::ZPlan best{0, 0};
  int best_mode = -1;
  double best_ms = -1.0;
  for (int mode : modes) {
    set_mode(g, mode);
    fzi::ZPlan b{0, 0};
    double ms = 0.0;
    // trials: the stage and band kernels of every member in this arrangement (the overlap of one
    // room's band kernels with another's stage kernels is what tells the arrangements apart)
    fzi::TuneHooks hooks;
    if (g->flat) {
      hooks.on_plan = [g]() { return ensure_flat_tables(g); };
      hooks.round = [g](int nrep) -> cudaError_t {
        auto it = g->tables.find(parity_key(g));
        if (it == g->tables.end()) return cudaErrorInvalidValue;
        return g->fp64 ? flat_trial_kernels<double>(g, it->second, nrep) : flat_trial_kernels<float>(g, it->second, nrep);
      };
    } else {
      hooks.round = [g](int nrep) { return member_trial_kernels(g, nrep); };
    }
    rc = fzi::tune(g->m, g->stream, cand, reps, &b, &ms, &hooks);
    if (rc != FZ_OK) break;
    if (best_ms < 0.0 || ms < best_ms) {
      best_ms = ms;
      best = b;
      best_mode = mode;
    }
  }
  if (rc == FZ_OK) {
    set_mode(g, best_mode);
    for (fz_handle* h : g->m) {
      rc = fzi::apply_z_plan(h, best);
      if (rc != FZ_OK) break;
    }
  }
  drop_graphs(g);  // captured with the old launch shape
  if (rc != FZ_OK) return rc;
  if (kz_chunk) *kz_chunk = best.depth;
  if (ms_per_step) *ms_per_step = best_ms;
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
