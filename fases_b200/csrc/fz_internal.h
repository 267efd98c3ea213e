// fz_internal.h -- host-side state of a solver handle (private to libfz.so).
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/fz.h"
#include "fz_device.cuh"

// NVTX range over a scope (host timeline markers for nsys / ncu; no cost without a tool attached)
struct fz_range {
  explicit fz_range(const char* name) { nvtxRangePushA(name); }
  ~fz_range() { nvtxRangePop(); }
  fz_range(const fz_range&) = delete;
  fz_range& operator=(const fz_range&) = delete;
};

struct fz_timing_rec {
  int kind;
  cudaEvent_t a, b;
};

struct fz_handle {
  fz_params prm{};
  std::string err;
  int device = 0;
  int nsm = 0;
  cudaStream_t stream = nullptr;
  bool fp64 = false;
  size_t rsize = 4;  // sizeof(real)

  // grid
  int Nx = 0, Ny = 0, Nz = 0;
  int64_t Sx = 0, plane = 0, ncell_dev = 0;
  double Lx = 0, Ly = 0, Lz = 0;  // padded domain size for header.txt
  bool have_geometry = false;
  std::vector<float> S_host;
  std::vector<uint8_t> oid_host;
  int64_t n_update = 0;
  // batch members: independent field sets stacked along z, member m at offset m * ncell_dev
  int nb = 1;

  // device fields: U[set][field], set 0..2, field p,u,v,w
  void* U[3][4] = {{nullptr}};
  int i0 = 0, i1 = 1, i2 = 2;
  uint8_t* d_cls = nullptr;
  std::vector<uint8_t> cls_host;

  // cPML
  bool pml_on = false;
  void* d_pml_coef[3] = {nullptr, nullptr, nullptr};
  void* d_psi[3] = {nullptr, nullptr, nullptr};

  // immersed band
  int64_t nB = 0;   // band records of all members (nB1 * nb)
  int64_t nB1 = 0;  // band cells of one member
  std::vector<int64_t> band_cell_ref;  // reference-layout cell index (for the material check)
  std::vector<int32_t> band_mat;
  int4* d_brec = nullptr;  // cell index (lo, hi), corner - cell, material
  void* d_bgeo = nullptr;
  void* d_bnrm = nullptr;
  double* d_ade[3][3] = {{nullptr}};  // [set][phi, psi1, psi2]
  int ph_old = 0, ph_cur = 1, ph_nu = 2;

  // materials
  int nMat = 0, K = 1, L = 1;
  std::vector<double> Rinf, A, zeta, B, C, alpha, beta;
  double* d_mat = nullptr;  // packed: Rinf | A | zeta | B | C | alpha | beta
  bool have_materials = false;

  // sources
  int nsrc = 0;
  std::vector<int32_t> src_ijk;
  std::vector<double> src_val, src_freq, u_s;
  int src_opt = 0;
  std::vector<int32_t> src_member;  // per source: member index, -1 = every member
  int nsrc_dev = 0;                 // device source records (sources x their members)
  int64_t* d_src_cell = nullptr;
  void* d_src_coef = nullptr;
  void* d_src_freq = nullptr;
  void* d_us = nullptr;
  int64_t n_us = 0;

  // receivers
  int nrec = 0;
  std::vector<int32_t> rec_ijk;
  int64_t rec_cap = 0;
  int64_t* d_rec_cell = nullptr;
  double* d_ir = nullptr;
  double* d_vel = nullptr;

  // animation slices (planes x = sl_i, y = sl_j, z = sl_k) every sl_step steps, up to sl_cap frames
  bool sl_on = false;
  int sl_i = 0, sl_j = 0, sl_k = 0;
  int64_t sl_step = 1, sl_cap = 0, sl_frame = 0;  // sl_frame: floats per frame
  float* d_slices = nullptr;

  // TMA descriptors: halo tiles of p, u, v and own tiles of p, u, v, w of each field set, and
  // the class bytes
  CUtensorMap halo_map[3][3];
  CUtensorMap own_map[3][4];
  CUtensorMap cls_map;
  // device error word written by kernels whose bounded waits gave up
  int32_t* d_err = nullptr;

  // step counter and bookkeeping
  int64_t* d_step = nullptr;
  double* d_scratch = nullptr;
  int64_t steps_enqueued = 0;
  bool finalized = false;
  int kz_chunk = 0;       // largest z chunk of the stage kernels
  int kz_heuristic = 0;  // the wave-filling choice of prepare (fz_set_kz_chunk(h, 0) returns to it)
  int zchunks = 1;       // z chunks per member
  std::vector<int> zsizes;  // their lengths in planes (sum = interior planes), longest first
  int stage_occ = 1;        // stage-kernel CTAs per SM
  dim3 stage_grid;

  // wait-test build: plane of each z chunk whose tile the stage kernels never issue (-1: none)
  int test_skip_plane = -1;

  // counts the events that invalidate captured launches (new launch shape, reallocated or rebound
  // arrays): a group compares it with the value its argument tables were built at
  uint64_t launch_gen = 0;

  // graphs, keyed by buffer parity
  int graph_steps = 10;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};

  // profiling
  bool profiling = false;
  std::vector<fz_timing_rec> timings;
  double prof_ms[8] = {0};
  int64_t prof_n[8] = {0};

  // output bookkeeping
  std::string scene_name;
};

namespace fzi {
int set_error(fz_handle* h, int code, const std::string& msg);
int set_global_error(int code, const std::string& msg);
int cuda_fail(fz_handle* h, cudaError_t e, const char* what);
// one cPML table entry of an axis of N cells (lo / hi: faces enabled): the psi tile index (-1
// outside the layer), the values (1/kappa - 1, b, ca) and d[value][param], the derivatives with
// respect to (pml_R0, pml_kappa_max, pml_alpha_max)
struct PmlEntry {
  int tile;
  double v[3];
  double d[3][3];
};
void pml_entry(const fz_params& p, int N, int lo, int hi, int i, PmlEntry* out);
// finalises the handle's setup (materials, sources, receivers, launch geometry); idempotent
int prepare(fz_handle* h);
// enqueues one time step on the handle's stream (or into the capture the stream takes part in)
cudaError_t enqueue(fz_handle* h);
// the parts of one step: stage st (stage kernel + band), then receivers and buffer rotation
cudaError_t enqueue_stage(fz_handle* h, int st);
cudaError_t enqueue_finish(fz_handle* h);
// points field set `set` at the four arrays f (same size and layout as the handle's own) and
// re-encodes its TMA maps; kernels already launched keep the maps they were launched with
int bind_field_set(fz_handle* h, int set, void* const* f);
// the stage kernel of stage st alone (no band), on the handle's stream: the autotuner's trial
cudaError_t enqueue_stage_kernel(fz_handle* h, int st);
// tile depth of the stage kernels (z planes per CTA; 0 = the wave-filling heuristic); drops the
// handle's captured graphs
void set_kz_chunk(fz_handle* h, int kz_chunk);
// z chunks of any lengths (summing to the interior planes, at most FZ_MAX_ZCHUNKS); drops graphs
int set_z_sizes(fz_handle* h, const std::vector<int>& sizes);
// a guided schedule: chunks of `depth` planes, then about one wave of CTAs at depth/2 and one at
// depth/4, so the last waves are short
std::vector<int> guided_z_sizes(fz_handle* h, int depth);
// Times the stage kernels of every handle in hs (launched on their own streams, forked from and
// joined to `ts`) for each candidate tile depth (0 = each handle's heuristic; others are clamped
// to a handle's planes) and leaves every handle on the fastest; the state is left as it was.
// A candidate launch shape: uniform z chunks of `depth` planes (0 = each handle's heuristic), or,
// with guided set, the guided schedule of that depth.
struct ZPlan {
  int depth;
  int guided;
};
// Custom trial of a tuning run (the group path times its one-launch-per-kind stage kernels):
// on_plan runs after each candidate has been applied to every handle, round(n) enqueues n steps'
// stage kernels on the tuning stream.
struct TuneHooks {
  std::function<int()> on_plan;
  std::function<cudaError_t(int)> round;
};
int tune(const std::vector<fz_handle*>& hs, cudaStream_t ts, const std::vector<ZPlan>& candidates, int reps,
         ZPlan* best, double* ms_per_step, const TuneHooks* hooks = nullptr);
// apply a candidate to one handle
int apply_z_plan(fz_handle* h, const ZPlan& p);
// Launch arguments of the handle's kernels for its current buffer roles (the group path lays the
// arguments of several handles side by side in device memory): stage st's kernel and TMA
// descriptors, stage st's band kernel, the receiver gather; rotate() advances the roles by one step
// as enqueue_finish does.
template <class R>
void stage_desc(fz_handle* h, int st, fz::StageArgs<R>* a, fz::StageMaps* m);
template <class R>
void band_desc(fz_handle* h, int st, fz::BandArgs<R>* b);
template <class R>
void rec_desc(fz_handle* h, fz::RecArgs<R>* r);
void rotate(fz_handle* h);
// the launch shapes worth timing for one handle: the heuristic, the best-filling uniform depths and
// guided schedules of the best of them
std::vector<ZPlan> kz_candidates(fz_handle* h);
}  // namespace fzi
