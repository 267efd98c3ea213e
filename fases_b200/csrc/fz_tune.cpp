// fz_tune.cpp -- launch-shape autotuner of the stage kernels. The tile of a stage-kernel CTA is
// 32 x 16 columns by one z chunk of planes; the chunk lengths decide how many CTAs a stage
// launches (and so how whole waves of the 148 SMs fill), and each CTA pays about 1.5 planes of
// start-up work (two extra z centres, the TMA ring fill). prepare() picks a uniform depth from a
// wave-filling model; the tuner times the stage kernels of the real room for the uniform depths
// worth trying and for guided schedules (long chunks first, short ones for the last waves, so the
// start-up cost stays low without a long tail) and keeps the fastest. For a group of rooms the depths are timed with every member's kernels running side
// by side, as the group's graphs run them. The reference launches fixed TP(32,4,4) blocks
// (3D-solver/core/main3D.cu:1280-1306) and has no tuner.
//
// The trials launch the three stage kernels only. Their outputs land in the field sets U1 and U2,
// whose updated cells the next real step rewrites before reading; the cPML psi tiles (advanced by
// stage 2) and the output cells of sources in skipped cells (which accumulate) are saved before
// and restored after, so the solve continues exactly as it would have.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "fz_internal.h"

using fz::GHOST;

namespace {

struct Saved {
  std::vector<void*> psi_dev, psi_copy;
  std::vector<size_t> psi_bytes;
  // (field set, device index) of outputs that trials change and the next step reads
  std::vector<std::pair<void*, std::vector<char>>> cells;
};

int save_state(fz_handle* h, Saved& sv) {
  const int64_t d2 = 2 * (int64_t)h->prm.pml_cells;
  const int64_t tile_n[3] = {d2 * h->Ny * h->Nz * h->nb, (int64_t)h->Nx * d2 * h->Nz * h->nb,
                             (int64_t)h->Nx * h->Ny * d2 * h->nb};
  for (int a = 0; a < 3; a++) {
    if (!h->d_psi[a]) continue;
    const size_t b = (size_t)tile_n[a] * 2 * h->rsize;
    void* c = nullptr;
    cudaError_t e = cudaMalloc(&c, b);
    if (e != cudaSuccess) return fzi::cuda_fail(h, e, "autotune: psi copy");
    sv.psi_dev.push_back(h->d_psi[a]);
    sv.psi_copy.push_back(c);
    sv.psi_bytes.push_back(b);
    e = cudaMemcpy(c, h->d_psi[a], b, cudaMemcpyDeviceToDevice);
    if (e != cudaSuccess) return fzi::cuda_fail(h, e, "autotune: psi save");
  }
  if (h->nsrc_dev > 0) {
    std::vector<int64_t> cells((size_t)h->nsrc_dev);
    cudaError_t e = cudaMemcpy(cells.data(), h->d_src_cell, cells.size() * 8, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fzi::cuda_fail(h, e, "autotune: source cells");
    for (int64_t g : cells) {
      if (h->cls_host[(size_t)g] & fz::CLS_UPDATE) continue;
      for (int set : {h->i1, h->i2}) {
        char* p = (char*)h->U[set][0] + (size_t)g * h->rsize;
        std::vector<char> v(h->rsize);
        e = cudaMemcpy(v.data(), p, h->rsize, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return fzi::cuda_fail(h, e, "autotune: source cell save");
        sv.cells.emplace_back(p, v);
      }
    }
  }
  return FZ_OK;
}

int restore_state(fz_handle* h, Saved& sv) {
  cudaError_t e = cudaSuccess;
  for (size_t q = 0; q < sv.psi_dev.size() && e == cudaSuccess; q++)
    e = cudaMemcpy(sv.psi_dev[q], sv.psi_copy[q], sv.psi_bytes[q], cudaMemcpyDeviceToDevice);
  for (auto& c : sv.cells)
    if (e == cudaSuccess) e = cudaMemcpy(c.first, c.second.data(), c.second.size(), cudaMemcpyHostToDevice);
  for (void* c : sv.psi_copy) cudaFree(c);
  sv.psi_copy.clear();
  if (e != cudaSuccess) return fzi::cuda_fail(h, e, "autotune: restore");
  return FZ_OK;
}

}  // namespace

namespace fzi {

int apply_z_plan(fz_handle* h, const ZPlan& p) {
  if (p.guided) return set_z_sizes(h, guided_z_sizes(h, p.depth));
  set_kz_chunk(h, p.depth);
  return FZ_OK;
}

std::vector<ZPlan> kz_candidates(fz_handle* h) {
  const int nzi = h->Nz - 2 * GHOST;
  std::vector<ZPlan> out{{0, 0}};
  if (nzi <= 1) return out;
  // every distinct depth ceil(nzi / nk) of at least 4 planes, ranked by the heuristic's model
  const int occ = std::max(1, h->stage_occ);
  const int ntx = (h->Nx - 2 * GHOST + fz::TX - 1) / fz::TX;
  const int nty = (h->Ny - 2 * GHOST + fz::TY - 1) / fz::TY;
  const int64_t slots = (int64_t)h->nsm * occ;
  std::vector<std::pair<double, int>> ranked;
  int last = -1;
  for (int nk = 1; nk <= nzi; nk++) {
    const int c = (nzi + nk - 1) / nk;
    if (c < 4) break;
    if (c == last) continue;
    last = c;
    const int64_t items = (int64_t)ntx * nty * ((nzi + c - 1) / c) * h->nb;
    const int64_t waves = (items + slots - 1) / slots;
    ranked.push_back({((double)items / (double)(waves * slots)) * ((double)c / (c + 1.5)), c});
  }
  std::sort(ranked.begin(), ranked.end(), [](const std::pair<double, int>& a, const std::pair<double, int>& b) {
    return a.first > b.first || (a.first == b.first && a.second > b.second);
  });
  for (size_t q = 0; q < ranked.size() && out.size() < 9; q++)
    if (ranked[q].second != h->kz_heuristic) out.push_back({ranked[q].second, 0});
  // guided schedules: long chunks first, short ones for the last waves (single rooms; a batch's
  // members run one after another in the grid, so its tail is one member's)
  if (h->nb == 1)
    for (int D : {h->kz_heuristic, nzi / 2, nzi / 3, nzi / 4, 64, 48, 32})
      if (D >= 8 && D <= nzi) out.push_back({D, 1});
  return out;
}

int tune(const std::vector<fz_handle*>& hs, cudaStream_t ts, const std::vector<ZPlan>& candidates, int reps,
         ZPlan* best, double* ms_per_step, const TuneHooks* hooks) {
  if (hs.empty() || candidates.empty()) return set_global_error(FZ_EINVAL, "autotune: nothing to tune");
  reps = std::max(1, std::min(reps, 100));
  for (fz_handle* h : hs) {
    const int rc = fz_sync(h, 0);
    if (rc != FZ_OK) return rc;
  }
  cudaSetDevice(hs[0]->device);
  std::vector<Saved> saved(hs.size());
  for (size_t q = 0; q < hs.size(); q++) {
    const int rc = save_state(hs[q], saved[q]);
    if (rc != FZ_OK) {
      for (size_t r = 0; r <= q; r++) restore_state(hs[r], saved[r]);
      return rc;
    }
  }
  cudaEvent_t fork = nullptr, a = nullptr, b = nullptr;
  std::vector<cudaEvent_t> join(hs.size(), nullptr);
  cudaError_t e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreate(&a);
  if (e == cudaSuccess) e = cudaEventCreate(&b);
  for (size_t q = 0; q < hs.size() && e == cudaSuccess; q++) e = cudaEventCreateWithFlags(&join[q], cudaEventDisableTiming);
  // one round of `n` steps' stage kernels of every handle, side by side, forked from and joined to ts
  auto round = [&](int n) -> cudaError_t {
    if (hooks && hooks->round) return hooks->round(n);
    cudaError_t x = cudaEventRecord(fork, ts);
    for (size_t q = 0; q < hs.size() && x == cudaSuccess; q++) {
      fz_handle* h = hs[q];
      if (h->stream != ts) x = cudaStreamWaitEvent(h->stream, fork, 0);
      for (int r = 0; r < n && x == cudaSuccess; r++)
        for (int st = 0; st < 3 && x == cudaSuccess; st++) x = enqueue_stage_kernel(h, st);
      if (x == cudaSuccess && h->stream != ts) x = cudaEventRecord(join[q], h->stream);
      if (x == cudaSuccess && h->stream != ts) x = cudaStreamWaitEvent(ts, join[q], 0);
    }
    return x;
  };
  ZPlan chosen = candidates[0];
  double best_ms = -1.0;
  for (size_t c = 0; c < candidates.size() && e == cudaSuccess; c++) {
    for (fz_handle* h : hs) {
      const int rc = apply_z_plan(h, candidates[c]);
      if (rc != FZ_OK && e == cudaSuccess) e = cudaErrorInvalidValue;
    }
    if (e == cudaSuccess && hooks && hooks->on_plan && hooks->on_plan() != FZ_OK) e = cudaErrorInvalidValue;
    e = round(1);  // warm-up of this launch shape
    if (e == cudaSuccess) e = cudaEventRecord(a, ts);
    if (e == cudaSuccess) e = round(reps);
    if (e == cudaSuccess) e = cudaEventRecord(b, ts);
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    float x = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&x, a, b);
    if (e == cudaSuccess && (best_ms < 0.0 || x / reps < best_ms)) {
      best_ms = x / reps;
      chosen = candidates[c];
    }
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(ts);
  for (fz_handle* h : hs)
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (fork) cudaEventDestroy(fork);
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  for (cudaEvent_t j : join)
    if (j) cudaEventDestroy(j);
  for (fz_handle* h : hs) apply_z_plan(h, chosen);
  if (hooks && hooks->on_plan) hooks->on_plan();
  int rc = FZ_OK;
  for (size_t q = 0; q < hs.size(); q++) {
    const int r = restore_state(hs[q], saved[q]);
    if (rc == FZ_OK) rc = r;
  }
  if (e != cudaSuccess) return cuda_fail(hs[0], e, "autotune trial");
  if (rc != FZ_OK) return rc;
  for (fz_handle* h : hs) {  // a trial that ran into a bounded wait shows here
    const int r = fz_sync(h, 0);
    if (r != FZ_OK) return r;
  }
  if (best) *best = chosen;
  if (ms_per_step) *ms_per_step = best_ms;
  return FZ_OK;
}

}  // namespace fzi

extern "C" {

int fz_autotune(fz_handle* h, int32_t reps, int32_t* kz_chunk, double* ms_per_step) {
  fz_range nvtx_range("fz_autotune");
  if (!h) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  if (!h->have_geometry) return fzi::set_error(h, FZ_ESTATE, "fz_autotune before fz_load_geometry_raw");
  int rc = fzi::prepare(h);
  if (rc != FZ_OK) return rc;
  cudaSetDevice(h->device);
  fzi::ZPlan best{0, 0};
  rc = fzi::tune({h}, h->stream, fzi::kz_candidates(h), reps, &best, ms_per_step);
  if (rc != FZ_OK) return rc;
  if (kz_chunk) *kz_chunk = h->kz_chunk;
  return FZ_OK;
}

int fz_set_kz_chunk(fz_handle* h, int32_t kz_chunk) {
  if (!h) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  if (kz_chunk < 0) return fzi::set_error(h, FZ_EINVAL, "fz_set_kz_chunk: depth >= 0 (0 = heuristic)");
  if (!h->have_geometry) return fzi::set_error(h, FZ_ESTATE, "fz_set_kz_chunk before fz_load_geometry_raw");
  int rc = fzi::prepare(h);
  if (rc != FZ_OK) return rc;
  rc = fz_sync(h, 0);
  if (rc != FZ_OK) return rc;
  fzi::set_kz_chunk(h, kz_chunk);
  return FZ_OK;
}

int fz_get_z_schedule(fz_handle* h, int32_t* sizes, int32_t cap, int32_t* n) {
  if (!h) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  if (!h->have_geometry) return fzi::set_error(h, FZ_ESTATE, "fz_get_z_schedule before fz_load_geometry_raw");
  const int rc = fzi::prepare(h);
  if (rc != FZ_OK) return rc;
  if (n) *n = h->zchunks;
  if (sizes)
    for (int c = 0; c < h->zchunks && c < cap; c++) sizes[c] = h->zsizes[(size_t)c];
  return FZ_OK;
}

int fz_set_z_schedule(fz_handle* h, const int32_t* sizes, int32_t n) {
  if (!h) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  if (!sizes || n < 1) return fzi::set_error(h, FZ_EINVAL, "fz_set_z_schedule: sizes[n >= 1] required");
  if (!h->have_geometry) return fzi::set_error(h, FZ_ESTATE, "fz_set_z_schedule before fz_load_geometry_raw");
  int rc = fzi::prepare(h);
  if (rc != FZ_OK) return rc;
  rc = fz_sync(h, 0);
  if (rc != FZ_OK) return rc;
  return fzi::set_z_sizes(h, std::vector<int>(sizes, sizes + n));
}

int fz_get_kz_chunk(fz_handle* h, int32_t* kz_chunk, int32_t* heuristic) {
  if (!h) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  if (!h->have_geometry) return fzi::set_error(h, FZ_ESTATE, "fz_get_kz_chunk before fz_load_geometry_raw");
  const int rc = fzi::prepare(h);
  if (rc != FZ_OK) return rc;
  if (kz_chunk) *kz_chunk = h->kz_chunk;
  if (heuristic) *heuristic = h->kz_heuristic;
  return FZ_OK;
}

}  // extern "C"
