// fz_adjoint.cpp -- gradient of a receiver misfit (or a vector-Jacobian product of the receiver
// traces) with respect to the ADE material coefficients, the source strengths and waveform, the
// cPML profile parameters and the initial fields, by the discrete adjoint of the stepping scheme
// (kernels in fz_adjoint.cu). No counterpart in the reference: its material fit
// (common/fminconFIT.py:239-348) matches octave absorption in the frequency domain and never
// differentiates the time-domain solver.
//
// Schedule: one forward pass that saves the state (U0, the ADE "old" set, the cPML psi tiles)
// every `seg` steps; then, last segment first, restore the segment's checkpoint, recompute its
// steps while storing every stage input and ADE set, and sweep the segment backwards, three
// reversed stages per step (band adjoint, WENO-Z centre adjoint, gather).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "fz_adjoint.h"
#include "fz_internal.h"

using fz::GHOST;
using fz::XOFF;

namespace {

#define FZ_ACUDA(h, call, what)                                         \
  do {                                                                  \
    cudaError_t e__ = (call);                                           \
    if (e__ != cudaSuccess) return fzi::cuda_fail(h, e__, what);       \
  } while (0)

struct Arena {
  char* base = nullptr;
  size_t used = 0, cap = 0;
  void* take(size_t bytes) {
    const size_t a = (used + 255) & ~(size_t)255;
    if (a + bytes > cap) return nullptr;
    used = a + bytes;
    return base + a;
  }
};

size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

// One saved state: fields U0, ADE "old" set, psi tiles.
struct State {
  void* f[4] = {nullptr, nullptr, nullptr, nullptr};
  double* ade[3] = {nullptr, nullptr, nullptr};
  void* psi[3] = {nullptr, nullptr, nullptr};
};

template <class R>
int misfit_gradient(fz_handle* h, int64_t nsteps, int seg, const double* target, int64_t tsteps, double* J,
                    const fz_gradients& o, double* ms) {
  typedef typename fz::Pair<R>::T P;
  cudaStream_t s = h->stream;
  const int64_t N = h->ncell_dev;
  const size_t fb = (size_t)N * sizeof(R);
  const int64_t nB = h->nB;
  const int K = h->K, L = h->L;
  const int nMat = std::max(1, h->nMat);
  const int Pn = 1 + 2 * K + 4 * L;
  if (o.materials && o.materials_cap < (int64_t)nMat * Pn)
    return fzi::set_error(h, FZ_EINVAL, "fz_misfit_gradient: grad needs nMat*(1+2K+4L) = " +
                                            std::to_string((int64_t)nMat * Pn) + " elements");
  const int nsrc = h->nsrc_dev;
  const int64_t n_us = (h->src_opt == 2) ? 0 : h->n_us;
  const bool want_src = (o.source_sval || o.source_wave) && nsrc > 0;
  if (o.source_sval && o.source_sval_cap < h->nsrc)
    return fzi::set_error(h, FZ_EINVAL, "fz_misfit_gradient_ex: source_sval needs nsrc elements");
  if (o.source_wave && o.source_wave_cap < (int64_t)h->nsrc * n_us)
    return fzi::set_error(h, FZ_EINVAL, "fz_misfit_gradient_ex: source_wave needs nsrc * n_us elements");
  if (want_src && nsrc != h->nsrc)
    return fzi::set_error(h, FZ_EINVAL, "fz_misfit_gradient_ex: every source must belong to the solve");
  if (o.pml && o.pml_cap < 4) return fzi::set_error(h, FZ_EINVAL, "fz_misfit_gradient_ex: pml needs 4 elements");
  const bool want_pml = o.pml && h->pml_on;
  const int64_t nref = (int64_t)h->Nx * h->Ny * h->Nz;
  if (o.initial && o.initial_cap < 4 * nref)
    return fzi::set_error(h, FZ_EINVAL, "fz_misfit_gradient_ex: initial needs 4 * Nx * Ny * Nz elements");
  const size_t ade_b[3] = {(size_t)K * nB * 8, (size_t)L * nB * 8, (size_t)L * nB * 8};
  const int64_t d2 = 2 * (int64_t)h->prm.pml_cells;
  const int64_t tile_n[3] = {d2 * h->Ny * h->Nz, (int64_t)h->Nx * d2 * h->Nz, (int64_t)h->Nx * h->Ny * d2};
  size_t psi_b[3];
  for (int a = 0; a < 3; a++) psi_b[a] = h->d_psi[a] ? (size_t)tile_n[a] * sizeof(P) : 0;
  size_t ade_sum = 0, psi_sum = 0;
  for (int a = 0; a < 3; a++) {
    ade_sum += round256(ade_b[a]);
    psi_sum += round256(psi_b[a]);
  }
  const int64_t nseg = (nsteps + seg - 1) / seg;
  const size_t state_b = 4 * round256(fb) + ade_sum + psi_sum;
  const size_t seg_b = (size_t)seg * (3 * 4 * round256(fb) + 3 * ade_sum + (want_pml ? psi_sum : 0)) + ade_sum;
  const int d = h->prm.pml_cells;
  const size_t extra_b = round256((size_t)std::max(1, nsrc) * 8) * 2 + round256((size_t)std::max(1, nsrc) * std::max<int64_t>(1, n_us) * 8) +
                         round256((size_t)3 * 6 * d * 8);
  const size_t adj_b = 4 * 4 * round256(fb) + 4 * ade_sum + 2 * psi_sum +
                       round256((size_t)nMat * Pn * 8) + round256((size_t)Pn * nB * 8) + round256(4 * nB * sizeof(R)) +
                       round256((size_t)h->nrec * tsteps * 8);
  const size_t total = (size_t)(nseg + 1) * state_b + seg_b + adj_b + extra_b + 4096;
  size_t free_b = 0, tot_b = 0;
  FZ_ACUDA(h, cudaMemGetInfo(&free_b, &tot_b), "cudaMemGetInfo");
  if (total + ((size_t)256 << 20) > free_b)
    return fzi::set_error(h, FZ_ENOMEM, "fz_misfit_gradient: needs " + std::to_string(total >> 20) + " MiB, " +
                                            std::to_string(free_b >> 20) + " MiB free (shorten segment_steps)");
  Arena ar;
  ar.cap = total;
  FZ_ACUDA(h, cudaMalloc((void**)&ar.base, total), "cudaMalloc(adjoint)");
  struct Guard {
    char* p;
    ~Guard() { cudaFree(p); }
  } guard{ar.base};

  auto take_state = [&](State& st) {
    for (int f = 0; f < 4; f++) st.f[f] = ar.take(fb);
    for (int a = 0; a < 3; a++) st.ade[a] = (double*)ar.take(ade_b[a]);
    for (int a = 0; a < 3; a++) st.psi[a] = psi_b[a] ? ar.take(psi_b[a]) : nullptr;
  };
  std::vector<State> ck((size_t)nseg + 1);
  for (auto& st : ck) take_state(st);
  // per-step storage of one segment: stage inputs U0, U1, U2 and ADE sets phi^n, phi^(1), phi^(2),
  // phi^{n+1}; phi^n of step t > 0 is phi^{n+1} of step t - 1 (the same array)
  std::vector<void*> S[3];
  std::vector<double*> Ad[4][3];
  std::vector<void*> Ps[3];  // psi^n of every step of the segment (cPML gradient only)
  for (int t = 0; t < seg; t++) {
    for (int q = 0; q < 3; q++)
      for (int f = 0; f < 4; f++) S[q].push_back(ar.take(fb));
    for (int q = 1; q < 4; q++)
      for (int a = 0; a < 3; a++) Ad[q][a].push_back((double*)ar.take(ade_b[a]));
    for (int a = 0; a < 3; a++) Ad[0][a].push_back(t == 0 ? (double*)ar.take(ade_b[a]) : Ad[3][a][(size_t)t - 1]);
    if (want_pml)
      for (int a = 0; a < 3; a++) Ps[a].push_back(psi_b[a] ? ar.take(psi_b[a]) : nullptr);
  }
  R* lam[4][4];  // adjoint field sets A (carried), B, C, D
  for (int q = 0; q < 4; q++)
    for (int f = 0; f < 4; f++) lam[q][f] = (R*)ar.take(fb);
  double* lade[4][3];  // ADE adjoint sets: next, old, 1, 2
  for (int q = 0; q < 4; q++)
    for (int a = 0; a < 3; a++) lade[q][a] = (double*)ar.take(ade_b[a]);
  P* lpsi[2][3];  // adjoint of psi^{n+1} (read) and of psi^n (written), swapped every step
  for (int q = 0; q < 2; q++)
    for (int a = 0; a < 3; a++) lpsi[q][a] = psi_b[a] ? (P*)ar.take(psi_b[a]) : nullptr;
  double* d_grad = (double*)ar.take((size_t)nMat * Pn * 8);
  double* d_gcell = (double*)ar.take((size_t)Pn * nB * 8);
  R* d_probe = (R*)ar.take(4 * nB * sizeof(R));
  double* d_target = (double*)ar.take((size_t)h->nrec * tsteps * 8);
  double* d_sval = (double*)ar.take((size_t)std::max(1, nsrc) * 8);
  double* d_gsval = (double*)ar.take((size_t)std::max(1, nsrc) * 8);
  double* d_gwave = (double*)ar.take((size_t)std::max(1, nsrc) * std::max<int64_t>(1, n_us) * 8);
  double* d_gpml = (double*)ar.take((size_t)3 * 6 * d * 8);
  if (!d_gpml) return fzi::set_error(h, FZ_ENOMEM, "fz_misfit_gradient: arena layout overflow");

  // the handle's own field arrays by set and ADE arrays by role slot, put back after every
  // recompute (which points them at the segment storage)
  void* own[3][4];
  for (int q = 0; q < 3; q++)
    for (int f = 0; f < 4; f++) own[q][f] = h->U[q][f];
  double* own_ade[3][3];
  for (int r = 0; r < 3; r++)
    for (int a = 0; a < 3; a++) own_ade[r][a] = h->d_ade[r][a];
  auto unbind = [&]() -> int {
    for (int r = 0; r < 3; r++)
      for (int a = 0; a < 3; a++) h->d_ade[r][a] = own_ade[r][a];
    for (int q = 0; q < 3; q++) {
      const int rc = fzi::bind_field_set(h, q, own[q]);
      if (rc != FZ_OK) return rc;
    }
    return FZ_OK;
  };
#define FZ_ARC(call)                \
  do {                              \
    const int rc__ = (call);        \
    if (rc__ != FZ_OK) {            \
      unbind();                     \
      return rc__;                  \
    }                               \
  } while (0)
  auto save = [&](const State& st) -> cudaError_t {
    cudaError_t e = cudaSuccess;
    for (int f = 0; f < 4 && e == cudaSuccess; f++)
      e = cudaMemcpyAsync(st.f[f], h->U[h->i0][f], fb, cudaMemcpyDeviceToDevice, s);
    for (int a = 0; a < 3 && e == cudaSuccess; a++)
      if (ade_b[a]) e = cudaMemcpyAsync(st.ade[a], h->d_ade[h->ph_old][a], ade_b[a], cudaMemcpyDeviceToDevice, s);
    for (int a = 0; a < 3 && e == cudaSuccess; a++)
      if (psi_b[a]) e = cudaMemcpyAsync(st.psi[a], h->d_psi[a], psi_b[a], cudaMemcpyDeviceToDevice, s);
    return e;
  };
  auto restore = [&](const State& st, int64_t step) -> cudaError_t {
    cudaError_t e = cudaSuccess;
    for (int f = 0; f < 4 && e == cudaSuccess; f++)
      e = cudaMemcpyAsync(h->U[h->i0][f], st.f[f], fb, cudaMemcpyDeviceToDevice, s);
    for (int a = 0; a < 3 && e == cudaSuccess; a++)
      if (ade_b[a]) e = cudaMemcpyAsync(h->d_ade[h->ph_old][a], st.ade[a], ade_b[a], cudaMemcpyDeviceToDevice, s);
    for (int a = 0; a < 3 && e == cudaSuccess; a++)
      if (psi_b[a]) e = cudaMemcpyAsync(h->d_psi[a], st.psi[a], psi_b[a], cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->d_step, &step, sizeof(step), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the step value lives on this stack frame
    return e;
  };

  // cells no kernel writes stay constant through a run: make them zero in every field set, so
  // that a checkpoint of U0 alone reproduces the whole state
  for (int q = 0; q < 3; q++)
    for (int f = 0; f < 4; f++)
      FZ_ACUDA(h, fz::launch_clear_inactive<R>((R*)h->U[q][f], h->d_cls, N, s), "clear inactive");

  cudaEvent_t ev[4];
  for (auto& e : ev) FZ_ACUDA(h, cudaEventCreate(&e), "event");
  struct EvGuard {
    cudaEvent_t* e;
    ~EvGuard() {
      for (int i = 0; i < 4; i++) cudaEventDestroy(e[i]);
    }
  } evg{ev};

  // ---- forward with checkpoints
  nvtxRangePushA("adjoint: forward with checkpoints");
  FZ_ACUDA(h, cudaEventRecord(ev[0], s), "event record");
  for (int64_t q = 0; q < nseg; q++) {
    FZ_ACUDA(h, save(ck[(size_t)q]), "checkpoint");
    const int rc = fz_run(h, std::min<int64_t>(seg, nsteps - q * seg));
    if (rc != FZ_OK) return rc;
  }
  FZ_ACUDA(h, save(ck[(size_t)nseg]), "checkpoint");
  FZ_ACUDA(h, cudaEventRecord(ev[1], s), "event record");
  nvtxRangePop();
  int rc = fz_sync(h, 0);
  if (rc != FZ_OK) return rc;

  // ---- misfit
  std::vector<double> ir((size_t)h->nrec * h->rec_cap);
  FZ_ACUDA(h, cudaMemcpy(ir.data(), h->d_ir, ir.size() * 8, cudaMemcpyDeviceToHost), "IR D2H");
  double Jv = 0.0;
  for (int r = 0; r < h->nrec; r++)
    for (int64_t n = 0; n < nsteps; n++) {
      const double x = ir[(size_t)r * h->rec_cap + n], t = target[(size_t)r * tsteps + n];
      Jv += o.cotangent ? t * x : (x - t) * (x - t);
    }
  if (J) *J = Jv;
  FZ_ACUDA(h, cudaMemcpy(d_target, target, (size_t)h->nrec * tsteps * 8, cudaMemcpyHostToDevice), "target H2D");

  // ---- backward
  for (int f = 0; f < 4; f++) FZ_ACUDA(h, cudaMemsetAsync(lam[0][f], 0, fb, s), "memset");
  for (int a = 0; a < 3; a++)
    if (ade_b[a]) FZ_ACUDA(h, cudaMemsetAsync(lade[0][a], 0, ade_b[a], s), "memset");
  for (int q = 0; q < 2; q++)
    for (int a = 0; a < 3; a++)
      if (psi_b[a]) FZ_ACUDA(h, cudaMemsetAsync(lpsi[q][a], 0, psi_b[a], s), "memset");
  if (nB > 0) FZ_ACUDA(h, cudaMemsetAsync(d_gcell, 0, (size_t)Pn * nB * 8, s), "memset");
  FZ_ACUDA(h, cudaMemsetAsync(d_gsval, 0, (size_t)std::max(1, nsrc) * 8, s), "memset");
  FZ_ACUDA(h, cudaMemsetAsync(d_gwave, 0, (size_t)std::max(1, nsrc) * std::max<int64_t>(1, n_us) * 8, s), "memset");
  FZ_ACUDA(h, cudaMemsetAsync(d_gpml, 0, (size_t)3 * 6 * d * 8, s), "memset");
  if (nsrc > 0)
    FZ_ACUDA(h, cudaMemcpy(d_sval, h->src_val.data(), (size_t)nsrc * 8, cudaMemcpyHostToDevice), "sval H2D");
  // source injection per unit strength (the stage kernels' src_coef / sval)
  const double src_unit = h->prm.dt * h->prm.c * h->prm.c * h->prm.rho * (6.0 * h->prm.h * h->prm.h) /
                          (h->prm.h * h->prm.h * h->prm.h);

  const fz_params& p = h->prm;
  fz::AdjStageArgs<R> sa;
  std::memset(&sa, 0, sizeof(sa));
  sa.cls = h->d_cls;
  sa.Nx = h->Nx; sa.Ny = h->Ny; sa.Nz = h->Nz;
  sa.Sx = h->Sx; sa.plane = h->plane;
  sa.inv_h = (R)(1.0 / p.h);
  sa.fc = (R)(0.5 * p.c);
  sa.frc2 = (R)(0.5 * p.rho * p.c * p.c);
  sa.firho = (R)(0.5 / p.rho);
  sa.pml_on = h->pml_on ? 1 : 0;
  sa.pml_d2 = (int)d2;
  sa.err = h->d_err;
  sa.nfield = N;
  for (int a = 0; a < 3; a++) sa.npsi[a] = (int64_t)(psi_b[a] / sizeof(P));
  sa.pcx = (const fz::PmlCoef<R>*)h->d_pml_coef[0];
  sa.pcy = (const fz::PmlCoef<R>*)h->d_pml_coef[1];
  sa.pcz = (const fz::PmlCoef<R>*)h->d_pml_coef[2];
  // launch geometry of the fused stage adjoint: z chunks that fill whole waves, each chunk paying
  // four extra centre planes
  const int ntx = (h->Nx - 2 * GHOST + fz::ATX - 1) / fz::ATX, nty = (h->Ny - 2 * GHOST + fz::ATY - 1) / fz::ATY;
  const int nzi = h->Nz - 2 * GHOST;
  const size_t smem_max = fz::adj_stage_smem<R>(nzi);
  FZ_ACUDA(h, fz::adj_stage_setup<R>(smem_max), "adjoint setup");
  int occ = 1;
  FZ_ACUDA(h, fz::adj_stage_occupancy<R>(&occ, smem_max), "adjoint occupancy");
  occ = std::max(1, occ);
  const int64_t slots = (int64_t)h->nsm * occ;
  int best = 1;
  double best_eff = -1.0;
  for (int nk = 1; nk <= std::max(1, nzi / 8); nk++) {
    const int chunk = (nzi + nk - 1) / nk;
    const int64_t items = (int64_t)ntx * nty * ((nzi + chunk - 1) / chunk);
    const int64_t waves = (items + slots - 1) / slots;
    const double eff = ((double)items / (double)(waves * slots)) * ((double)chunk / (chunk + 4.0));
    if (eff > best_eff + 1e-9) {
      best_eff = eff;
      best = nk;
    }
  }
  sa.kz_chunk = (nzi + best - 1) / best;
  const dim3 agrid((unsigned)ntx, (unsigned)nty, (unsigned)((nzi + sa.kz_chunk - 1) / sa.kz_chunk));
  int ps = 0;  // lpsi[ps]: adjoint of psi^{n+1}; lpsi[1 - ps]: of psi^n

  fz::AdjBandArgs<R> ba;
  std::memset(&ba, 0, sizeof(ba));
  ba.nB = nB;
  ba.rec = h->d_brec;
  ba.geo = (const R*)h->d_bgeo;
  ba.nrm = (const R*)h->d_bnrm;
  ba.Sx = h->Sx; ba.plane = h->plane;
  ba.Z0 = p.rho * p.c;
  ba.dt = p.dt;
  ba.K = K; ba.L = L; ba.nMat = nMat;
  {
    const double* m = h->d_mat;
    ba.Rinf = m; m += nMat;
    ba.A = m; m += (size_t)nMat * K;
    ba.zeta = m; m += (size_t)nMat * K;
    ba.B = m; m += (size_t)nMat * L;
    ba.C = m; m += (size_t)nMat * L;
    ba.alpha = m; m += (size_t)nMat * L;
    ba.beta = m;
  }
  ba.gcell = d_gcell;
  ba.err = h->d_err;
  ba.nfield = N;
  ba.probe = d_probe;

  // buffer roles: A = adjoint of the step's output, B/D = of the stage-2/stage-1 inputs, C = of U0
  int iA = 0, iB = 1, iC = 2, iD = 3;
  int jN = 0, jO = 1, j1 = 2, j2 = 3;  // ADE adjoint sets: next, old, after stage 0, after stage 1
  auto set_in = [&](auto& x, const void* const* f) {
    x.pi = (const R*)f[0]; x.ui = (const R*)f[1]; x.vi = (const R*)f[2]; x.wi = (const R*)f[3];
  };

  FZ_ACUDA(h, cudaEventRecord(ev[2], s), "event record");
  // cells no kernel writes read zero in every stored stage input, as in the handle's own sets
  for (int q = 0; q < 3; q++)
    for (void* p : S[q]) FZ_ACUDA(h, cudaMemsetAsync(p, 0, fb, s), "memset");
  for (int64_t q = nseg - 1; q >= 0; q--) {
    const int len = (int)std::min<int64_t>(seg, nsteps - q * seg);
    FZ_ACUDA(h, restore(ck[(size_t)q], q * seg), "restore");
    // recompute the segment with the stage kernels writing straight into the segment storage
    // (field sets bound to the stored arrays): the step input is S[0][t], stage 0 writes S[1][t],
    // stage 1 S[2][t], stage 2 the next step's S[0][t+1]. Likewise the band kernels' ADE outputs:
    // the role slots the band arguments name point at Ad[1][t] (stage 0), Ad[2][t] (stage 1) and
    // Ad[3][t] (stage 2), which the step's role swap makes the next step's input Ad[0][t+1]; only
    // the segment's first input set (the restored checkpoint) is copied
    {
      cudaError_t e = cudaSuccess;
      for (int f = 0; f < 4 && e == cudaSuccess; f++)
        e = cudaMemcpyAsync(S[0][f], h->U[h->i0][f], fb, cudaMemcpyDeviceToDevice, s);
      for (int a = 0; a < 3 && e == cudaSuccess; a++)
        if (ade_b[a]) e = cudaMemcpyAsync(Ad[0][a][0], h->d_ade[h->ph_old][a], ade_b[a], cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) return fzi::cuda_fail(h, e, "adjoint recompute");
    }
    FZ_ARC(fzi::bind_field_set(h, h->i0, &S[0][0]));
    auto point_ade = [&](int role, int q, int t) {
      for (int a = 0; a < 3; a++) h->d_ade[role][a] = Ad[q][a][(size_t)t];
    };
    point_ade(h->ph_old, 0, 0);
    for (int t = 0; t < len; t++) {
      cudaError_t e = cudaSuccess;
      for (int a = 0; a < 3 && e == cudaSuccess && want_pml; a++)
        if (psi_b[a]) e = cudaMemcpyAsync(Ps[a][(size_t)t], h->d_psi[a], psi_b[a], cudaMemcpyDeviceToDevice, s);
      FZ_ARC(fzi::bind_field_set(h, h->i1, &S[1][(size_t)t * 4]));
      point_ade(h->ph_cur, 1, t);
      if (e == cudaSuccess) e = fzi::enqueue_stage(h, 0);
      FZ_ARC(fzi::bind_field_set(h, h->i2, &S[2][(size_t)t * 4]));
      point_ade(h->ph_nu, 2, t);
      if (e == cudaSuccess) e = fzi::enqueue_stage(h, 1);
      // the last step's output is the next segment's checkpoint, not stored: a free own set takes it
      FZ_ARC(fzi::bind_field_set(h, h->i1, (t + 1 < len) ? &S[0][(size_t)(t + 1) * 4] : own[0]));
      point_ade(h->ph_cur, 3, t);
      if (e == cudaSuccess) e = fzi::enqueue_stage(h, 2);
      if (e == cudaSuccess) e = fzi::enqueue_finish(h);
      if (e != cudaSuccess) {
        unbind();
        return fzi::cuda_fail(h, e, "adjoint recompute");
      }
    }
    FZ_ARC(unbind());
    // reverse sweep
    fz_range sweep_range("adjoint: reverse sweep of a segment");
    for (int t = len - 1; t >= 0; t--) {
      const int64_t n = q * seg + t;
      // the ADE adjoint sets jO, j1, j2 need no zeroing: the band adjoint's first write to each in a
      // step assigns (k_adj_band)
      FZ_ACUDA(h, fz::launch_adj_receivers<R>(lam[iA][0], h->d_rec_cell, h->nrec, h->d_ir, h->rec_cap, d_target,
                                               tsteps, n, o.cotangent ? 1 : 0, s), "adjoint receivers");
      const void* const* in_st[3] = {&S[0][(size_t)t * 4], &S[1][(size_t)t * 4], &S[2][(size_t)t * 4]};
      for (int st = 2; st >= 0; st--) {
        // adjoint of the stage output (out), of its input (inb) and of U0 (base)
        const int out = (st == 2) ? iA : (st == 1) ? iB : iD;
        const int inb = (st == 2) ? iB : (st == 1) ? iD : iC;
        // ADE value sets (left, middle, right) and their adjoints, as band_args assigns them
        const int vL = (st == 0) ? 1 : (st == 1) ? 2 : 3, vM = 0, vR = (st == 0) ? 0 : (st == 1) ? 1 : 2;
        const int gL = (st == 0) ? j1 : (st == 1) ? j2 : jN;
        const int gR = (st == 0) ? jO : (st == 1) ? j1 : j2;
        if (nB > 0) {
          set_in(ba, in_st[st]);
          ba.lp = lam[out][0]; ba.lu = lam[out][1]; ba.lv = lam[out][2]; ba.lw = lam[out][3];
          ba.ip = lam[inb][0]; ba.iu = lam[inb][1]; ba.iv = lam[inb][2]; ba.iw = lam[inb][3];
          ba.phL = Ad[vL][0][(size_t)t]; ba.phM = Ad[vM][0][(size_t)t]; ba.phR = Ad[vR][0][(size_t)t];
          ba.s1L = Ad[vL][1][(size_t)t]; ba.s1M = Ad[vM][1][(size_t)t]; ba.s1R = Ad[vR][1][(size_t)t];
          ba.s2L = Ad[vL][2][(size_t)t]; ba.s2M = Ad[vM][2][(size_t)t]; ba.s2R = Ad[vR][2][(size_t)t];
          ba.gphL = lade[gL][0]; ba.gphM = lade[jO][0]; ba.gphR = lade[gR][0];
          ba.gs1L = lade[gL][1]; ba.gs1M = lade[jO][1]; ba.gs1R = lade[gR][1];
          ba.gs2L = lade[gL][2]; ba.gs2M = lade[jO][2]; ba.gs2R = lade[gR][2];
          FZ_ACUDA(h, fz::launch_adj_band<R>(st, ba, s), "adjoint band");
        }
        const double w = (st == 0) ? 1.0 : (st == 1) ? 0.25 : 2.0 / 3.0;
        // parameter gradients of this stage, from the adjoint of its output (band cells scaled)
        if (want_src)
          FZ_ACUDA(h, fz::launch_adj_source<R>(lam[out][0], h->d_src_cell, nsrc, d_sval, src_unit, (const R*)h->d_us,
                                               n_us, h->src_opt, (const R*)h->d_src_freq, (R)(0.5 * p.dt), w,
                                               2 * n + ((st == 0) ? 0 : (st == 1) ? 2 : 1), o.source_sval ? d_gsval : nullptr,
                                               o.source_wave ? d_gwave : nullptr, s),
                   "adjoint sources");
        if (want_pml)
          for (int a = 0; a < 3; a++) {
            if (!psi_b[a]) continue;
            fz::AdjPmlArgs<R> pa;
            std::memset(&pa, 0, sizeof(pa));
            pa.pi = (const R*)in_st[st][0];
            pa.vi = (const R*)in_st[st][1 + a];
            pa.lp = lam[out][0];
            pa.lv = lam[out][1 + a];
            pa.lpsi = lpsi[ps][a];
            pa.psin = (const P*)Ps[a][(size_t)t];
            pa.pc = (const fz::PmlCoef<R>*)h->d_pml_coef[a];
            pa.cls = h->d_cls;
            pa.axis = a;
            pa.Nx = h->Nx; pa.Ny = h->Ny; pa.Nz = h->Nz;
            pa.d = d;
            pa.stage = st;
            pa.Sx = h->Sx; pa.plane = h->plane;
            pa.inv_h = sa.inv_h; pa.frc2 = sa.frc2; pa.firho = sa.firho; pa.fc = sa.fc;
            pa.wdt = w * p.dt;
            pa.g = d_gpml + (size_t)a * 6 * d;
            pa.err = h->d_err;
            pa.nfield = N;
            pa.npsi = (int64_t)(psi_b[a] / sizeof(P));
            FZ_ACUDA(h, fz::launch_adj_pml_grad<R>(pa, h->nsm, s), "adjoint cPML gradient");
          }
        set_in(sa, in_st[st]);
        sa.lp = lam[out][0]; sa.lu = lam[out][1]; sa.lv = lam[out][2]; sa.lw = lam[out][3];
        sa.ip = lam[inb][0]; sa.iu = lam[inb][1]; sa.iv = lam[inb][2]; sa.iw = lam[inb][3];
        sa.bp = lam[iC][0]; sa.bu = lam[iC][1]; sa.bv = lam[iC][2]; sa.bw = lam[iC][3];
        sa.stage = st;
        sa.b_in = (R)w;
        sa.a_base = (R)((st == 0) ? 0.0 : (st == 1) ? 0.75 : 1.0 / 3.0);
        sa.cb = (R)(w * p.dt / p.h);
        sa.wdt = (R)(w * p.dt);
        sa.lpsix = lpsi[ps][0]; sa.lpsiy = lpsi[ps][1]; sa.lpsiz = lpsi[ps][2];
        sa.opsix = lpsi[1 - ps][0]; sa.opsiy = lpsi[1 - ps][1]; sa.opsiz = lpsi[1 - ps][2];
        // stage 2 stores both adjoints fresh; stage 1 stores the input's and adds to U0's; stage 0's
        // input is U0, whose adjoint the later stages have started
        sa.acc_in = (st == 0) ? 1 : 0;
        sa.acc_base = (st == 1) ? 1 : 0;
        FZ_ACUDA(h, fz::launch_adj_stage<R>(sa, agrid, s), "adjoint stage");
        if (nB > 0) FZ_ACUDA(h, fz::launch_adj_probe_scatter<R>(ba, s), "adjoint probe scatter");
      }
      std::swap(iA, iC);  // the adjoint of U0^n is the next (earlier) step's output adjoint
      std::swap(jN, jO);
      ps = 1 - ps;
    }
  }
#undef FZ_ARC
  FZ_ACUDA(h, fz::launch_adj_grad_reduce(h->d_brec, d_gcell, nB, Pn, nMat, d_grad, s), "gradient reduce");
  FZ_ACUDA(h, cudaEventRecord(ev[3], s), "event record");
  FZ_ACUDA(h, cudaStreamSynchronize(s), "adjoint sync");
  if (o.materials)
    FZ_ACUDA(h, cudaMemcpy(o.materials, d_grad, (size_t)nMat * Pn * 8, cudaMemcpyDeviceToHost), "grad D2H");
  if (o.source_sval) {
    std::fill(o.source_sval, o.source_sval + h->nsrc, 0.0);
    if (want_src) FZ_ACUDA(h, cudaMemcpy(o.source_sval, d_gsval, (size_t)nsrc * 8, cudaMemcpyDeviceToHost), "grad D2H");
  }
  if (o.source_wave && h->nsrc > 0 && n_us > 0) {
    std::fill(o.source_wave, o.source_wave + (size_t)h->nsrc * n_us, 0.0);
    if (want_src)
      FZ_ACUDA(h, cudaMemcpy(o.source_wave, d_gwave, (size_t)nsrc * n_us * 8, cudaMemcpyDeviceToHost), "grad D2H");
  }
  if (o.pml) {
    // chain rule from the table entries to (R0, kappa_max, alpha_max) through the host's table
    std::fill(o.pml, o.pml + 4, 0.0);
    if (want_pml) {
      std::vector<double> g((size_t)3 * 6 * d);
      FZ_ACUDA(h, cudaMemcpy(g.data(), d_gpml, g.size() * 8, cudaMemcpyDeviceToHost), "grad D2H");
      const int lo[3] = {p.pml[3] != 0, p.pml[5] != 0, p.pml[1] != 0};
      const int hi[3] = {p.pml[2] != 0, p.pml[4] != 0, p.pml[0] != 0};
      const int Na[3] = {h->Nx, h->Ny, h->Nz};
      for (int a = 0; a < 3; a++) {
        if (!psi_b[a]) continue;
        for (int tl = 0; tl < 2 * d; tl++) {
          const int ca = (tl < d) ? GHOST + tl : Na[a] - GHOST - 2 * d + tl;
          fzi::PmlEntry e;
          fzi::pml_entry(p, Na[a], lo[a], hi[a], ca, &e);
          if (e.tile != tl) continue;
          for (int v = 0; v < 3; v++)
            for (int r = 0; r < 3; r++) o.pml[r] += g[(size_t)a * 6 * d + 3 * tl + v] * e.d[v][r];
        }
      }
    }
  }
  if (o.initial) {
    // after the sweep the carried adjoint is that of the step-0 state; cells no kernel writes were
    // set to zero before the forward pass, so J does not depend on their initial values
    const size_t rowb = (size_t)h->Nx * sizeof(R);
    std::vector<R> tmp((size_t)nref);
    for (int f = 0; f < 4; f++) {
      FZ_ACUDA(h, cudaMemcpy2D(tmp.data(), rowb, lam[iA][f] + XOFF, (size_t)h->Sx * sizeof(R), rowb,
                               (size_t)h->Ny * h->Nz, cudaMemcpyDeviceToHost), "grad D2H");
      double* out = o.initial + (size_t)f * nref;
      for (int k = 0; k < h->Nz; k++)
        for (int j = 0; j < h->Ny; j++)
          for (int i = 0; i < h->Nx; i++) {
            const size_t c = (size_t)i + (size_t)h->Nx * ((size_t)j + (size_t)h->Ny * k);
            const int64_t g = XOFF + i + h->Sx * ((int64_t)j + (int64_t)h->Ny * k);
            out[c] = (h->cls_host[(size_t)g] & (fz::CLS_UPDATE | fz::CLS_BAND)) ? (double)tmp[c] : 0.0;
          }
    }
  }
  if (ms) {
    float a = 0.f, b = 0.f;
    FZ_ACUDA(h, cudaEventElapsedTime(&a, ev[0], ev[1]), "event elapsed");
    FZ_ACUDA(h, cudaEventElapsedTime(&b, ev[2], ev[3]), "event elapsed");
    ms[0] = a;
    ms[1] = b;
  }
  // leave the handle at the end of the forward run
  FZ_ACUDA(h, restore(ck[(size_t)nseg], nsteps), "restore final state");
  return fz_sync(h, 0);
}

}  // namespace

extern "C" {

int fz_material_layout(fz_handle* h, int32_t* nMat, int32_t* K, int32_t* L) {
  if (!h) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  const int rc = fzi::prepare(h);
  if (rc != FZ_OK) return rc;
  if (nMat) *nMat = std::max(1, h->nMat);
  if (K) *K = h->K;
  if (L) *L = h->L;
  return FZ_OK;
}

int fz_misfit_gradient(fz_handle* h, int64_t nsteps, int32_t segment_steps, const double* target,
                       int64_t target_steps, double* J, double* grad, int64_t grad_cap, double* ms) {
  if (!h) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  if (!grad) return fzi::set_error(h, FZ_EINVAL, "fz_misfit_gradient: grad required");
  fz_gradients o;
  std::memset(&o, 0, sizeof(o));
  o.materials = grad;
  o.materials_cap = grad_cap;
  return fz_misfit_gradient_ex(h, nsteps, segment_steps, target, target_steps, J, &o, ms);
}

int fz_misfit_gradient_ex(fz_handle* h, int64_t nsteps, int32_t segment_steps, const double* target,
                          int64_t target_steps, double* J, fz_gradients* out, double* ms) {
  fz_range nvtx_range("fz_misfit_gradient");
  if (!h) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  if (nsteps < 1 || segment_steps < 1 || !target || !out || target_steps < nsteps)
    return fzi::set_error(h, FZ_EINVAL, "fz_misfit_gradient: nsteps >= 1, segment_steps >= 1, target of "
                                        "[n_rec][target_steps >= nsteps] and outputs required");
  if (h->prm.two_d || h->nb != 1)
    return fzi::set_error(h, FZ_EINVAL, "fz_misfit_gradient: 3D single-member solves only");
  int rc = fzi::prepare(h);
  if (rc != FZ_OK) return rc;
  if (h->nrec < 1 || h->rec_cap < nsteps)
    return fzi::set_error(h, FZ_EINVAL, "fz_misfit_gradient: receivers with capacity >= nsteps required");
  if (h->steps_enqueued != 0)
    return fzi::set_error(h, FZ_ESTATE, "fz_misfit_gradient: the handle must be at step 0 (set fields, then call)");
  for (int q = 0; q < h->nsrc; q++) {
    const int64_t c = (int64_t)XOFF + h->src_ijk[3 * q] +
                      h->Sx * ((int64_t)h->src_ijk[3 * q + 1] + (int64_t)h->Ny * h->src_ijk[3 * q + 2]);
    if (!(h->cls_host[(size_t)c] & fz::CLS_UPDATE))
      return fzi::set_error(h, FZ_EINVAL, "fz_misfit_gradient: a source sits in a cell the stage kernels skip");
  }
  cudaSetDevice(h->device);
  segment_steps = (int32_t)std::min<int64_t>(segment_steps, nsteps);  // no storage for steps never run
  return h->fp64 ? misfit_gradient<double>(h, nsteps, segment_steps, target, target_steps, J, *out, ms)
                 : misfit_gradient<float>(h, nsteps, segment_steps, target, target_steps, J, *out, ms);
}

}  // extern "C"
