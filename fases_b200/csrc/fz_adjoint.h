// fz_adjoint.h -- kernels of the discrete adjoint of one SSP-RK3 step (fz_adjoint.cu) and the
// arguments they take. The adjoint is of the scheme the stepping kernels compute
// (3D-solver/core/functions3D.cuh:56-78, 426-565, 661-1001, 1086-1327); the reference has no
// adjoint or gradient of any kind.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fz_device.cuh"

namespace fz {

// Adjoint of the stage kernel of one stage: the stage output is
//   out = a U0 + b (in + dt/h sum_d dF_d(in)) + w dt sum_d [pml_d] ((1/kappa_d - 1) dF_d/h + psi_d)
// on update cells (dF_d = flux difference along axis d), and psi^{n+1} = b_d psi^n + ca_d dF_d/h
// in stage 2.
template <class R>
struct AdjStageArgs {
  typedef typename Pair<R>::T P;
  const R* pi;  // stage input (stored forward state)
  const R* ui;
  const R* vi;
  const R* wi;
  const R* lp;  // adjoint of the stage output (after the band adjoint scaled band cells)
  const R* lu;
  const R* lv;
  const R* lw;
  R* ip;  // adjoint of the stage input (accumulated)
  R* iu;
  R* iv;
  R* iw;
  R* bp;  // adjoint of U0 (accumulated; stages 1 and 2)
  R* bu;
  R* bv;
  R* bw;
  const uint8_t* cls;
  int32_t Nx, Ny, Nz;
  int64_t Sx, plane;
  R cb;      // b dt / h
  R a_base;  // a
  R b_in;    // b
  R wdt;     // w dt
  R inv_h;
  R fc, frc2, firho;  // Godunov: c/2, rho c^2 / 2, 1 / (2 rho)
  int32_t stage;
  int32_t pml_on, pml_d2;
  const PmlCoef<R>* pcx;
  const PmlCoef<R>* pcy;
  const PmlCoef<R>* pcz;
  const P* lpsix;  // adjoint of psi^{n+1} (read by stage 2's flux weights)
  const P* lpsiy;
  const P* lpsiz;
  P* opsix;  // adjoint of psi^n: stage 2 writes b lpsi + w dt out, stages 1 and 0 add w dt out
  P* opsiy;
  P* opsiz;
  int32_t kz_chunk;  // z planes per CTA of the fused stage adjoint
  int32_t acc_in;    // 1: add to the input adjoint (it holds U0's adjoint already), 0: store it
  int32_t acc_base;  // 1: add to U0's adjoint, 0: store it (stages 1 and 2)
  // bounds-checked build: device error word, elements of one field array and of the psi tiles
  int32_t* err;
  int64_t nfield;
  int64_t npsi[3];
};

// Adjoint of the immersed band of one stage (functions3D.cuh:426-565), with the gradient of the
// misfit with respect to the ADE coefficients accumulated per material.
template <class R>
struct AdjBandArgs {
  int64_t nB;
  const int4* rec;
  const R* geo;
  const R* nrm;
  const R* pi;  // stage input (probe source)
  const R* ui;
  const R* vi;
  const R* wi;
  R* lp;  // adjoint of the stage output: read, then scaled by (1 - chi) at band cells
  R* lu;
  R* lv;
  R* lw;
  R* ip;  // adjoint of the stage input: probe contributions scattered with atomics
  R* iu;
  R* iv;
  R* iw;
  R* probe;  // [4][nB]: adjoint of the probed p, u, v, w of every band cell
  int64_t Sx, plane;
  double Z0, dt;
  int32_t K, L, nMat;
  const double* Rinf;
  const double* A;
  const double* zeta;
  const double* B;
  const double* C;
  const double* alpha;
  const double* beta;
  // ADE state values of the stage (left = written, middle, right), [q*nB + b]
  const double* phL;
  const double* phM;
  const double* phR;
  const double* s1L;
  const double* s1M;
  const double* s1R;
  const double* s2L;
  const double* s2M;
  const double* s2R;
  // their adjoints: left read, middle and right accumulated
  const double* gphL;
  double* gphM;
  double* gphR;
  const double* gs1L;
  double* gs1M;
  double* gs1R;
  const double* gs2L;
  double* gs2M;
  double* gs2R;
  double* gcell;  // [1 + 2K + 4L][nB]: per band cell, d J / d (Rinf, A[K], zeta[K], B[L], C[L],
                  // alpha[L], beta[L]) of its material, accumulated over stages and steps
  int32_t* err;     // bounds-checked build: device error word, elements of one field array
  int64_t nfield;
};

// Gradient with respect to the cPML table entries (1/kappa - 1, b, ca) of one axis from one stage.
// The forward correction (stage kernel) is  out += w dt ((1/kappa - 1) D + psi^n)  for the pressure
// and the velocity along the axis, and in stage 2  psi^{n+1} = b psi^n + ca D,  with D the flux
// difference along the axis over h. Per cPML cell of the axis this recomputes D from the stage
// input exactly as the stage kernel does and adds
//   g_kinv1 += w dt (lp Dp + lv Dv);   stage 2: g_b += lpsi . psi^n,   g_ca += lpsi . D
// into g[tile][3] (tile = index in the psi tile's 2d layers).
template <class R>
struct AdjPmlArgs {
  typedef typename Pair<R>::T P;
  const R* pi;  // stage input: pressure and the velocity along the axis
  const R* vi;
  const R* lp;  // adjoint of the stage output (after the band adjoint)
  const R* lv;
  const P* lpsi;  // adjoint of psi^{n+1} (stage 2)
  const P* psin;  // psi^n (stage 2)
  const PmlCoef<R>* pc;
  const uint8_t* cls;
  int32_t axis, Nx, Ny, Nz, d, stage;
  int64_t Sx, plane;
  R inv_h, frc2, firho, fc;
  double wdt;
  double* g;
  int32_t* err;  // bounds-checked build: device error word, elements of a field array and psi tile
  int64_t nfield, npsi;
};
template <class R>
cudaError_t launch_adj_pml_grad(const AdjPmlArgs<R>& a, int nsm, cudaStream_t s);

// Gradient with respect to the source strengths sval[q] and the waveform samples u_s[nn] from one
// stage (the stage kernel adds w * unit * sval[q] * u_s[nn] to p at the source cell, unit =
// dt c^2 rho A_s / h^3): gsval[q] += lp w unit amp(nn), gwave[q][nn] += lp w unit sval[q].
template <class R>
cudaError_t launch_adj_source(const R* lp, const int64_t* cell, int nsrc, const double* sval, double unit,
                              const R* u_s, int64_t n_us, int src_opt, const R* freq, R half_dt, double w, int64_t nn,
                              double* gsval, double* gwave, cudaStream_t s);

// fused adjoint of one stage kernel launch over the interior cells, grid (x tiles, y tiles, z chunks)
template <class R>
cudaError_t launch_adj_stage(const AdjStageArgs<R>& a, dim3 grid, cudaStream_t s);
template <class R>
size_t adj_stage_smem(int kz_chunk);
template <class R>
cudaError_t adj_stage_setup(size_t smem_bytes);
template <class R>
cudaError_t adj_stage_occupancy(int* blocks_per_sm, size_t smem_bytes);
// the band cells' probe adjoints (k_adj_band's output) into the stage input's adjoint
template <class R>
cudaError_t launch_adj_probe_scatter(const AdjBandArgs<R>& a, cudaStream_t s);
template <class R>
cudaError_t launch_adj_band(int stage, const AdjBandArgs<R>& a, cudaStream_t s);
// grad[m][e] = sum over the band cells of material m of gcell[e][b]
cudaError_t launch_adj_grad_reduce(const int4* rec, const double* gcell, int64_t nB, int P, int nMat, double* grad,
                                   cudaStream_t s);
// adjoint of the receiver gather: lp[cell_r] += 2 (ir[r][n] - target[r][n]), or += target[r][n]
// when target holds a cotangent of the traces
template <class R>
cudaError_t launch_adj_receivers(R* lp, const int64_t* rcell, int nrec, const double* ir, int64_t cap,
                                 const double* target, int64_t tlen, int64_t n, int cotangent, cudaStream_t s);
// zero every field value of cells no kernel writes (class bytes without UPDATE or BAND)
template <class R>
cudaError_t launch_clear_inactive(R* f, const uint8_t* cls, int64_t n, cudaStream_t s);

}  // namespace fz
