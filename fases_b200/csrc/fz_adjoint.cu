// fz_adjoint.cu -- discrete adjoint of one SSP-RK3 step of the stepping kernels: the transposed
// linearisation of WENO-Z (weights included; |beta0 - beta2| takes the subgradient sign(0) = 0),
// the Godunov flux, the RK combination, the cPML correction and psi recursion, the immersed band
// (trilinear probe, characteristic split, chi blend) and the ADE pole recursion, with the
// gradient with respect to the ADE coefficients. The forward scheme is the reference's
// (3D-solver/core/functions3D.cuh:56-78, 411-565, 661-1001, 1086-1327); the reference has no
// adjoint. Arithmetic follows the restated formulas (as the CPU oracle writes them), not the
// forward kernels' rearranged forms: both are the same function.
#include "fz_adjoint.h"

namespace fz {

namespace {

template <class R>
struct WenoTables {
  // candidate rows (main3D.cu:834-837), beta second-term rows (839-841), linear weights (843)
  static __device__ __forceinline__ R crl(int row, int l) {
    const R t[4][3] = {{R(11.0 / 6.0), R(-7.0 / 6.0), R(1.0 / 3.0)},
                       {R(1.0 / 3.0), R(5.0 / 6.0), R(-1.0 / 6.0)},
                       {R(-1.0 / 6.0), R(5.0 / 6.0), R(1.0 / 3.0)},
                       {R(1.0 / 3.0), R(-7.0 / 6.0), R(11.0 / 6.0)}};
    return t[row][l];
  }
  static __device__ __forceinline__ R brl(int r, int l) {
    const R t[3][3] = {{R(3), R(-4), R(1)}, {R(1), R(0), R(-1)}, {R(1), R(-4), R(3)}};
    return t[r][l];
  }
  static __device__ __forceinline__ R dd(int i) {
    const R t[3] = {R(0.3), R(0.6), R(0.1)};
    return t[i];
  }
};

// Reverse mode of one WENO-Z cell centre: u[0..4] are the values at c-2 .. c+2; the centre gives
// V-(c+1/2) (side 1) and V+(c-1/2) (side 0) from one set of smoothness indicators. g[0..4] +=
// lam_m dV-/du + lam_p dV+/du.
template <class R>
__device__ __forceinline__ void weno_centre_rev(const R u[5], R lam_m, R lam_p, R g[5]) {
  typedef WenoTables<R> T;
  const R eps = R(1e-10);
  R b1[3], b2[3], beta[3];
#pragma unroll
  for (int r = 0; r < 3; r++) {
    b1[r] = u[2 - r] - R(2) * u[3 - r] + u[4 - r];
    b2[r] = T::brl(r, 0) * u[2 - r] + T::brl(r, 1) * u[3 - r] + T::brl(r, 2) * u[4 - r];
    beta[r] = R(13.0 / 12.0) * b1[r] * b1[r] + R(0.25) * b2[r] * b2[r];
  }
  const R diff = beta[0] - beta[2];
  const R tau = diff >= R(0) ? diff : -diff;
  const R sg = (diff > R(0)) ? R(1) : ((diff < R(0)) ? R(-1) : R(0));
  R ib[3];
#pragma unroll
  for (int r = 0; r < 3; r++) ib[r] = R(1) / (beta[r] + eps);
  R lbeta[3] = {R(0), R(0), R(0)};
  R ltau = R(0);
#pragma unroll
  for (int side = 0; side < 2; side++) {
    const R lam = side ? lam_m : lam_p;
    R cand[3], alpha[3], S = R(0), num = R(0);
#pragma unroll
    for (int r = 0; r < 3; r++) {
      cand[r] = T::crl(r + side, 0) * u[2 - r] + T::crl(r + side, 1) * u[3 - r] + T::crl(r + side, 2) * u[4 - r];
      alpha[r] = T::dd(side ? r : 2 - r) * (R(1) + tau * ib[r]);
      S += alpha[r];
      num += alpha[r] * cand[r];
    }
    const R iS = R(1) / S;
    const R V = num * iS;
#pragma unroll
    for (int r = 0; r < 3; r++) {
      const R lc = alpha[r] * iS * lam;
      g[2 - r] += T::crl(r + side, 0) * lc;
      g[3 - r] += T::crl(r + side, 1) * lc;
      g[4 - r] += T::crl(r + side, 2) * lc;
      const R la = (cand[r] - V) * iS * lam;
      const R d = T::dd(side ? r : 2 - r);
      ltau += d * ib[r] * la;
      lbeta[r] -= d * tau * ib[r] * ib[r] * la;
    }
  }
  lbeta[0] += sg * ltau;
  lbeta[2] -= sg * ltau;
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const R l1 = R(13.0 / 6.0) * b1[r] * lbeta[r];
    const R l2 = R(0.5) * b2[r] * lbeta[r];
    g[2 - r] += l1 + T::brl(r, 0) * l2;
    g[3 - r] += R(-2) * l1 + T::brl(r, 1) * l2;
    g[4 - r] += l1 + T::brl(r, 2) * l2;
  }
}

// psi tile index of cell (i, j, k) on axis d with tile index t along d (the stage kernel's
// indexing of psix / psiy / psiz)
template <class R>
__device__ __forceinline__ int64_t psi_index(const AdjStageArgs<R>& A, int d, int i, int j, int k, int t) {
  const int64_t d2 = A.pml_d2;
  if (d == 0) return t + d2 * ((int64_t)j + (int64_t)A.Ny * k);
  if (d == 1) return (int64_t)i + (int64_t)A.Nx * ((int64_t)t + d2 * k);
  return (int64_t)i + (int64_t)A.Nx * ((int64_t)j + (int64_t)A.Ny * t);
}

// Weighted output adjoint of cell (i, j, k) for the flux differences along axis d, as the pair
// (pressure, velocity d): the coefficient of (F_lo - F_hi) in the cell's outputs (and, in stage 2,
// in psi^{n+1}) applied to their adjoints. Zero for cells the stage kernel does not update.
template <class R>
__device__ __forceinline__ void adj_g(const AdjStageArgs<R>& A, int d, int i, int j, int k, R& gp, R& gv) {
  typedef typename Pair<R>::T P;
  const int64_t c = XOFF + i + A.Sx * ((int64_t)j + (int64_t)A.Ny * k);
  gp = R(0);
  gv = R(0);
  if (!(A.cls[c] & CLS_UPDATE)) return;
  const R* lvel = (d == 0) ? A.lu : (d == 1) ? A.lv : A.lw;
  R coef = A.cb;
  if (A.pml_on) {
    const PmlCoef<R> pc = (d == 0) ? A.pcx[i] : (d == 1) ? A.pcy[j] : A.pcz[k];
    if (pc.tile >= 0) {
      coef += A.wdt * pc.kinv1 * A.inv_h;
      if (A.stage == 2) {
        const P* lpsi = (d == 0) ? A.lpsix : (d == 1) ? A.lpsiy : A.lpsiz;
        const P l = lpsi[psi_index(A, d, i, j, k, pc.tile)];
        gp = pc.ca * A.inv_h * l.x;
        gv = pc.ca * A.inv_h * l.y;
      }
    }
  }
  gp += coef * A.lp[c];
  gv += coef * lvel[c];
}

template <class R>
__global__ void __launch_bounds__(256) k_adj_centres(const AdjStageArgs<R> A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= A.Nx || j >= A.Ny || k >= A.Nz) return;
  const int64_t c = XOFF + i + A.Sx * ((int64_t)j + (int64_t)A.Ny * k);
  const int64_t st[3] = {1, A.Sx, A.plane};
  const int N[3] = {A.Nx, A.Ny, A.Nz};
  const int cd[3] = {i, j, k};
  for (int d = 0; d < 3; d++) {
    R gP[5] = {R(0), R(0), R(0), R(0), R(0)};
    R gV[5] = {R(0), R(0), R(0), R(0), R(0)};
    if (cd[d] >= 2 && cd[d] <= N[d] - 3) {
      R gpm, gvm, gp0, gv0, gpp, gvp;
      const int di = (d == 0), dj = (d == 1), dk = (d == 2);
      adj_g(A, d, i - di, j - dj, k - dk, gpm, gvm);
      adj_g(A, d, i, j, k, gp0, gv0);
      adj_g(A, d, i + di, j + dj, k + dk, gpp, gvp);
      if (gpm != R(0) || gvm != R(0) || gp0 != R(0) || gv0 != R(0) || gpp != R(0) || gvp != R(0)) {
        // face adjoints: F(c+1/2) enters L(c) with -1 and L(c+1) with +1
        const R lFp_hi = gpp - gp0, lFu_hi = gvp - gv0;
        const R lFp_lo = gp0 - gpm, lFu_lo = gv0 - gvm;
        // V-(c+1/2) is the left state of face c+1/2, V+(c-1/2) the right state of face c-1/2
        const R lpm = A.fc * lFp_hi + A.firho * lFu_hi;
        const R lum = A.frc2 * lFp_hi + A.fc * lFu_hi;
        const R lpp = -A.fc * lFp_lo + A.firho * lFu_lo;
        const R lup = A.frc2 * lFp_lo - A.fc * lFu_lo;
        const R* vel = (d == 0) ? A.ui : (d == 1) ? A.vi : A.wi;
        R up[5], uv[5];
#pragma unroll
        for (int q = 0; q < 5; q++) {
          up[q] = A.pi[c + (q - 2) * st[d]];
          uv[q] = vel[c + (q - 2) * st[d]];
        }
        weno_centre_rev<R>(up, lpm, lpp, gP);
        weno_centre_rev<R>(uv, lum, lup, gV);
      }
    }
#pragma unroll
    for (int q = 0; q < 5; q++) {
      A.contrib[(int64_t)((d * 5 + q) * 2 + 0) * A.ncell + c] = gP[q];
      A.contrib[(int64_t)((d * 5 + q) * 2 + 1) * A.ncell + c] = gV[q];
    }
  }
}

template <class R>
__global__ void __launch_bounds__(256) k_adj_gather(const AdjStageArgs<R> A) {
  typedef typename Pair<R>::T P;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= A.Nx || j >= A.Ny || k >= A.Nz) return;
  const int64_t c = XOFF + i + A.Sx * ((int64_t)j + (int64_t)A.Ny * k);
  const int64_t st[3] = {1, A.Sx, A.plane};
  const int N[3] = {A.Nx, A.Ny, A.Nz};
  const int cd[3] = {i, j, k};
  R sp = R(0), sv[3] = {R(0), R(0), R(0)};
  for (int d = 0; d < 3; d++) {
#pragma unroll
    for (int q = 0; q < 5; q++) {
      const int src = cd[d] - (q - 2);  // the centre whose offset q - 2 lands on this cell
      if (src < 0 || src >= N[d]) continue;
      const int64_t cc = c - (q - 2) * st[d];
      sp += A.contrib[(int64_t)((d * 5 + q) * 2 + 0) * A.ncell + cc];
      sv[d] += A.contrib[(int64_t)((d * 5 + q) * 2 + 1) * A.ncell + cc];
    }
  }
  R ap = sp, au = sv[0], av = sv[1], aw = sv[2];
  if (A.cls[c] & CLS_UPDATE) {
    const R Lp = A.lp[c], Lu = A.lu[c], Lv = A.lv[c], Lw = A.lw[c];
    ap += A.b_in * Lp;
    au += A.b_in * Lu;
    av += A.b_in * Lv;
    aw += A.b_in * Lw;
    if (A.stage > 0) {
      A.bp[c] += A.a_base * Lp;
      A.bu[c] += A.a_base * Lu;
      A.bv[c] += A.a_base * Lv;
      A.bw[c] += A.a_base * Lw;
    }
    if (A.pml_on) {
      const PmlCoef<R> pc[3] = {A.pcx[i], A.pcy[j], A.pcz[k]};
      const R Lvel[3] = {Lu, Lv, Lw};
      P* lpsi[3] = {A.lpsix, A.lpsiy, A.lpsiz};
      for (int d = 0; d < 3; d++) {
        if (pc[d].tile < 0) continue;
        const int64_t x = psi_index(A, d, i, j, k, pc[d].tile);
        P l = lpsi[d][x];
        if (A.stage == 2) {  // psi^{n+1} = b psi^n + ca D: carry b, then psi^n's own uses
          l.x *= pc[d].b;
          l.y *= pc[d].b;
        }
        l.x += A.wdt * Lp;
        l.y += A.wdt * Lvel[d];
        lpsi[d][x] = l;
      }
    }
  }
  A.ip[c] += ap;
  A.iu[c] += au;
  A.iv[c] += av;
  A.iw[c] += aw;
}

template <class R, int STAGE>
__global__ void __launch_bounds__(256) k_adj_band(const AdjBandArgs<R> B, int use_smem) {
  extern __shared__ double sgrad[];
  const int P = 1 + 2 * B.K + 4 * B.L;
  const int ng = B.nMat * P;
  if (use_smem) {
    for (int e = threadIdx.x; e < ng; e += blockDim.x) sgrad[e] = 0.0;
    __syncthreads();
  }
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b < B.nB) {
    double* gacc = use_smem ? sgrad : B.grad;
    const int4 rc = B.rec[b];
    const int64_t cell = (int64_t)(((uint64_t)(uint32_t)rc.y << 32) | (uint32_t)rc.x);
    const int64_t q = cell + rc.z;
    const int m = rc.w;
    const R sx = B.geo[4 * b + 0], sy = B.geo[4 * b + 1], sz = B.geo[4 * b + 2], chi = B.geo[4 * b + 3];
    const R nx = B.nrm[4 * b + 0], ny = B.nrm[4 * b + 1], nz = B.nrm[4 * b + 2];
    const int64_t Sx = B.Sx, pl = B.plane;
    const int64_t off[8] = {0, 1, Sx, Sx + 1, pl, pl + 1, pl + Sx, pl + Sx + 1};
    const R wt[8] = {(R(1) - sx) * (R(1) - sy) * (R(1) - sz), sx * (R(1) - sy) * (R(1) - sz),
                     (R(1) - sx) * sy * (R(1) - sz),           sx * sy * (R(1) - sz),
                     (R(1) - sx) * (R(1) - sy) * sz,           sx * (R(1) - sy) * sz,
                     (R(1) - sx) * sy * sz,                    sx * sy * sz};
    // forward values needed by the linearisation (the probe as the forward evaluates it)
    auto tri = [&](const R* f) {
      const R c00 = f[q] * (R(1) - sx) + f[q + 1] * sx;
      const R c10 = f[q + Sx] * (R(1) - sx) + f[q + Sx + 1] * sx;
      const R c01 = f[q + pl] * (R(1) - sx) + f[q + pl + 1] * sx;
      const R c11 = f[q + pl + Sx] * (R(1) - sx) + f[q + pl + Sx + 1] * sx;
      const R c0 = c00 * (R(1) - sy) + c10 * sy, c1 = c01 * (R(1) - sy) + c11 * sy;
      return c0 * (R(1) - sz) + c1 * sz;
    };
    const R pD = tri(B.pi), uD = tri(B.ui), vD = tri(B.vi), wD = tri(B.wi);
    const R un = uD * nx + vD * ny + wD * nz;
    const double Z0 = B.Z0, dt = B.dt;
    const double wout = (double)pD + Z0 * (double)un;
    constexpr double aa = (STAGE == 0) ? 0.0 : (STAGE == 1) ? 3.0 : 1.0;
    constexpr double bb = (STAGE == 2) ? 2.0 : 1.0;
    constexpr double ic = (STAGE == 0) ? 1.0 : (STAGE == 1) ? 0.25 : 1.0 / 3.0;
    // output adjoint at the band cell: blend out = (1 - chi) pre + chi (pb, ub)
    const R Lp = B.lp[cell], Lu = B.lu[cell], Lv = B.lv[cell], Lw = B.lw[cell];
    const R omc = R(1) - chi;
    B.lp[cell] = omc * Lp;
    B.lu[cell] = omc * Lu;
    B.lv[cell] = omc * Lv;
    B.lw[cell] = omc * Lw;
    const double lpb = (double)chi * Lp;
    const double lux = (double)chi * Lu, luy = (double)chi * Lv, luz = (double)chi * Lw;
    const double lunb = nx * lux + ny * luy + nz * luz;
    const double lwin = 0.5 * lpb - lunb / (2.0 * Z0);
    double lwout = 0.5 * lpb + lunb / (2.0 * Z0);
    double* g = gacc + (int64_t)m * P;
    const int64_t nB = B.nB;
    atomicAdd(&g[0], wout * lwin);
    lwout += B.Rinf[m] * lwin;
    for (int k = 0; k < B.K; ++k) {
      const int mi = m * B.K + k;
      const int64_t si = (int64_t)k * nB + b;
      const double lphi = B.gphL[si] + B.A[mi] * lwin;
      const double phR = B.phR[si];
      atomicAdd(&g[1 + k], B.phL[si] * lwin);
      atomicAdd(&g[1 + B.K + k], -bb * dt * phR * ic * lphi);
      B.gphR[si] += bb * (1.0 - dt * B.zeta[mi]) * ic * lphi;
      if (STAGE > 0) B.gphM[si] += aa * ic * lphi;
      lwout += bb * dt * ic * lphi;
    }
    const int o = 1 + 2 * B.K;
    for (int l = 0; l < B.L; ++l) {
      const int mi = m * B.L + l;
      const int64_t si = (int64_t)l * nB + b;
      const double l1 = B.gs1L[si] + B.B[mi] * lwin;
      const double l2 = B.gs2L[si] + B.C[mi] * lwin;
      const double r1 = B.s1R[si], r2 = B.s2R[si];
      const double al = B.alpha[mi], be = B.beta[mi];
      const double kd = bb * dt * ic;
      atomicAdd(&g[o + l], B.s1L[si] * lwin);
      atomicAdd(&g[o + B.L + l], B.s2L[si] * lwin);
      atomicAdd(&g[o + 2 * B.L + l], kd * (-r1 * l1 - r2 * l2));
      atomicAdd(&g[o + 3 * B.L + l], kd * (-r2 * l1 + r1 * l2));
      B.gs1R[si] += bb * ic * l1 - kd * al * l1 + kd * be * l2;
      B.gs2R[si] += -kd * be * l1 + bb * ic * l2 - kd * al * l2;
      if (STAGE > 0) {
        B.gs1M[si] += aa * ic * l1;
        B.gs2M[si] += aa * ic * l2;
      }
      lwout += kd * l1;
    }
    // wout = pD + Z0 un; ub = unb n + (uD - un n)
    const double lun = Z0 * lwout - (nx * lux + ny * luy + nz * luz);
    const R lpD = (R)lwout;
    const R luD = (R)(lux + lun * nx), lvD = (R)(luy + lun * ny), lwD = (R)(luz + lun * nz);
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const int64_t x = q + off[e];
      atomicAdd(B.ip + x, wt[e] * lpD);
      atomicAdd(B.iu + x, wt[e] * luD);
      atomicAdd(B.iv + x, wt[e] * lvD);
      atomicAdd(B.iw + x, wt[e] * lwD);
    }
  }
  if (use_smem) {
    __syncthreads();
    for (int e = threadIdx.x; e < ng; e += blockDim.x)
      if (sgrad[e] != 0.0) atomicAdd(&B.grad[e], sgrad[e]);
  }
}

template <class R>
__global__ void k_adj_receivers(R* lp, const int64_t* rcell, int nrec, const double* ir, int64_t cap,
                                const double* target, int64_t tlen, int64_t n) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int r = 0; r < nrec; r++)  // one thread: receivers may share a cell
    lp[rcell[r]] += (R)(2.0 * (ir[(int64_t)r * cap + n] - target[(int64_t)r * tlen + n]));
}

template <class R>
__global__ void k_clear_inactive(R* f, const uint8_t* cls, int64_t n) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
    if (!(cls[c] & (CLS_UPDATE | CLS_BAND))) f[c] = R(0);
}

template <class R>
dim3 cell_grid(const AdjStageArgs<R>& a) {
  return dim3((unsigned)((a.Nx + 63) / 64), (unsigned)((a.Ny + 3) / 4), (unsigned)a.Nz);
}

}  // namespace

template <class R>
cudaError_t launch_adj_centres(const AdjStageArgs<R>& a, cudaStream_t s) {
  k_adj_centres<R><<<cell_grid(a), dim3(64, 4, 1), 0, s>>>(a);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_adj_gather(const AdjStageArgs<R>& a, cudaStream_t s) {
  k_adj_gather<R><<<cell_grid(a), dim3(64, 4, 1), 0, s>>>(a);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_adj_band(int stage, const AdjBandArgs<R>& a, cudaStream_t s) {
  if (a.nB <= 0) return cudaSuccess;
  const int bs = 256;
  const unsigned nb = (unsigned)((a.nB + bs - 1) / bs);
  const size_t gbytes = (size_t)a.nMat * (1 + 2 * a.K + 4 * a.L) * sizeof(double);
  const int use_smem = gbytes <= 32768 ? 1 : 0;
  const size_t smem = use_smem ? gbytes : 0;
  if (stage == 0)
    k_adj_band<R, 0><<<nb, bs, smem, s>>>(a, use_smem);
  else if (stage == 1)
    k_adj_band<R, 1><<<nb, bs, smem, s>>>(a, use_smem);
  else
    k_adj_band<R, 2><<<nb, bs, smem, s>>>(a, use_smem);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_adj_receivers(R* lp, const int64_t* rcell, int nrec, const double* ir, int64_t cap,
                                 const double* target, int64_t tlen, int64_t n, cudaStream_t s) {
  k_adj_receivers<R><<<1, 32, 0, s>>>(lp, rcell, nrec, ir, cap, target, tlen, n);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_clear_inactive(R* f, const uint8_t* cls, int64_t n, cudaStream_t s) {
  k_clear_inactive<R><<<592, 256, 0, s>>>(f, cls, n);
  return cudaGetLastError();
}

#define FZ_ADJ_INSTANTIATE(R)                                                                        \
  template cudaError_t launch_adj_centres<R>(const AdjStageArgs<R>&, cudaStream_t);                  \
  template cudaError_t launch_adj_gather<R>(const AdjStageArgs<R>&, cudaStream_t);                   \
  template cudaError_t launch_adj_band<R>(int, const AdjBandArgs<R>&, cudaStream_t);                 \
  template cudaError_t launch_adj_receivers<R>(R*, const int64_t*, int, const double*, int64_t,      \
                                               const double*, int64_t, int64_t, cudaStream_t);       \
  template cudaError_t launch_clear_inactive<R>(R*, const uint8_t*, int64_t, cudaStream_t);

FZ_ADJ_INSTANTIATE(float)
FZ_ADJ_INSTANTIATE(double)

}  // namespace fz
