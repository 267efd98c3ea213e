// fz_adjoint.cu -- discrete adjoint of one SSP-RK3 step of the stepping kernels: the transposed
// linearisation of WENO-Z (weights included; |beta0 - beta2| takes the subgradient sign(0) = 0),
// the Godunov flux, the RK combination, the cPML correction and psi recursion, the immersed band
// (trilinear probe, characteristic split, chi blend) and the ADE pole recursion, with the
// gradient with respect to the ADE coefficients. The forward scheme is the reference's
// (3D-solver/core/functions3D.cuh:56-78, 411-565, 661-1001, 1086-1327); the reference has no
// adjoint. Arithmetic follows the restated formulas (as the CPU oracle writes them), not the
// forward kernels' rearranged forms: both are the same function.
#include <algorithm>

#include "fz_adjoint.h"
#include "fz_pair.cuh"

namespace fz {

namespace {

// Reverse mode of one WENO-Z cell centre for a pair of variables (pressure and the velocity
// component along the sweep): u[0..4] are the values at c-2 .. c+2; the centre gives V-(c+1/2)
// (lam_m, its adjoint) and V+(c-1/2) (lam_p) from one set of smoothness indicators, as the
// stepping kernels' weno_core computes them (first differences a..d, second differences D_r,
// E_r, 12/13-scaled indicators B_r, q_r = 1 + tau/B_r, normalisers Sm, Sp). g[0..4] += lam_m
// dV-/du + lam_p dV+/du. The forward part is recomputed; reciprocals are differentiated as exact
// 1/x. tau = |B0 - B2| takes the subgradient sign(0) = 0.
template <class R>
__device__ __forceinline__ void weno_centre_rev(const typename Pair<R>::T u[5], typename Pair<R>::T lam_m,
                                                typename Pair<R>::T lam_p, typename Pair<R>::T g[5]) {
  typedef typename Pair<R>::T P;
  auto K = [](double x) { return psplat<R>(R(x)); };
  // ---- forward (weno_core)
  const P a = psub(u[1], u[0]), b = psub(u[2], u[1]), c = psub(u[3], u[2]), d = psub(u[4], u[3]);
  const P D2 = psub(b, a), D1 = psub(c, b), D0 = psub(d, c);
  const P E2 = pfma(b, K(2.0), D2), E1 = padd(b, c), E0 = pfma(c, K(-2.0), D0);
  const P k313 = K(3.0 / 13.0), eps = K(1e-10 * 12.0 / 13.0);
  const P B0 = pfma(D0, D0, pfma(pmul(E0, k313), E0, eps));
  const P B1 = pfma(D1, D1, pfma(pmul(E1, k313), E1, eps));
  const P B2 = pfma(D2, D2, pfma(pmul(E2, k313), E2, eps));
  const P diff = psub(B0, B2);
  const P tau = pabs(diff);
  const P rB0 = prcp(B0), rB1 = prcp(B1), rB2 = prcp(B2);
  const P one = K(1.0);
  const P q0 = pfma(tau, rB0, one), q1 = pfma(tau, rB1, one), q2 = pfma(tau, rB2, one);
  const P t1 = pmul(q1, K(0.6));
  const P Sm = pfma(q0, K(0.3), pfma(q2, K(0.1), t1));
  const P Sp = pfma(q0, K(0.1), pfma(q2, K(0.3), t1));
  const P h1 = pmul(D1, K(0.05));
  const P em0 = pfma(c, K(0.15), pmul(D0, K(-0.05)));
  const P ep0 = pfma(c, K(-0.05), pmul(D0, K(1.0 / 30.0)));
  const P em1 = pfma(E1, K(0.15), h1);
  const P ep1 = pfma(E1, K(-0.15), h1);
  const P em2 = pfma(b, K(0.05), pmul(D2, K(1.0 / 30.0)));
  const P ep2 = pfma(b, K(-0.15), pmul(D2, K(-0.05)));
  const P Nm = pfma(q2, em2, pfma(q1, em1, pmul(q0, em0)));
  const P Np = pfma(q2, ep2, pfma(q1, ep1, pmul(q0, ep0)));
  const P rSm = prcp(Sm), rSp = prcp(Sp);
  // ---- reverse: vm = q0c + Nm / Sm, vp = q0c + Np / Sp
  const P tm = pmul(lam_m, rSm), tp = pmul(lam_p, rSp);  // adjoints of Nm, Np
  const P lSm = pmul(tm, pmul(Nm, rSm)), lSp = pmul(tp, pmul(Np, rSp));  // minus the adjoints of Sm, Sp
  // adjoints of q_r (with the Sm, Sp signs folded in)
  const P lq0 = pfma(tp, ep0, pfma(tm, em0, pfma(lSm, K(-0.3), pmul(lSp, K(-0.1)))));
  const P lq1 = pfma(tp, ep1, pfma(tm, em1, pmul(padd(lSm, lSp), K(-0.6))));
  const P lq2 = pfma(tp, ep2, pfma(tm, em2, pfma(lSm, K(-0.1), pmul(lSp, K(-0.3)))));
  // adjoints of the first and second differences through em_r, ep_r (d/d em_r = tm q_r, d/d ep_r = tp q_r)
  P lc = pmul(q0, pfma(tm, K(0.15), pmul(tp, K(-0.05))));
  P lD0 = pmul(q0, pfma(tm, K(-0.05), pmul(tp, K(1.0 / 30.0))));
  P lE1 = pmul(pmul(q1, K(0.15)), psub(tm, tp));
  P lD1 = pmul(pmul(q1, K(0.05)), padd(tm, tp));
  P lb = pmul(q2, pfma(tm, K(0.05), pmul(tp, K(-0.15))));
  P lD2 = pmul(q2, pfma(tm, K(1.0 / 30.0), pmul(tp, K(-0.05))));
  // q_r = 1 + tau rB_r: d/dtau = rB_r, d/dB_r = -tau rB_r^2 = -(q_r - 1) rB_r
  const P ltau = pfma(lq2, rB2, pfma(lq1, rB1, pmul(lq0, rB0)));
  const P sl = pmk(diff.x > R(0) ? ltau.x : (diff.x < R(0) ? -ltau.x : R(0)),
                   diff.y > R(0) ? ltau.y : (diff.y < R(0) ? -ltau.y : R(0)));
  // twice the adjoints of B_r (B_r = D_r^2 + 3/13 E_r^2 + eps)
  const P m2 = K(-2.0);
  const P lB0 = pfma(pmul(lq0, psub(q0, one)), pmul(rB0, m2), padd(sl, sl));
  const P lB1 = pmul(pmul(lq1, psub(q1, one)), pmul(rB1, m2));
  const P lB2 = psub(pmul(pmul(lq2, psub(q2, one)), pmul(rB2, m2)), padd(sl, sl));
  lD0 = pfma(D0, lB0, lD0);
  lD1 = pfma(D1, lB1, lD1);
  lD2 = pfma(D2, lB2, lD2);
  const P lE0 = pmul(pmul(E0, k313), lB0);
  lE1 = pfma(pmul(E1, k313), lB1, lE1);
  const P lE2 = pmul(pmul(E2, k313), lB2);
  // E2 = 2b + D2, E1 = b + c, E0 = -2c + D0
  lb = pfma(lE2, K(2.0), padd(lb, lE1));
  lD2 = padd(lD2, lE2);
  lc = pfma(lE0, K(-2.0), padd(lc, lE1));
  lD0 = padd(lD0, lE0);
  // D2 = b - a, D1 = c - b, D0 = d - c
  lb = psub(padd(lb, lD2), lD1);
  lc = psub(padd(lc, lD1), lD0);
  const P la = pmul(lD2, K(-1.0));
  const P ld = lD0;
  // a = u1 - u0, b = u2 - u1, c = u3 - u2, d = u4 - u3; u2 is also the value both faces start from
  g[0] = psub(g[0], la);
  g[1] = padd(g[1], psub(la, lb));
  g[2] = padd(g[2], padd(psub(lb, lc), padd(lam_m, lam_p)));
  g[3] = padd(g[3], psub(lc, ld));
  g[4] = padd(g[4], ld);
}

// Adjoint of the Godunov flux of a face: the adjoints of its left state (from the face's
// adjoint lF) and of its right state, each as a (pressure, velocity) pair.
template <class R>
__device__ __forceinline__ typename Pair<R>::T god_left(const AdjStageArgs<R>& A, typename Pair<R>::T lF) {
  return pfma(psplat<R>(A.fc), lF, pmul(pswap(lF), pmk(A.firho, A.frc2)));
}
template <class R>
__device__ __forceinline__ typename Pair<R>::T god_right(const AdjStageArgs<R>& A, typename Pair<R>::T lF) {
  return pfma(psplat<R>(-A.fc), lF, pmul(pswap(lF), pmk(A.firho, A.frc2)));
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

// Shared-memory layout of the fused stage adjoint (units of R). Two buffers of raw plane tiles
// with a 4-cell x/y halo (40 x 24): the stage input p, u, v, the output adjoint lp, lu, lv and the
// class bytes -- the next plane's arrives while the current one is worked on. Then the
// flux-difference weights g of the x faces (38 x 16 pairs) and y faces (32 x 22 pairs), and the
// five stencil contributions of every x centre (36 x 16) and y centre (32 x 20) of the tile and
// its 2-cell halo.
template <class R>
struct AdjSmem {
  static constexpr int TW = ATX + 8, TH = ATY + 8, TN = TW * TH;
  static constexpr int GXW = ATX + 6, GYH = ATY + 6;
  static constexpr int XCW = ATX + 4, YCH = ATY + 4;
  static constexpr int NX_C = XCW * ATY, NY_C = ATX * YCH;
  static constexpr int RAW = 6 * TN;  // p, u, v, lp, lu, lv of one plane
  static constexpr int G_X = 2 * RAW;
  static constexpr int G_Y = G_X + 2 * GXW * ATY;
  static constexpr int X_C = G_Y + 2 * ATX * GYH;
  static constexpr int Y_C = X_C + 2 * 5 * NX_C;
  static constexpr int END = Y_C + 2 * 5 * NY_C;
  static constexpr size_t CLS_OFF = (size_t)END * sizeof(R);  // two class-byte tiles
  static constexpr size_t PML_OFF = (CLS_OFF + 2 * TN + 31) & ~(size_t)31;
  // cPML coefficients of the tile's x range (38), y range (22) and the chunk's z range (chunk + 6)
  static size_t bytes(int kz_chunk) { return PML_OFF + (size_t)(ATX + 6 + ATY + 6 + kz_chunk + 6) * sizeof(PmlCoef<R>); }
};

// Weighted output adjoint of cell (i, j, k) for the flux differences along axis d, as the pair
// (pressure, velocity d): the coefficient of (F_lo - F_hi) in the cell's outputs (and, in stage 2,
// in psi^{n+1}) applied to their adjoints; lp, lvel are the cell's output adjoints, pc its cPML
// coefficient along d. Zero for cells the stage kernel does not update.
template <class R>
__device__ __forceinline__ void adj_g_local(const AdjStageArgs<R>& A, int d, int i, int j, int k, uint8_t cls,
                                            R lp, R lvel, const PmlCoef<R>& pc, R& gp, R& gv) {
  typedef typename Pair<R>::T P;
  gp = R(0);
  gv = R(0);
  if (!(cls & CLS_UPDATE)) return;
  R coef = A.cb;
  if (A.pml_on && pc.tile >= 0) {
    coef += A.wdt * pc.kinv1 * A.inv_h;
    if (A.stage == 2) {
      const P* lpsi = (d == 0) ? A.lpsix : (d == 1) ? A.lpsiy : A.lpsiz;
      const int64_t x = psi_index(A, d, i, j, k, pc.tile);
      if (fz_inb(A.err, x, A.npsi[d])) {
        const P l = lpsi[x];
        gp = pc.ca * A.inv_h * l.x;
        gv = pc.ca * A.inv_h * l.y;
      }
    }
  }
  gp += coef * lp;
  gv += coef * lvel;
}

// Adjoint of one stage kernel launch. CTA = 32 x 16 columns marching up a z chunk, as the forward
// stage kernel. At centre plane kc: the x and y centres of the tile and its 2-cell halo through
// shared memory (each centre's five contributions written once, then gathered by the five cells
// they land on), the z centre of every column (register queues of p, w and of the z weights),
// and the flush of plane kc - 2, whose z contributions are complete once centre kc is done. The
// global loads of the next plane, of the z queues and of the flush are issued at the top of the
// iteration and consumed after the x/y work. Two barriers per plane: after the face weights, and
// after the centres (which also publishes the next plane's raw tiles, stashed just before it).
template <class R>
__global__ void __launch_bounds__(ANTHREADS, 1) k_adj_stage(const AdjStageArgs<R> A) {
  typedef typename Pair<R>::T P;
  typedef AdjSmem<R> S;
  extern __shared__ __align__(16) unsigned char adj_smem[];
  R* sm = reinterpret_cast<R*>(adj_smem);
  P* gX = reinterpret_cast<P*>(sm + S::G_X);
  P* gY = reinterpret_cast<P*>(sm + S::G_Y);
  P* xC = reinterpret_cast<P*>(sm + S::X_C);
  P* yC = reinterpret_cast<P*>(sm + S::Y_C);
  uint8_t* clsT = adj_smem + S::CLS_OFF;
  PmlCoef<R>* sPx = reinterpret_cast<PmlCoef<R>*>(adj_smem + S::PML_OFF);  // x = i0 - 3 + q
  PmlCoef<R>* sPy = sPx + (ATX + 6);                                         // y = j0 - 3 + q
  PmlCoef<R>* sPz = sPy + (ATY + 6);                                         // k = kb - 3 + q

  const int tx = threadIdx.x, ty = threadIdx.y, lt = ty * ATX + tx;
  const int i0 = GHOST + blockIdx.x * ATX, j0 = GHOST + blockIdx.y * ATY;
  const int i = i0 + tx, j = j0 + ty;
  const int kb = GHOST + blockIdx.z * A.kz_chunk;
  const int ke = min(kb + A.kz_chunk, A.Nz - GHOST);
  if (kb >= ke) return;
  const int Nx = A.Nx, Ny = A.Ny, Nz = A.Nz;
  const int64_t Sx = A.Sx, plane = A.plane;
  const bool col_in = (i < Nx) && (j < Ny);
  const bool valid = (i < Nx - GHOST) && (j < Ny - GHOST);
  const int64_t col = XOFF + i + Sx * (int64_t)j;

  // raw-tile elements of this thread: e = lt and e = lt + 512 (when < 960)
  constexpr int NE = (S::TN + ANTHREADS - 1) / ANTHREADS;
  int64_t roff[NE];
  bool rin[NE];
#pragma unroll
  for (int q = 0; q < NE; q++) {
    const int e = lt + q * ANTHREADS;
    const int r = e / S::TW, ci = e - r * S::TW;
    const int x = i0 - 4 + ci, y = j0 - 4 + r;
    rin[q] = (e < S::TN) && x >= 0 && x < Nx && y >= 0 && y < Ny;
    roff[q] = rin[q] ? (XOFF + x + Sx * (int64_t)y) : 0;
  }
  R pre[NE][6];
  uint8_t prc[NE];
  auto prefetch = [&](int k) {
#pragma unroll
    for (int q = 0; q < NE; q++) {
      const int64_t g = roff[q] + plane * (int64_t)k;
      const bool ok = rin[q] && k < Nz && fz_inb(A.err, g, A.nfield);
      pre[q][0] = ok ? A.pi[g] : R(0);
      pre[q][1] = ok ? A.ui[g] : R(0);
      pre[q][2] = ok ? A.vi[g] : R(0);
      pre[q][3] = ok ? A.lp[g] : R(0);
      pre[q][4] = ok ? A.lu[g] : R(0);
      pre[q][5] = ok ? A.lv[g] : R(0);
      prc[q] = ok ? A.cls[g] : (uint8_t)0;
    }
  };
  auto stash = [&](int buf) {
    R* raw = sm + buf * S::RAW;
#pragma unroll
    for (int q = 0; q < NE; q++) {
      const int e = lt + q * ANTHREADS;
      if (e < S::TN) {
#pragma unroll
        for (int f = 0; f < 6; f++) raw[f * S::TN + e] = pre[q][f];
        clsT[buf * S::TN + e] = prc[q];
      }
    }
  };
  auto ldz = [&](const R* f, int k) -> R {
    return (col_in && k >= 0 && k < Nz && fz_inb(A.err, col + plane * k, A.nfield)) ? f[col + plane * k] : R(0);
  };

  // z queues at centre plane kc: values at kc-2 .. kc+2, weights at kc-1 .. kc+1, contribution
  // windows for planes kc-2 .. kc+2
  P zq[5], gzq[3], acq[5];  // (p, w) pairs
#pragma unroll
  for (int q = 0; q < 4; q++) zq[q] = pmk(ldz(A.pi, kb - 4 + q), ldz(A.wi, kb - 4 + q));
  {
    PmlCoef<R> none;
    none.tile = -1;
    none.kinv1 = none.b = none.ca = R(0);
    const int nz_t = A.kz_chunk + 6;
    for (int e = lt; e < ATX + 6 + ATY + 6 + nz_t; e += ANTHREADS) {
      PmlCoef<R> c = none;
      if (e < ATX + 6) {
        const int x = i0 - 3 + e;
        if (x >= 0 && x < Nx) c = A.pcx[x];
      } else if (e < ATX + 6 + ATY + 6) {
        const int y = j0 - 3 + (e - (ATX + 6));
        if (y >= 0 && y < Ny) c = A.pcy[y];
      } else {
        const int k = kb - 3 + (e - (ATX + 6 + ATY + 6));
        if (k >= 0 && k < Nz) c = A.pcz[k];
      }
      sPx[e] = c;
    }
  }
  __syncthreads();
  const PmlCoef<R> pci = sPx[tx + 3], pcj = sPy[ty + 3];
  auto gz_cell = [&](int k) -> P {
    R gp = R(0), gv = R(0);
    if (col_in && k >= 0 && k < Nz && fz_inb(A.err, col + plane * (int64_t)k, A.nfield)) {
      const int64_t c = col + plane * (int64_t)k;
      adj_g_local(A, 2, i, j, k, A.cls[c], A.lp[c], A.lw[c], sPz[k - kb + 3], gp, gv);
    }
    return pmk(gp, gv);
  };
  gzq[0] = gz_cell(kb - 3);
  gzq[1] = gz_cell(kb - 2);
#pragma unroll
  for (int q = 0; q < 5; q++) acq[q] = psplat<R>(R(0));
  R d1p = R(0), d1u = R(0), d1v = R(0), d2p = R(0), d2u = R(0), d2v = R(0);  // x/y sums of kc-1, kc-2

  prefetch(kb);
  stash(kb & 1);
  __syncthreads();  // raw tiles of plane kb stashed

  const int nit = (ke - kb) + 4;
  for (int it = 0; it < nit; ++it) {
    const int kc = kb - 2 + it;
    const bool xy = (kc >= kb && kc < ke);  // block-uniform
    // ---- loads for later in this iteration and for the next plane
    zq[4] = pmk(ldz(A.pi, kc + 2), ldz(A.wi, kc + 2));
    const int kz1 = kc + 1;
    const int64_t cz1 = col + plane * (int64_t)kz1;
    const bool z1 = col_in && kz1 >= 0 && kz1 < Nz && fz_inb(A.err, cz1, A.nfield);
    const uint8_t cls_z1 = z1 ? A.cls[cz1] : (uint8_t)0;
    const R lpz1 = z1 ? A.lp[cz1] : R(0), lwz1 = z1 ? A.lw[cz1] : R(0);
    const int kf = kc - 2;
    const int64_t cf = col + plane * (int64_t)kf;
    const bool fl = (kf >= kb) && valid && fz_inb(A.err, cf, A.nfield);
    const uint8_t cls_f = fl ? A.cls[cf] : (uint8_t)0;
    R Lf[4] = {R(0), R(0), R(0), R(0)};
    R Pf[4] = {R(0), R(0), R(0), R(0)};  // the accumulator this stage adds to (input or U0 adjoint)
    if (fl) {
      Lf[0] = A.lp[cf];
      Lf[1] = A.lu[cf];
      Lf[2] = A.lv[cf];
      Lf[3] = A.lw[cf];
      if (A.acc_in) {
        Pf[0] = A.ip[cf];
        Pf[1] = A.iu[cf];
        Pf[2] = A.iv[cf];
        Pf[3] = A.iw[cf];
      } else if (A.acc_base) {
        Pf[0] = A.bp[cf];
        Pf[1] = A.bu[cf];
        Pf[2] = A.bv[cf];
        Pf[3] = A.bw[cf];
      }
    }
    const bool nxt = (kc + 1 >= kb && kc + 1 < ke && kc + 1 > kb);  // plane kb is already stashed
    if (nxt) prefetch(kc + 1);

    // ---- x and y centres of plane kc
    R xyp = R(0), xyu = R(0), xyv = R(0);
    if (xy) {
      const R* raw = sm + (kc & 1) * S::RAW;
      const R* tP = raw;
      const R* tU = raw + S::TN;
      const R* tV = raw + 2 * S::TN;
      const R* tLp = raw + 3 * S::TN;
      const R* tLu = raw + 4 * S::TN;
      const R* tLv = raw + 5 * S::TN;
      const uint8_t* tC = clsT + (kc & 1) * S::TN;
      for (int e = lt; e < S::GXW * ATY + ATX * S::GYH; e += ANTHREADS) {
        R a, b;
        if (e < S::GXW * ATY) {
          const int r = e / S::GXW, ci = e - r * S::GXW;
          const int t = (r + 4) * S::TW + ci + 1;
          adj_g_local(A, 0, i0 - 3 + ci, j0 + r, kc, tC[t], tLp[t], tLu[t], sPx[ci], a, b);
          gX[e] = pmk(a, b);
        } else {
          const int f = e - S::GXW * ATY;
          const int r = f / ATX, ci = f - r * ATX;
          const int t = (r + 1) * S::TW + ci + 4;
          adj_g_local(A, 1, i0 + ci, j0 - 3 + r, kc, tC[t], tLp[t], tLv[t], sPy[r], a, b);
          gY[f] = pmk(a, b);
        }
      }
      __syncthreads();
      for (int e = lt; e < S::NX_C + S::NY_C; e += ANTHREADS) {
        P cc[5];
#pragma unroll
        for (int q = 0; q < 5; q++) cc[q] = psplat<R>(R(0));
        const bool isx = e < S::NX_C;
        const int f = isx ? e : e - S::NX_C;
        int r, ci, cpos, npos;
        P gm, g0, gp;
        if (isx) {
          r = f / S::XCW;
          ci = f - r * S::XCW;
          cpos = i0 - 2 + ci;
          npos = Nx;
          gm = gX[r * S::GXW + ci];
          g0 = gX[r * S::GXW + ci + 1];
          gp = gX[r * S::GXW + ci + 2];
        } else {
          r = f / ATX;
          ci = f - r * ATX;
          cpos = j0 - 2 + r;
          npos = Ny;
          gm = gY[r * ATX + ci];
          g0 = gY[(r + 1) * ATX + ci];
          gp = gY[(r + 2) * ATX + ci];
        }
        if (cpos >= 2 && cpos <= npos - 3) {
          // face adjoints: F(c+1/2) enters L(c) with -1 and L(c+1) with +1
          const P lF_hi = psub(gp, g0), lF_lo = psub(g0, gm);
          if (lF_hi.x != R(0) || lF_hi.y != R(0) || lF_lo.x != R(0) || lF_lo.y != R(0)) {
            // stencil cpos-2 .. cpos+2: tile columns ci .. ci+4 of row r+4 (x), or rows r .. r+4 of
            // column ci+4 (y)
            const int t0 = isx ? (r + 4) * S::TW + ci : r * S::TW + ci + 4;
            const int st = isx ? 1 : S::TW;
            const R* tw = isx ? tU : tV;
            P uq[5];
#pragma unroll
            for (int q = 0; q < 5; q++) uq[q] = pmk(tP[t0 + q * st], tw[t0 + q * st]);
            // V-(c+1/2) is the left state of face c+1/2, V+(c-1/2) the right state of face c-1/2
            weno_centre_rev<R>(uq, god_left(A, lF_hi), god_right(A, lF_lo), cc);
          }
        }
        P* dst = isx ? xC + f * 5 : yC + f * 5;
#pragma unroll
        for (int q = 0; q < 5; q++) dst[q] = cc[q];
      }
      // the next plane's raw tiles go into the other buffer (last read before the previous plane's
      // second barrier); the barrier below publishes them, so the next plane's weights (the first
      // phase) need no barrier of their own and share a phase with this plane's gather, z centre
      // and flush
      if (nxt) stash((kc + 1) & 1);
      __syncthreads();
      // cell (i, j) receives offset q - 2 of the x centre i - (q - 2) and of the y centre j - (q - 2)
#pragma unroll
      for (int q = 0; q < 5; q++) {
        const P a = xC[(ty * S::XCW + tx + 4 - q) * 5 + q];
        const P b = yC[((ty + 4 - q) * ATX + tx) * 5 + q];
        xyp += a.x + b.x;
        xyu += a.y;
        xyv += b.y;
      }
    }
    // ---- z centre kc
    {
      R gp, gv;
      adj_g_local(A, 2, i, j, kz1, cls_z1, lpz1, lwz1, sPz[kz1 - kb + 3], gp, gv);
      gzq[2] = pmk(gp, gv);
    }
    if (col_in && kc >= 2 && kc <= Nz - 3) {
      const P lF_hi = psub(gzq[2], gzq[1]), lF_lo = psub(gzq[1], gzq[0]);
      if (lF_hi.x != R(0) || lF_hi.y != R(0) || lF_lo.x != R(0) || lF_lo.y != R(0))
        weno_centre_rev<R>(zq, god_left(A, lF_hi), god_right(A, lF_lo), acq);
    }
    // ---- flush plane kc - 2: the stage input's adjoint (and U0's) at every interior cell
    if (fl) {
      R ip = d2p + acq[0].x, iu = d2u, iv = d2v, iw = acq[0].y;
      R bq[4] = {R(0), R(0), R(0), R(0)};
      if (cls_f & CLS_UPDATE) {
        ip += A.b_in * Lf[0];
        iu += A.b_in * Lf[1];
        iv += A.b_in * Lf[2];
        iw += A.b_in * Lf[3];
#pragma unroll
        for (int f = 0; f < 4; f++) bq[f] = A.a_base * Lf[f];
        if (A.pml_on) {
          const PmlCoef<R> pc[3] = {pci, pcj, sPz[kf - kb + 3]};
          const P* lin[3] = {A.lpsix, A.lpsiy, A.lpsiz};
          P* lout[3] = {A.opsix, A.opsiy, A.opsiz};
#pragma unroll
          for (int d = 0; d < 3; d++) {
            if (pc[d].tile < 0) continue;
            const int64_t x = psi_index(A, d, i, j, kf, pc[d].tile);
            if (!fz_inb(A.err, x, A.npsi[d])) continue;
            P l;
            if (A.stage == 2) {  // psi^{n+1} = b psi^n + ca D: carry b, then psi^n's own uses
              const P o = lin[d][x];
              l = pmk(pc[d].b * o.x, pc[d].b * o.y);
            } else {
              l = lout[d][x];
            }
            l.x += A.wdt * Lf[0];
            l.y += A.wdt * Lf[1 + d];
            lout[d][x] = l;
          }
        }
      }
      if (A.acc_in) {
        ip += Pf[0];
        iu += Pf[1];
        iv += Pf[2];
        iw += Pf[3];
      }
      A.ip[cf] = ip;
      A.iu[cf] = iu;
      A.iv[cf] = iv;
      A.iw[cf] = iw;
      if (A.stage > 0) {
        if (A.acc_base) {
#pragma unroll
          for (int f = 0; f < 4; f++) bq[f] += Pf[f];
        }
        A.bp[cf] = bq[0];
        A.bu[cf] = bq[1];
        A.bv[cf] = bq[2];
        A.bw[cf] = bq[3];
      }
    }
    // ---- advance the queues
    d2p = d1p; d2u = d1u; d2v = d1v;
    d1p = xyp; d1u = xyu; d1v = xyv;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      zq[q] = zq[q + 1];
      acq[q] = acq[q + 1];
    }
    acq[4] = psplat<R>(R(0));
    gzq[0] = gzq[1];
    gzq[1] = gzq[2];
  }
}

// One thread per band cell. Each cell's contributions to the coefficient gradients go to its own
// slots gcell[e][b] (no atomics); k_adj_grad_reduce sums them per material once, at the end.
template <class R, int STAGE>
__global__ void __launch_bounds__(256) k_adj_band(const AdjBandArgs<R> B) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B.nB) return;
  const int4 rc = B.rec[b];
  const int64_t cell = (int64_t)(((uint64_t)(uint32_t)rc.y << 32) | (uint32_t)rc.x);
  const int64_t q = cell + rc.z;
  const int m = rc.w;
  const int64_t nB = B.nB;
  if (!fz_inb(B.err, cell, B.nfield) || !fz_inb(B.err, q, B.nfield) ||
      !fz_inb(B.err, q + B.plane + B.Sx + 1, B.nfield))
    return;
  double* gc = B.gcell + b;
  auto gadd = [&](int e, double v) { gc[(int64_t)e * nB] += v; };
  const R sx = B.geo[4 * b + 0], sy = B.geo[4 * b + 1], sz = B.geo[4 * b + 2], chi = B.geo[4 * b + 3];
  const R nx = B.nrm[4 * b + 0], ny = B.nrm[4 * b + 1], nz = B.nrm[4 * b + 2];
  const int64_t Sx = B.Sx, pl = B.plane;
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
  // The ADE-state adjoints of the step (sweep order: stage 2, 1, 0): stage 2 writes the right set
  // (after stage 1) and the middle set (step start) first, stage 1 its right set (after stage 0)
  // first, so those writes assign and nothing has to zero the sets between steps; the others add.
  constexpr bool R_FIRST = STAGE > 0, M_FIRST = STAGE == 2;
  auto acc_r = [](double& x, double v) { x = R_FIRST ? v : x + v; };
  auto acc_m = [](double& x, double v) { x = M_FIRST ? v : x + v; };
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
  gadd(0, wout * lwin);
  lwout += B.Rinf[m] * lwin;
  for (int k = 0; k < B.K; ++k) {
    const int mi = m * B.K + k;
    const int64_t si = (int64_t)k * nB + b;
    const double lphi = B.gphL[si] + B.A[mi] * lwin;
    const double phR = B.phR[si];
    gadd(1 + k, B.phL[si] * lwin);
    gadd(1 + B.K + k, -bb * dt * phR * ic * lphi);
    acc_r(B.gphR[si], bb * (1.0 - dt * B.zeta[mi]) * ic * lphi);
    if (STAGE > 0) acc_m(B.gphM[si], aa * ic * lphi);
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
    gadd(o + l, B.s1L[si] * lwin);
    gadd(o + B.L + l, B.s2L[si] * lwin);
    gadd(o + 2 * B.L + l, kd * (-r1 * l1 - r2 * l2));
    gadd(o + 3 * B.L + l, kd * (-r2 * l1 + r1 * l2));
    acc_r(B.gs1R[si], bb * ic * l1 - kd * al * l1 + kd * be * l2);
    acc_r(B.gs2R[si], -kd * be * l1 + bb * ic * l2 - kd * al * l2);
    if (STAGE > 0) {
      acc_m(B.gs1M[si], aa * ic * l1);
      acc_m(B.gs2M[si], aa * ic * l2);
    }
    lwout += kd * l1;
  }
  // wout = pD + Z0 un; ub = unb n + (uD - un n)
  const double lun = Z0 * lwout - (nx * lux + ny * luy + nz * luz);
  const R lpD = (R)lwout;
  const R luD = (R)(lux + lun * nx), lvD = (R)(luy + lun * ny), lwD = (R)(luz + lun * nz);
  // the probe's adjoint, scattered into the stage input's adjoint after the stage adjoint
  B.probe[b] = lpD;
  B.probe[nB + b] = luD;
  B.probe[2 * nB + b] = lvD;
  B.probe[3 * nB + b] = lwD;
}

// Transposed trilinear probe: adds each band cell's probe adjoint to the 8 corner cells of the
// stage input's adjoint (corners of neighbouring band cells overlap, hence the atomics).
template <class R>
__global__ void __launch_bounds__(256) k_adj_probe_scatter(const AdjBandArgs<R> B) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B.nB) return;
  const int4 rc = B.rec[b];
  const int64_t cell = (int64_t)(((uint64_t)(uint32_t)rc.y << 32) | (uint32_t)rc.x);
  const int64_t q = cell + rc.z;
  if (!fz_inb(B.err, q, B.nfield) || !fz_inb(B.err, q + B.plane + B.Sx + 1, B.nfield)) return;
  const R sx = B.geo[4 * b + 0], sy = B.geo[4 * b + 1], sz = B.geo[4 * b + 2];
  const int64_t nB = B.nB, Sx = B.Sx, pl = B.plane;
  const R lpD = B.probe[b], luD = B.probe[nB + b], lvD = B.probe[2 * nB + b], lwD = B.probe[3 * nB + b];
  const int64_t off[8] = {0, 1, Sx, Sx + 1, pl, pl + 1, pl + Sx, pl + Sx + 1};
  const R wt[8] = {(R(1) - sx) * (R(1) - sy) * (R(1) - sz), sx * (R(1) - sy) * (R(1) - sz),
                   (R(1) - sx) * sy * (R(1) - sz),           sx * sy * (R(1) - sz),
                   (R(1) - sx) * (R(1) - sy) * sz,           sx * (R(1) - sy) * sz,
                   (R(1) - sx) * sy * sz,                    sx * sy * sz};
#pragma unroll
  for (int e = 0; e < 8; e++) {
    const int64_t x = q + off[e];
    atomicAdd(B.ip + x, wt[e] * lpD);
    atomicAdd(B.iu + x, wt[e] * luD);
    atomicAdd(B.iv + x, wt[e] * lvD);
    atomicAdd(B.iw + x, wt[e] * lwD);
  }
}

// grad[m][e] += sum of gcell[e][b] over the band cells b of material m (grad zeroed before): blocks
// (coefficient slot e, chunk of band cells), per-material bins in shared memory, one global atomic
// per bin and block.
constexpr int GRAD_CHUNK = 256 * 32;
__global__ void __launch_bounds__(256) k_adj_grad_reduce(const int4* rec, const double* gcell, int64_t nB, int P,
                                                         int nMat, double* grad) {
  extern __shared__ double bins[];
  const int e = blockIdx.x;
  for (int m = threadIdx.x; m < nMat; m += blockDim.x) bins[m] = 0.0;
  __syncthreads();
  const int64_t b0 = (int64_t)blockIdx.y * GRAD_CHUNK, b1 = min(nB, b0 + (int64_t)GRAD_CHUNK);
  for (int64_t b = b0 + threadIdx.x; b < b1; b += blockDim.x) atomicAdd(&bins[rec[b].w], gcell[(int64_t)e * nB + b]);
  __syncthreads();
  for (int m = threadIdx.x; m < nMat; m += blockDim.x)
    if (bins[m] != 0.0) atomicAdd(&grad[(int64_t)m * P + e], bins[m]);
}

template <class R>
__global__ void k_adj_receivers(R* lp, const int64_t* rcell, int nrec, const double* ir, int64_t cap,
                                const double* target, int64_t tlen, int64_t n, int cotangent) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int r = 0; r < nrec; r++) {  // one thread: receivers may share a cell
    const double t = target[(int64_t)r * tlen + n];
    lp[rcell[r]] += (R)(cotangent ? t : 2.0 * (ir[(int64_t)r * cap + n] - t));
  }
}

template <class R>
__global__ void k_adj_source(const R* lp, const int64_t* cell, int nsrc, const double* sval, double unit,
                             const R* u_s, int64_t n_us, int src_opt, const R* freq, R half_dt, double w, int64_t nn,
                             double* gsval, double* gwave) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nsrc) return;
  const double lam = (double)lp[cell[q]] * w * unit;
  double amp;
  if (src_opt == 2)  // the stage kernel's sine, in its precision
    amp = (double)(R)sin(2.0 * 3.14159265358979323846 * (double)freq[q] * (double)nn * (double)half_dt);
  else
    amp = (nn < n_us) ? (double)u_s[nn] : 0.0;
  if (gsval) gsval[q] += lam * amp;
  if (gwave && src_opt != 2 && nn < n_us) gwave[(int64_t)q * n_us + nn] += lam * sval[q];
}

template <class R>
__global__ void __launch_bounds__(256) k_adj_pml_grad(const AdjPmlArgs<R> A) {
  typedef typename Pair<R>::T P;
  extern __shared__ double gs[];  // [2d][3]
  const int d2 = 2 * A.d;
  for (int e = threadIdx.x; e < 3 * d2; e += blockDim.x) gs[e] = 0.0;
  __syncthreads();
  const int ex = A.Nx - 2 * GHOST, ey = A.Ny - 2 * GHOST, ez = A.Nz - 2 * GHOST;
  const int64_t E0 = (A.axis == 0) ? d2 : ex, E1 = (A.axis == 1) ? d2 : ey, E2 = (A.axis == 2) ? d2 : ez;
  const int Na = (A.axis == 0) ? A.Nx : (A.axis == 1) ? A.Ny : A.Nz;
  const int64_t st = (A.axis == 0) ? 1 : (A.axis == 1) ? A.Sx : A.plane;
  const int64_t total = E0 * E1 * E2;
  const P kA = pmk(A.frc2, A.firho);
  const P kC = psplat<R>(-A.fc);
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a0 = t % E0, r = t / E0;
    const int64_t a1 = r % E1, a2 = r / E1;
    const int tile = (int)((A.axis == 0) ? a0 : (A.axis == 1) ? a1 : a2);
    // psi tile index -> coordinate along the axis (layers [3, 3+d) and [N-3-d, N-3))
    const int ca = (tile < A.d) ? GHOST + tile : Na - GHOST - d2 + tile;
    if (A.pc[ca].tile != tile) continue;  // that face is not a cPML face
    const int i = (A.axis == 0) ? ca : GHOST + (int)a0;
    const int j = (A.axis == 1) ? ca : GHOST + (int)a1;
    const int k = (A.axis == 2) ? ca : GHOST + (int)a2;
    const int64_t g = XOFF + i + A.Sx * ((int64_t)j + (int64_t)A.Ny * k);
    if (!fz_inb(A.err, g - 3 * st, A.nfield) || !fz_inb(A.err, g + 3 * st, A.nfield)) continue;
    if (!(A.cls[g] & CLS_UPDATE)) continue;
    P q[7];
#pragma unroll
    for (int o = 0; o < 7; o++) q[o] = pmk(A.pi[g + (o - 3) * st], A.vi[g + (o - 3) * st]);
    P ml, pl, mc, pc, mr, pr;
    weno_center<R>(q[0], q[1], q[2], q[3], q[4], ml, pl);
    weno_center<R>(q[1], q[2], q[3], q[4], q[5], mc, pc);
    weno_center<R>(q[2], q[3], q[4], q[5], q[6], mr, pr);
    const P L = psub(godunov<R>(ml, pc, kA, kC), godunov<R>(mc, pr, kA, kC));
    const R Dp = L.x * A.inv_h, Dv = L.y * A.inv_h;
    atomicAdd(&gs[3 * tile], A.wdt * ((double)A.lp[g] * (double)Dp + (double)A.lv[g] * (double)Dv));
    if (A.stage == 2) {
      const int64_t X = (A.axis == 0)   ? tile + (int64_t)d2 * ((int64_t)j + (int64_t)A.Ny * k)
                        : (A.axis == 1) ? i + (int64_t)A.Nx * ((int64_t)tile + (int64_t)d2 * k)
                                        : i + (int64_t)A.Nx * ((int64_t)j + (int64_t)A.Ny * tile);
      if (!fz_inb(A.err, X, A.npsi)) continue;
      const P lps = A.lpsi[X], ps = A.psin[X];
      atomicAdd(&gs[3 * tile + 1], (double)lps.x * (double)ps.x + (double)lps.y * (double)ps.y);
      atomicAdd(&gs[3 * tile + 2], (double)lps.x * (double)Dp + (double)lps.y * (double)Dv);
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 3 * d2; e += blockDim.x)
    if (gs[e] != 0.0) atomicAdd(&A.g[e], gs[e]);
}

template <class R>
__global__ void k_clear_inactive(R* f, const uint8_t* cls, int64_t n) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
    if (!(cls[c] & (CLS_UPDATE | CLS_BAND))) f[c] = R(0);
}

}  // namespace

template <class R>
size_t adj_stage_smem(int kz_chunk) {
  return AdjSmem<R>::bytes(kz_chunk);
}

template <class R>
cudaError_t adj_stage_setup(size_t smem_bytes) {
  return cudaFuncSetAttribute((const void*)k_adj_stage<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem_bytes);
}

template <class R>
cudaError_t adj_stage_occupancy(int* blocks_per_sm, size_t smem_bytes) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_adj_stage<R>, ANTHREADS, smem_bytes);
}

template <class R>
cudaError_t launch_adj_stage(const AdjStageArgs<R>& a, dim3 grid, cudaStream_t s) {
  k_adj_stage<R><<<grid, dim3(ATX, ATY, 1), AdjSmem<R>::bytes(a.kz_chunk), s>>>(a);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_adj_probe_scatter(const AdjBandArgs<R>& a, cudaStream_t s) {
  if (a.nB <= 0) return cudaSuccess;
  k_adj_probe_scatter<R><<<(unsigned)((a.nB + 255) / 256), 256, 0, s>>>(a);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_adj_band(int stage, const AdjBandArgs<R>& a, cudaStream_t s) {
  if (a.nB <= 0) return cudaSuccess;
  const int bs = 256;
  const unsigned nb = (unsigned)((a.nB + bs - 1) / bs);
  if (stage == 0)
    k_adj_band<R, 0><<<nb, bs, 0, s>>>(a);
  else if (stage == 1)
    k_adj_band<R, 1><<<nb, bs, 0, s>>>(a);
  else
    k_adj_band<R, 2><<<nb, bs, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_adj_grad_reduce(const int4* rec, const double* gcell, int64_t nB, int P, int nMat, double* grad,
                                   cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(grad, 0, (size_t)nMat * P * sizeof(double), s);
  if (e != cudaSuccess || nB <= 0) return e;
  const dim3 grid((unsigned)P, (unsigned)((nB + GRAD_CHUNK - 1) / GRAD_CHUNK));
  k_adj_grad_reduce<<<grid, 256, (size_t)nMat * sizeof(double), s>>>(rec, gcell, nB, P, nMat, grad);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_adj_receivers(R* lp, const int64_t* rcell, int nrec, const double* ir, int64_t cap,
                                 const double* target, int64_t tlen, int64_t n, int cotangent, cudaStream_t s) {
  k_adj_receivers<R><<<1, 32, 0, s>>>(lp, rcell, nrec, ir, cap, target, tlen, n, cotangent);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_adj_source(const R* lp, const int64_t* cell, int nsrc, const double* sval, double unit,
                              const R* u_s, int64_t n_us, int src_opt, const R* freq, R half_dt, double w, int64_t nn,
                              double* gsval, double* gwave, cudaStream_t s) {
  if (nsrc <= 0) return cudaSuccess;
  k_adj_source<R><<<(unsigned)((nsrc + 127) / 128), 128, 0, s>>>(lp, cell, nsrc, sval, unit, u_s, n_us, src_opt, freq,
                                                                 half_dt, w, nn, gsval, gwave);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_adj_pml_grad(const AdjPmlArgs<R>& a, int nsm, cudaStream_t s) {
  const int64_t ex = a.Nx - 2 * GHOST, ey = a.Ny - 2 * GHOST, ez = a.Nz - 2 * GHOST;
  const int64_t total = 2 * (int64_t)a.d * ((a.axis == 0) ? ey * ez : (a.axis == 1) ? ex * ez : ex * ey);
  if (total <= 0) return cudaSuccess;
  const int64_t nblk = std::min<int64_t>((total + 255) / 256, (int64_t)nsm * 8);
  k_adj_pml_grad<R><<<(unsigned)nblk, 256, (size_t)6 * a.d * sizeof(double), s>>>(a);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_clear_inactive(R* f, const uint8_t* cls, int64_t n, cudaStream_t s) {
  k_clear_inactive<R><<<592, 256, 0, s>>>(f, cls, n);
  return cudaGetLastError();
}

#define FZ_ADJ_INSTANTIATE(R)                                                                        \
  template size_t adj_stage_smem<R>(int);                                                            \
  template cudaError_t adj_stage_setup<R>(size_t);                                                   \
  template cudaError_t adj_stage_occupancy<R>(int*, size_t);                                         \
  template cudaError_t launch_adj_probe_scatter<R>(const AdjBandArgs<R>&, cudaStream_t);             \
  template cudaError_t launch_adj_stage<R>(const AdjStageArgs<R>&, dim3, cudaStream_t);              \
  template cudaError_t launch_adj_band<R>(int, const AdjBandArgs<R>&, cudaStream_t);                 \
  template cudaError_t launch_adj_receivers<R>(R*, const int64_t*, int, const double*, int64_t,      \
                                               const double*, int64_t, int64_t, int, cudaStream_t);  \
  template cudaError_t launch_adj_source<R>(const R*, const int64_t*, int, const double*, double,    \
                                            const R*, int64_t, int, const R*, R, double, int64_t,    \
                                            double*, double*, cudaStream_t);                         \
  template cudaError_t launch_adj_pml_grad<R>(const AdjPmlArgs<R>&, int, cudaStream_t);              \
  template cudaError_t launch_clear_inactive<R>(R*, const uint8_t*, int64_t, cudaStream_t);

FZ_ADJ_INSTANTIATE(float)
FZ_ADJ_INSTANTIATE(double)

}  // namespace fz
