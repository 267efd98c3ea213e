// fz_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// A CPU restatement, in FP64, of the FASES 3D time-domain solver update loop
// (vitorotri/fases v0.9). Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
// load this library. It follows, function by function:
//   - Godunov fluxes                     3D-solver/core/functions3D.cuh:56-78
//   - WENO-Z reconstruction              functions3D.cuh:763-1001 (tables main3D.cu:834-843,
//                                        eps = 1e-10 main3D.cu:770)
//   - SSP-RK3 stage kernels              functions3D.cuh:1086-1327
//   - CFS-cPML                           functions3D.cuh:661-756
//   - source injection                   functions3D.cuh:1039-1047
//   - trilinear probe, chi, ADE, BC      functions3D.cuh:263-271, 411-565
//   - boundary map                       common/filterABC.h:95-108
//   - time loop, buffer rotation and receiver sampling   3D-solver/core/main3D.cu:1280-1319,
//                                        1399-1414
//   - PCS / Ricker waveform and scaling  main3D.cu:963-1110
// The per-cell structure is deliberately the reference's (24 reconstructions per cell and stage,
// both faces of every cell evaluated from each side), so that it is an independent check of the
// face-once formulation the CUDA kernels use.
//
// Parity pin: the restatement is checked against outputs of the reference solver itself, built
// from its own sources for sm_100a (oracle/build_ref.sh) and run on a B200 on the scenes that
// tests/golden/make_golden.py writes; the resulting receiver traces are committed as fixtures
// under tests/golden/.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef double R;

inline size_t at3(int i, int j, int k, int Nx, int Ny) {
  return (size_t)i + (size_t)Nx * ((size_t)j + (size_t)k * Ny);
}

// ---- WENO-Z (Borges et al. 2008, q = 1) restated from functions3D.cuh:763-1001 ----
// Candidate-polynomial rows (main3D.cu:834-837), beta second-term rows (839-841), linear
// weights (843).
const R CRL[4][3] = {{11.0 / 6.0, -7.0 / 6.0, 1.0 / 3.0},
                     {1.0 / 3.0, 5.0 / 6.0, -1.0 / 6.0},
                     {-1.0 / 6.0, 5.0 / 6.0, 1.0 / 3.0},
                     {1.0 / 3.0, -7.0 / 6.0, 11.0 / 6.0}};
const R BRL[3][3] = {{3.0, -4.0, 1.0}, {1.0, 0.0, -1.0}, {1.0, -4.0, 3.0}};
const R DD[3] = {3.0 / 10.0, 3.0 / 5.0, 1.0 / 10.0};
const R WENO_EPS = 1e-10;

// One-sided value at a face of the cell whose value is q[0]; neighbours at q[m*s].
// side = 1: the value V- at the cell's upper face (reference idx = 1);
// side = 0: the value V+ at the cell's lower face (reference idx = 0).
inline R weno_face(const R* q, ptrdiff_t s, int side) {
  R cand[3], beta[3];
  for (int r = 0; r < 3; r++) {
    R v = 0.0, b2 = 0.0;
    for (int l = 0; l < 3; l++) {
      const R ql = q[(ptrdiff_t)(l - r) * s];
      v += CRL[r + side][l] * ql;
      b2 += BRL[r][l] * ql;
    }
    const R b1 = q[(ptrdiff_t)(-r) * s] - 2.0 * q[(ptrdiff_t)(1 - r) * s] +
                 q[(ptrdiff_t)(2 - r) * s];
    cand[r] = v;
    beta[r] = 13.0 * b1 * b1 / 12.0 + 0.25 * b2 * b2;
  }
  const R tau = std::fabs(beta[0] - beta[2]);
  R alpha[3], asum = 0.0;
  for (int r = 0; r < 3; r++) {
    const int di = side ? r : 2 - r;  // |2*SS - r| with SS = |idx - 1|
    alpha[r] = DD[di] * (1.0 + tau / (beta[r] + WENO_EPS));
    asum += alpha[r];
  }
  R out = 0.0;
  for (int r = 0; r < 3; r++) out += (alpha[r] / asum) * cand[r];
  return out;
}

// Godunov flux for linear acoustics (functions3D.cuh:56-78): pressure and normal velocity.
inline R flux_p(R pM, R pP, R uM, R uP, R rho, R c) {
  return 0.5 * (rho * c * c * (uP + uM) - c * (pP - pM));
}
inline R flux_u(R pM, R pP, R uM, R uP, R rho, R c) {
  return 0.5 * ((pP + pM) / rho - c * (uP - uM));
}

struct Fields {
  std::vector<R> p, u, v, w;
  void alloc(size_t n) {
    p.assign(n, 0.0); u.assign(n, 0.0); v.assign(n, 0.0); w.assign(n, 0.0);
  }
};

}  // namespace

extern "C" {

typedef struct orc_setup {
  int32_t Nx, Ny, Nz;
  double h, c, rho, dt;
  int32_t pml[6];  // U D R L F B
  int32_t pml_cells;
  double tol;  // absolute blending band (reference: 3h)
  const float* S;
  const uint8_t* oid;
  int32_t nMat, K, L;
  const double *Rinf, *A, *zeta, *B, *C, *alpha, *beta;
  int32_t nsrc;
  const int64_t* src_cell;  // flat indices
  const double* sval;
  int32_t src_opt;
  const double* src_freq;
  const double* u_s;
  int64_t n_us;
  int32_t nrec;
  const int64_t* rec_cell;
  int64_t max_steps;
  int32_t two_d;  // 1: one updated z-plane, no z fluxes (the 3D scheme restricted to 2D)
} orc_setup;

}  // extern "C"

namespace {

struct Oracle {
  orc_setup cfg;
  int Nx, Ny, Nz;
  size_t N;
  std::vector<float> S;
  std::vector<uint8_t> oid;
  std::vector<int32_t> bmap;
  int nB = 0;
  int K = 1, L = 1, nMat = 0;
  std::vector<R> Rinf, A, zeta, B, C, alpha, beta;
  std::vector<R> phi, phi_old, phi_nu, ps1, ps1_old, ps1_nu, ps2, ps2_old, ps2_nu;
  Fields U[3];
  int i0 = 0, i1 = 1, i2 = 2;  // U0, U1, U2 buffer ids (rotated by the swap)
  bool pml_on = false;
  std::vector<R> psi_px, psi_ux, psi_py, psi_vy, psi_pz, psi_wz;
  std::vector<int64_t> src_cell;
  std::vector<R> sval, src_freq, u_s;
  std::vector<int64_t> rec_cell;
  std::vector<R> ir, vel;
  int64_t n = 0;

  Fields& F(int id) { return U[id]; }

  // cPML: restated from functions3D.cuh:681-756.
  void cpml(Fields& out, size_t c, int i, int j, int k, R Lpx, R Lpy, R Lpz, R Lux, R Lvy, R Lwz,
            R ssp_w, bool advance) {
    const int d = cfg.pml_cells, ng = 3;
    const R lnR0 = std::log(1.0 / 1e-7), m = 2.0;
    const R kappa_max = 5.0, alpha_max = M_PI * 20.0, alpha_min = 0.1 * alpha_max;
    const R Uf = cfg.pml[0], Df = cfg.pml[1], Rf = cfg.pml[2], Lf = cfg.pml[3], Ff = cfg.pml[4],
            Bf = cfg.pml[5];
    auto cl = [](R x) { return std::min(1.0, std::max(0.0, x)); };
    const R xm = cl(((R)(ng + d) - i) / d), xp = cl((i - ((R)(Nx - 1 - ng) - d)) / d);
    const R ym = cl(((R)(ng + d) - j) / d), yp = cl((j - ((R)(Ny - 1 - ng) - d)) / d);
    const R zm = cl(((R)(ng + d) - k) / d), zp = cl((k - ((R)(Nz - 1 - ng) - d)) / d);
    const R pref = 0.5 * cfg.c * (m + 1.0) * lnR0 / ((R)d * cfg.h);
    const R sx = Lf * pref * std::pow(xm, m) + Rf * pref * std::pow(xp, m);
    const R sy = Bf * pref * std::pow(ym, m) + Ff * pref * std::pow(yp, m);
    const R sz = Df * pref * std::pow(zm, m) + Uf * pref * std::pow(zp, m);
    const R dx = Lf * xm + Rf * xp, dy = Bf * ym + Ff * yp, dz = Df * zm + Uf * zp;
    const R kapx = 1.0 + (kappa_max - 1.0) * std::pow(dx, m);
    const R kapy = 1.0 + (kappa_max - 1.0) * std::pow(dy, m);
    const R kapz = 1.0 + (kappa_max - 1.0) * std::pow(dz, m);
    const R ax = alpha_min + (alpha_max - alpha_min) * (1.0 - dx);
    const R ay = alpha_min + (alpha_max - alpha_min) * (1.0 - dy);
    const R az = alpha_min + (alpha_max - alpha_min) * (1.0 - dz);
    const bool bx = (Lf > 0 && i >= ng && i < ng + d) || (Rf > 0 && i >= Nx - ng - d && i <= Nx - 1 - ng);
    const bool by = (Bf > 0 && j >= ng && j < ng + d) || (Ff > 0 && j >= Ny - ng - d && j <= Ny - 1 - ng);
    const bool bz = (Df > 0 && k >= ng && k < ng + d) || (Uf > 0 && k >= Nz - ng - d && k <= Nz - 1 - ng);
    const R wdt = ssp_w * cfg.dt;
    auto corr = [](R D, R kap, R psi) { return (1.0 / kap - 1.0) * D + psi; };
    auto adv = [&](R D, R kap, R sig, R alp, R& psi) {
      const R b = std::exp(-(alp + sig / kap) * cfg.dt);
      const R ca = (sig > 0.0) ? (sig / (kap * (sig + kap * alp))) * (b - 1.0) : 0.0;
      psi = b * psi + ca * D;
    };
    if (bx) {
      const int ix = (i < ng + d) ? (i - ng) : (i - (Nx - ng - d) + d);
      const size_t X = (size_t)ix + (size_t)(2 * d) * ((size_t)j + (size_t)Ny * k);
      out.p[c] += wdt * corr(Lpx, kapx, psi_px[X]);
      out.u[c] += wdt * corr(Lux, kapx, psi_ux[X]);
      if (advance) { adv(Lpx, kapx, sx, ax, psi_px[X]); adv(Lux, kapx, sx, ax, psi_ux[X]); }
    }
    if (by) {
      const int jy = (j < ng + d) ? (j - ng) : (j - (Ny - ng - d) + d);
      const size_t Y = (size_t)i + (size_t)Nx * ((size_t)jy + (size_t)(2 * d) * k);
      out.p[c] += wdt * corr(Lpy, kapy, psi_py[Y]);
      out.v[c] += wdt * corr(Lvy, kapy, psi_vy[Y]);
      if (advance) { adv(Lpy, kapy, sy, ay, psi_py[Y]); adv(Lvy, kapy, sy, ay, psi_vy[Y]); }
    }
    if (bz) {
      const int kt = (k < ng + d) ? (k - ng) : (k - (Nz - ng - d) + d);
      const size_t Z = (size_t)i + (size_t)Nx * ((size_t)j + (size_t)Ny * kt);
      out.p[c] += wdt * corr(Lpz, kapz, psi_pz[Z]);
      out.w[c] += wdt * corr(Lwz, kapz, psi_wz[Z]);
      if (advance) { adv(Lpz, kapz, sz, az, psi_pz[Z]); adv(Lwz, kapz, sz, az, psi_wz[Z]); }
    }
  }

  // One SSP-RK3 stage (functions3D.cuh:1086-1327). in = stage input, base = U0, out = output.
  void stage(int st, const Fields& in, const Fields& base, Fields& out) {
    const R rho = cfg.rho, c = cfg.c, h = cfg.h, dt = cfg.dt;
    const ptrdiff_t sx = 1, sy = Nx, sz = (ptrdiff_t)Nx * Ny;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 3; k < Nz - 3; k++)
      for (int j = 3; j < Ny - 3; j++)
        for (int i = 3; i < Nx - 3; i++) {
          const size_t ci = at3(i, j, k, Nx, Ny);
          if (S[ci] < (float)cfg.h) continue;  // functions3D.cuh:1097
          R fl[3][4];  // per axis: Fp+, Fp-, Fvel+, Fvel-
          const R* vel[3] = {in.u.data(), in.v.data(), in.w.data()};
          const ptrdiff_t st3[3] = {sx, sy, sz};
          for (int a = 0; a < 3; a++) {
            if (a == 2 && cfg.two_d) {
              fl[2][0] = fl[2][1] = fl[2][2] = fl[2][3] = 0.0;
              continue;
            }
            const R* pp = in.p.data() + ci;
            const R* qq = vel[a] + ci;
            const ptrdiff_t s = st3[a];
            // compute_Vs_*: [V-(i+1/2), V+(i+1/2) from i+1, V-(i-1/2) from i-1, V+(i-1/2)]
            const R pV0 = weno_face(pp, s, 1), pV1 = weno_face(pp + s, s, 0);
            const R pV2 = weno_face(pp - s, s, 1), pV3 = weno_face(pp, s, 0);
            const R qV0 = weno_face(qq, s, 1), qV1 = weno_face(qq + s, s, 0);
            const R qV2 = weno_face(qq - s, s, 1), qV3 = weno_face(qq, s, 0);
            fl[a][0] = flux_p(pV0, pV1, qV0, qV1, rho, c);
            fl[a][1] = flux_p(pV2, pV3, qV2, qV3, rho, c);
            fl[a][2] = flux_u(pV0, pV1, qV0, qV1, rho, c);
            fl[a][3] = flux_u(pV2, pV3, qV2, qV3, rho, c);
          }
          const R Lu = (-fl[0][2] + fl[0][3]) / h, Lv = (-fl[1][2] + fl[1][3]) / h,
                  Lw = (-fl[2][2] + fl[2][3]) / h;
          const R Lpx = (-fl[0][0] + fl[0][1]) / h, Lpy = (-fl[1][0] + fl[1][1]) / h,
                  Lpz = (-fl[2][0] + fl[2][1]) / h;
          const R Lp = (-fl[0][0] + fl[0][1] - fl[1][0] + fl[1][1] - fl[2][0] + fl[2][1]) / h;
          R ssp_w;
          if (st == 0) {
            out.u[ci] = in.u[ci] + dt * Lu; out.v[ci] = in.v[ci] + dt * Lv;
            out.w[ci] = in.w[ci] + dt * Lw; out.p[ci] = in.p[ci] + dt * Lp;
            ssp_w = 1.0;
          } else if (st == 1) {
            out.u[ci] = 0.75 * base.u[ci] + 0.25 * (in.u[ci] + dt * Lu);
            out.v[ci] = 0.75 * base.v[ci] + 0.25 * (in.v[ci] + dt * Lv);
            out.w[ci] = 0.75 * base.w[ci] + 0.25 * (in.w[ci] + dt * Lw);
            out.p[ci] = 0.75 * base.p[ci] + 0.25 * (in.p[ci] + dt * Lp);
            ssp_w = 0.25;
          } else {
            out.u[ci] = (base.u[ci] + 2.0 * (in.u[ci] + dt * Lu)) / 3.0;
            out.v[ci] = (base.v[ci] + 2.0 * (in.v[ci] + dt * Lv)) / 3.0;
            out.w[ci] = (base.w[ci] + 2.0 * (in.w[ci] + dt * Lw)) / 3.0;
            out.p[ci] = (base.p[ci] + 2.0 * (in.p[ci] + dt * Lp)) / 3.0;
            ssp_w = 2.0 / 3.0;
          }
          if (pml_on) cpml(out, ci, i, j, k, Lpx, Lpy, Lpz, Lu, Lv, Lw, ssp_w, st == 2);
        }
  }

  // kernel_inject_src_SSP (functions3D.cuh:1039-1047).
  void inject(Fields& out, R w, int64_t nn) {
    const R As = 6.0 * cfg.h * cfg.h;
    for (size_t s = 0; s < src_cell.size(); s++) {
      R amp;
      if (cfg.src_opt == 2)
        amp = std::sin(2.0 * M_PI * src_freq[s] * (R)nn * (0.5 * cfg.dt));
      else
        amp = (nn < (int64_t)u_s.size()) ? u_s[nn] : 0.0;
      out.p[src_cell[s]] += w * cfg.dt * cfg.c * cfg.c * sval[s] * amp * cfg.rho * As /
                            (cfg.h * cfg.h * cfg.h);
    }
  }

  // trilinear_interp (functions3D.cuh:411-422).
  R trilin(const std::vector<R>& f, R Dx, R Dy, R Dz) const {
    const R h = cfg.h;
    const R gx = Dx / h - 0.5, gy = Dy / h - 0.5, gz = Dz / h - 0.5;
    int i = (int)std::floor(gx), j = (int)std::floor(gy), k = (int)std::floor(gz);
    i = std::max(0, std::min(i, Nx - 2));
    j = std::max(0, std::min(j, Ny - 2));
    k = std::max(0, std::min(k, Nz - 2));
    const R sx = gx - i, sy = gy - j, sz = gz - k;
    auto F3 = [&](int a, int b, int cc) { return f[at3(a, b, cc, Nx, Ny)]; };
    const R c00 = F3(i, j, k) * (1 - sx) + F3(i + 1, j, k) * sx;
    const R c10 = F3(i, j + 1, k) * (1 - sx) + F3(i + 1, j + 1, k) * sx;
    const R c01 = F3(i, j, k + 1) * (1 - sx) + F3(i + 1, j, k + 1) * sx;
    const R c11 = F3(i, j + 1, k + 1) * (1 - sx) + F3(i + 1, j + 1, k + 1) * sx;
    const R c0 = c00 * (1 - sy) + c10 * sy, c1 = c01 * (1 - sy) + c11 * sy;
    return c0 * (1 - sz) + c1 * sz;
  }

  // kernel_apply_BC_immersed_sdf + ADE_solver (functions3D.cuh:426-565).
  void bc(Fields& out, const Fields& old, R a_ssp, R b_ssp, R c_ssp, std::vector<R>& phL,
          const std::vector<R>& phM, const std::vector<R>& phR, std::vector<R>& p1L,
          const std::vector<R>& p1M, const std::vector<R>& p1R, std::vector<R>& p2L,
          const std::vector<R>& p2M, const std::vector<R>& p2R) {
    const R h = cfg.h, rho = cfg.rho, c = cfg.c, dt = cfg.dt, tol = cfg.tol;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 3; k < Nz - 3; k++)
      for (int j = 3; j < Ny - 3; j++)
        for (int i = 3; i < Nx - 3; i++) {
          const size_t ci = at3(i, j, k, Nx, Ny);
          const uint8_t o = oid[ci];
          const int b = bmap[ci];
          if (o == 0 || o == 0xFF || b < 0) continue;
          const R s = S[ci];
          const R gx = ((R)S[at3(i + 1, j, k, Nx, Ny)] - (R)S[at3(i - 1, j, k, Nx, Ny)]) * (0.5 / h);
          const R gy = ((R)S[at3(i, j + 1, k, Nx, Ny)] - (R)S[at3(i, j - 1, k, Nx, Ny)]) * (0.5 / h);
          const R gz = ((R)S[at3(i, j, k + 1, Nx, Ny)] - (R)S[at3(i, j, k - 1, Nx, Ny)]) * (0.5 / h);
          const R gn = std::max(std::sqrt(gx * gx + gy * gy + gz * gz), 1e-12);
          const R nx = -gx / gn, ny = -gy / gn, nz = -gz / gn;
          const R Cx = (i + 0.5) * h, Cy = (j + 0.5) * h, Cz = (k + 0.5) * h;
          const R Wx = Cx + s * nx, Wy = Cy + s * ny, Wz = Cz + s * nz;
          const R l = s + 2.0 * h;
          const R Dx = Wx - l * nx, Dy = Wy - l * ny, Dz = Wz - l * nz;
          const R pD = trilin(old.p, Dx, Dy, Dz), uD = trilin(old.u, Dx, Dy, Dz),
                  vD = trilin(old.v, Dx, Dy, Dz), wD = trilin(old.w, Dx, Dy, Dz);
          const R un = uD * nx + vD * ny + wD * nz;
          const R utx = uD - un * nx, uty = vD - un * ny, utz = wD - un * nz;
          const R Z0 = rho * c;
          const R wout = pD + Z0 * un;
          const int m = o - 1;
          // ADE_solver: SSP-RK3 stage on the pole states.
          R sumA = 0.0, sumBC = 0.0;
          for (int q = 0; q < K; q++) {
            const int mi = m * K + q, si = b * K + q;
            const R Lphi = wout - zeta[mi] * phR[si];
            phL[si] = (a_ssp * phM[si] + b_ssp * (phR[si] + dt * Lphi)) / c_ssp;
            sumA += A[mi] * phL[si];
          }
          for (int q = 0; q < L; q++) {
            const int mi = m * L + q, si = b * L + q;
            const R L1 = wout - (alpha[mi] * p1R[si] + beta[mi] * p2R[si]);
            const R L2 = beta[mi] * p1R[si] - alpha[mi] * p2R[si];
            const R n1 = (a_ssp * p1M[si] + b_ssp * (p1R[si] + dt * L1)) / c_ssp;
            const R n2 = (a_ssp * p2M[si] + b_ssp * (p2R[si] + dt * L2)) / c_ssp;
            p1L[si] = n1;
            p2L[si] = n2;
            sumBC += B[mi] * n1 + C[mi] * n2;
          }
          const R win = Rinf[m] * wout + sumA + sumBC;
          const R pb = 0.5 * (win + wout), unb = (wout - win) / (2.0 * Z0);
          const R ub = unb * nx + utx, vb = unb * ny + uty, wb = unb * nz + utz;
          // chi_layered (functions3D.cuh:263-271)
          R chi;
          if (s >= tol) chi = 0.0;
          else if (s <= h) chi = 1.0;
          else {
            const R r = (s - h) / (tol - h);
            chi = 1.0 - r * r * (3.0 - 2.0 * r);
          }
          out.u[ci] = (1.0 - chi) * out.u[ci] + chi * ub;
          out.v[ci] = (1.0 - chi) * out.v[ci] + chi * vb;
          out.w[ci] = (1.0 - chi) * out.w[ci] + chi * wb;
          out.p[ci] = (1.0 - chi) * out.p[ci] + chi * pb;
        }
  }

  void sample() {
    const Fields& u0 = U[i0];
    const int64_t cap = cfg.max_steps;
    if (n >= cap) return;
    for (size_t r = 0; r < rec_cell.size(); r++) {
      const int64_t c = rec_cell[r];
      ir[r * cap + n] = u0.p[c];
      vel[(r * cap + n) * 3 + 0] = u0.u[c];
      vel[(r * cap + n) * 3 + 1] = u0.v[c];
      vel[(r * cap + n) * 3 + 2] = u0.w[c];
    }
  }

  // One time step: main3D.cu:1280-1319 then the receiver sampling 1399-1414.
  void step() {
    Fields& A0 = U[i0];
    Fields& A1 = U[i1];
    Fields& A2 = U[i2];
    stage(0, A0, A0, A1);
    inject(A1, 1.0, 2 * n);
    bc(A1, A0, 0.0, 1.0, 1.0, phi, phi_old, phi_old, ps1, ps1_old, ps1_old, ps2, ps2_old, ps2_old);
    stage(1, A1, A0, A2);
    inject(A2, 0.25, 2 * n + 2);
    bc(A2, A1, 3.0, 1.0, 4.0, phi_nu, phi_old, phi, ps1_nu, ps1_old, ps1, ps2_nu, ps2_old, ps2);
    stage(2, A2, A0, A1);
    inject(A1, 2.0 / 3.0, 2 * n + 1);
    bc(A1, A2, 1.0, 2.0, 3.0, phi, phi_old, phi_nu, ps1, ps1_old, ps1_nu, ps2, ps2_old, ps2_nu);
    std::swap(i0, i1);
    std::swap(phi_old, phi);
    std::swap(ps1_old, ps1);
    std::swap(ps2_old, ps2);
    sample();
    n += 1;
  }
};

}  // namespace

extern "C" {

void* orc_create(const orc_setup* s) {
  if (!s || s->Nx < 7 || s->Ny < 7 || s->Nz < 7 || !s->S || !s->oid) return nullptr;
  Oracle* o = new Oracle();
  o->cfg = *s;
  o->Nx = s->Nx; o->Ny = s->Ny; o->Nz = s->Nz;
  o->N = (size_t)s->Nx * s->Ny * s->Nz;
  o->S.assign(s->S, s->S + o->N);
  o->oid.assign(s->oid, s->oid + o->N);
  // build_boundary_map (common/filterABC.h:95-108)
  o->bmap.assign(o->N, -1);
  for (size_t c = 0; c < o->N; c++)
    if (o->oid[c] != 0xFF && o->oid[c] != 0) o->bmap[c] = o->nB++;
  o->nMat = s->nMat;
  o->K = std::max(1, s->K);  // main3D.cu:602-603
  o->L = std::max(1, s->L);
  const int nm = std::max(1, s->nMat);
  o->Rinf.assign(nm, 0.0);
  o->A.assign((size_t)nm * o->K, 0.0); o->zeta.assign((size_t)nm * o->K, 0.0);
  o->B.assign((size_t)nm * o->L, 0.0); o->C.assign((size_t)nm * o->L, 0.0);
  o->alpha.assign((size_t)nm * o->L, 0.0); o->beta.assign((size_t)nm * o->L, 0.0);
  for (int m = 0; m < s->nMat; m++) {
    if (s->Rinf) o->Rinf[m] = s->Rinf[m];
    for (int q = 0; q < s->K; q++) {
      if (s->A) o->A[(size_t)m * o->K + q] = s->A[(size_t)m * s->K + q];
      if (s->zeta) o->zeta[(size_t)m * o->K + q] = s->zeta[(size_t)m * s->K + q];
    }
    for (int q = 0; q < s->L; q++) {
      const size_t dst = (size_t)m * o->L + q, src = (size_t)m * s->L + q;
      if (s->B) o->B[dst] = s->B[src];
      if (s->C) o->C[dst] = s->C[src];
      if (s->alpha) o->alpha[dst] = s->alpha[src];
      if (s->beta) o->beta[dst] = s->beta[src];
    }
  }
  const size_t nk = (size_t)o->nB * o->K, nl = (size_t)o->nB * o->L;
  for (auto* v : {&o->phi, &o->phi_old, &o->phi_nu}) v->assign(nk, 0.0);
  for (auto* v : {&o->ps1, &o->ps1_old, &o->ps1_nu, &o->ps2, &o->ps2_old, &o->ps2_nu})
    v->assign(nl, 0.0);
  for (auto& f : o->U) f.alloc(o->N);
  o->pml_on = false;
  for (int f = 0; f < 6; f++) o->pml_on = o->pml_on || (s->pml[f] != 0);
  if (o->pml_on) {
    const size_t d2 = 2 * (size_t)s->pml_cells;
    const size_t nx_ = d2 * s->Ny * s->Nz, ny_ = (size_t)s->Nx * d2 * s->Nz,
                 nz_ = (size_t)s->Nx * s->Ny * d2;
    o->psi_px.assign(nx_, 0.0); o->psi_ux.assign(nx_, 0.0);
    o->psi_py.assign(ny_, 0.0); o->psi_vy.assign(ny_, 0.0);
    o->psi_pz.assign(nz_, 0.0); o->psi_wz.assign(nz_, 0.0);
  }
  for (int q = 0; q < s->nsrc; q++) {
    o->src_cell.push_back(s->src_cell[q]);
    o->sval.push_back(s->sval[q]);
    o->src_freq.push_back(s->src_freq ? s->src_freq[q] : 0.0);
  }
  if (s->u_s && s->n_us > 0) o->u_s.assign(s->u_s, s->u_s + s->n_us);
  for (int q = 0; q < s->nrec; q++) o->rec_cell.push_back(s->rec_cell[q]);
  o->ir.assign((size_t)s->nrec * std::max<int64_t>(s->max_steps, 1), 0.0);
  o->vel.assign((size_t)s->nrec * std::max<int64_t>(s->max_steps, 1) * 3, 0.0);
  return o;
}

int orc_set_fields(void* h, const double* p, const double* u, const double* v, const double* w) {
  Oracle* o = (Oracle*)h;
  if (!o) return -1;
  Fields& f = o->U[o->i0];
  if (p) std::copy(p, p + o->N, f.p.begin());
  if (u) std::copy(u, u + o->N, f.u.begin());
  if (v) std::copy(v, v + o->N, f.v.begin());
  if (w) std::copy(w, w + o->N, f.w.begin());
  return 0;
}

int orc_run(void* h, int64_t nsteps, int32_t nthreads) {
  Oracle* o = (Oracle*)h;
  if (!o) return -1;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  for (int64_t s = 0; s < nsteps; s++) o->step();
  return 0;
}

int orc_get_ir(void* h, double* ir, double* vel) {
  Oracle* o = (Oracle*)h;
  if (!o) return -1;
  if (ir) std::copy(o->ir.begin(), o->ir.end(), ir);
  if (vel) std::copy(o->vel.begin(), o->vel.end(), vel);
  return 0;
}

int orc_get_fields(void* h, double* p, double* u, double* v, double* w) {
  Oracle* o = (Oracle*)h;
  if (!o) return -1;
  const Fields& f = o->U[o->i0];
  if (p) std::copy(f.p.begin(), f.p.end(), p);
  if (u) std::copy(f.u.begin(), f.u.end(), u);
  if (v) std::copy(f.v.begin(), f.v.end(), v);
  if (w) std::copy(f.w.begin(), f.w.end(), w);
  return 0;
}

// Energy (functions3D.cuh:111-129), in FP64.
double orc_energy(void* h) {
  Oracle* o = (Oracle*)h;
  const Fields& f = o->U[o->i0];
  const R rc2 = o->cfg.rho * o->cfg.c * o->cfg.c;
  R s = 0.0;
  for (size_t c = 0; c < o->N; c++)
    s += f.p[c] * f.p[c] / rc2 + o->cfg.rho * (f.u[c] * f.u[c] + f.v[c] * f.v[c] + f.w[c] * f.w[c]);
  return 0.5 * s;
}

int64_t orc_n_band(void* h) { return ((Oracle*)h)->nB; }

void orc_destroy(void* h) { delete (Oracle*)h; }

// Scalar ADE recursion of ADE_solver (functions3D.cuh:426-459) for one band cell of one material,
// driven by w(t) sampled the way the time loop samples it: stage 0 at t_n, stage 1 at t_n + dt,
// stage 2 at t_n + dt/2. w_in[3*n + s] holds the input of stage s of step n; out[3*n + s] the
// returned w_in of that stage. Used by the known-answer test against the closed-form discrete
// response of the recursion.
int orc_ade_drive(int32_t K, int32_t L, double Rinf, const double* A, const double* zeta,
                  const double* B, const double* C, const double* alpha, const double* beta,
                  double dt, int64_t nsteps, const double* w_in, double* out) {
  const int Kc = std::max(1, K), Lc = std::max(1, L);
  std::vector<R> ph(Kc, 0.0), ph_old(Kc, 0.0), ph_nu(Kc, 0.0);
  std::vector<R> a1(Lc, 0.0), a1_old(Lc, 0.0), a1_nu(Lc, 0.0);
  std::vector<R> a2(Lc, 0.0), a2_old(Lc, 0.0), a2_nu(Lc, 0.0);
  auto run = [&](R w, R a, R b, R c, std::vector<R>& pL, const std::vector<R>& pM,
                 const std::vector<R>& pR, std::vector<R>& qL, const std::vector<R>& qM,
                 const std::vector<R>& qR, std::vector<R>& rL, const std::vector<R>& rM,
                 const std::vector<R>& rR) {
    R sA = 0.0, sBC = 0.0;
    for (int q = 0; q < K; q++) {
      const R Lp = w - zeta[q] * pR[q];
      pL[q] = (a * pM[q] + b * (pR[q] + dt * Lp)) / c;
      sA += A[q] * pL[q];
    }
    for (int q = 0; q < L; q++) {
      const R L1 = w - (alpha[q] * qR[q] + beta[q] * rR[q]);
      const R L2 = beta[q] * qR[q] - alpha[q] * rR[q];
      const R n1 = (a * qM[q] + b * (qR[q] + dt * L1)) / c;
      const R n2 = (a * rM[q] + b * (rR[q] + dt * L2)) / c;
      qL[q] = n1; rL[q] = n2;
      sBC += B[q] * n1 + C[q] * n2;
    }
    return Rinf * w + sA + sBC;
  };
  for (int64_t n = 0; n < nsteps; n++) {
    out[3 * n + 0] = run(w_in[3 * n + 0], 0, 1, 1, ph, ph_old, ph_old, a1, a1_old, a1_old, a2, a2_old, a2_old);
    out[3 * n + 1] = run(w_in[3 * n + 1], 3, 1, 4, ph_nu, ph_old, ph, a1_nu, a1_old, a1, a2_nu, a2_old, a2);
    out[3 * n + 2] = run(w_in[3 * n + 2], 1, 2, 3, ph, ph_old, ph_nu, a1, a1_old, a1_nu, a2, a2_old, a2_nu);
    std::swap(ph_old, ph); std::swap(a1_old, a1); std::swap(a2_old, a2);
  }
  return 0;
}

// Source waveform and scaling, restated from main3D.cu:963-1110.
// src_opt 0: PCS (Sheaffer, van Walstijn & Fazenda 2012): Gaussian force through the bilinear-
// transformed mass-spring-damper; 1: Ricker antiderivative. u_s and p_ref have 2*Nt+1 entries.
int orc_waveform(int32_t src_opt, double glob_f, double f_cutoff, double dt, int64_t Nt, double h,
                 double rho, double* u_s, double* p_ref, double* p_peak) {
  const int64_t n = 2 * Nt + 1;
  std::vector<R> us(n, 0.0);
  const R dth = 0.5 * dt;
  if (src_opt == 0) {
    const R Q = 1.0, f0 = glob_f, w0 = 2.0 * M_PI * f0;
    const R bs = w0 / std::tan(0.5 * w0 * dth);
    const R M = 0.025, Rs = w0 * M / Q, Ks = M * w0 * w0;
    const R den = M * bs * bs + Rs * bs + Ks;
    const R b0 = bs / den, b2 = -b0;
    const R a1 = 2.0 * (Ks - M * bs * bs) / den, a2 = 1.0 - 2.0 * Rs * bs / den;
    const R sig = 0.425 / f_cutoff;
    const int ts = (int)std::ceil(8.5 * sig / dth);
    std::vector<R> Fs(n, 0.0);
    for (int64_t t = 0; t < n; t++) {
      const R td = (t - ts) * dth;
      Fs[t] = std::exp(-td * td / (2.0 * sig * sig));
    }
    for (int64_t t = 2; t < n; t++) us[t] = b0 * Fs[t] + b2 * Fs[t - 2] - a1 * us[t - 1] - a2 * us[t - 2];
  } else if (src_opt == 1) {
    const R sig = 1.0 / (std::sqrt(2.0) * M_PI * glob_f);
    const R ts = (int)std::ceil(5.0 * sig / dth);
    for (int64_t t = 0; t < n; t++) {
      const R x = (t - ts) * dth / sig;
      us[t] = x * std::exp(-0.5 * x * x);
    }
  }
  const R As = 6.0 * h * h;
  R peak = 0.0;
  std::vector<R> pr(n, 0.0);
  for (int64_t t = 1; t < n - 1; t++) {
    const R dq = As * (us[t + 1] - us[t - 1]) / (2.0 * dth);
    pr[t] = rho * dq / (4.0 * M_PI);
    peak = std::max(peak, std::fabs(pr[t]));
  }
  if (u_s) std::copy(us.begin(), us.end(), u_s);
  if (p_ref) std::copy(pr.begin(), pr.end(), p_ref);
  if (p_peak) *p_peak = peak;
  return 0;
}

}  // extern "C"
