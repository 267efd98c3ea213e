// fz_legacy2d_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// A CPU restatement of the reference's 2D legacy solver (vitorotri/fases v0.9, `2D-solver/`),
// in FP64 or, to follow the reference's own float arithmetic, in FP32. It keeps the reference's
// structure: three separate passes per stage (stage update with the PML, ghost-row copy,
// immersed boundary), three field buffers with U0 <- U1 copied after each step, three ADE state
// sets with the old <- current copy. It follows:
//   - Godunov fluxes                       2D-solver/core/functions.cuh:199-213
//   - WENO5-JS reconstruction              functions.cuh:1029-1180 (tables main.cu:638-651,
//                                          eps main.cu:591)
//   - SSP-RK3 stage kernels                functions.cuh:1182-1390
//   - sPML                                 functions.cuh:936-965
//   - ghost rows of p and v (periodic_BC)  functions.cuh:268-298
//   - bicubic probe, chi, ADE, boundary    functions.cuh:421-478, 534-543, 635-740
//   - boundary map                         common/filterABC.h:95-108
//   - time loop, copies, receiver          2D-solver/core/main.cu:795-858
// The reference's ghost-row copy races with the interior writes of the same launch; this
// restatement copies after the whole stage update (the outcome when the copying threads run
// last), from columns that hold at least one cell with S >= h.
//
// The node loops run on OpenMP threads; every node writes only its own outputs and ADE states,
// so the results do not depend on the thread count.
//
// Parity pin: checked against receiver traces of the reference's own 2D solver, built from its
// sources (oracle/build_ref.sh) and run on a B200 by tests/golden/make_golden_legacy2d.py.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

template <class T>
struct Legacy2D {
  int Nx, Ny;
  T h, dt, rho, c, eps, tol;
  T keyN, keyS, keyE, keyW;
  const float* S;
  const uint8_t* oid;
  int K, L;
  std::vector<T> Rinf, A, zeta, B, C, alpha, beta;
  std::vector<T> p[3], u[3], v[3];
  std::vector<T> phi, phi_old, phi_nu, ps1, ps1_old, ps1_nu, ps2, ps2_old, ps2_nu;
  std::vector<int> bmap;
  std::vector<uint8_t> colfluid;

  size_t at(int i, int j) const { return (size_t)j * Nx + i; }

  // the candidate/smoothness tables and d_r of main.cu:638-651
  static T crl(int row, int l) {
    static const double t[4][3] = {{11.0 / 6.0, -7.0 / 6.0, 1.0 / 3.0},
                                   {1.0 / 3.0, 5.0 / 6.0, -1.0 / 6.0},
                                   {-1.0 / 6.0, 5.0 / 6.0, 1.0 / 3.0},
                                   {1.0 / 3.0, -7.0 / 6.0, 11.0 / 6.0}};
    return (T)t[row][l];
  }
  static T brl(int r, int l) {
    static const double t[3][3] = {{3, -4, 1}, {1, 0, -1}, {1, -4, 3}};
    return (T)t[r][l];
  }
  static T dd(int r) {
    static const double t[3] = {3.0 / 10.0, 3.0 / 5.0, 1.0 / 10.0};
    return (T)t[r];
  }

  // functions.cuh:1115-1123: the smoothness indicator, evaluated in double and rounded to T
  static T beta_r(T q0, T q1, T q2, int r) {
    const T b1 = q0 - (T)2 * q1 + q2;
    const T b2 = brl(r, 0) * q0 + brl(r, 1) * q1 + brl(r, 2) * q2;
    return (T)((13.0 * (double)b1 * (double)b1 / 12.0) + (0.25 * (double)b2 * (double)b2));
  }

  // WENO_x / WENO_y (functions.cuh:1125-1162): the value at the face i+1/2 (idx 1) or i-1/2
  // (idx 0) of node i of the line f (stride st)
  T weno(const T* f, size_t i, ptrdiff_t st, int idx) const {
    T V[3], bt[3], al[3];
    for (int r = 0; r < 3; r++) {
      T acc = 0;
      for (int l = 0; l < 3; l++) acc += crl(r + idx, l) * f[(ptrdiff_t)i + (l - r) * st];
      V[r] = acc;
      bt[r] = beta_r(f[(ptrdiff_t)i - r * st], f[(ptrdiff_t)i + (1 - r) * st], f[(ptrdiff_t)i + (2 - r) * st], r);
    }
    const int S = idx == 1 ? 0 : 1;
    for (int r = 0; r < 3; r++) {
      const T aux = bt[r] + eps;
      const int rr = S * 3 - S * 1 - r;
      al[r] = dd(rr < 0 ? -rr : rr) / (aux * aux);
    }
    T out = 0;
    for (int r = 0; r < 3; r++) {
      const T sum = al[0] + al[1] + al[2];
      out += (al[r] / sum) * V[r];
    }
    return out;
  }

  // compute_Vs_x / compute_Vs_y (functions.cuh:1164-1176)
  void vs(T* Q, const T* f, size_t i, ptrdiff_t st) const {
    Q[0] = weno(f, i, st, 1);
    Q[1] = weno(f, i + st, st, 0);
    Q[2] = weno(f, i - st, st, 1);
    Q[3] = weno(f, i, st, 0);
  }

  T Fp(T pM, T pP, T uM, T uP) const { return (T)(0.5 * (double)(rho * c * c * (uP + uM) - c * (pP - pM))); }
  T Fu(T pM, T pP, T uM, T uP) const { return (T)(0.5 * (double)((pP + pM) / rho - c * (uP - uM))); }
  T Gv(T pM, T pP, T vM, T vP) const { return (T)(0.5 * (double)((pM + pP) / rho - c * (vP - vM))); }

  // sPML (functions.cuh:941-965); the ramp half-width is computed in float as there
  T spml_s(int i, int j) const {
    const int max_idx = (int)(0.15f * (float)(Nx < Ny ? Nx : Ny));
    const T half = (T)max_idx;
    const T one = 1, zero = 0;
    const T rx = keyE * std::max(zero, std::min((T)(i - (Nx - half)) / half, one));
    const T lx = keyW * std::max(zero, std::min((half - i) / half, one));
    const T ly = keyS * std::max(zero, std::min((half - j) / half, one));
    const T uy = keyN * std::max(zero, std::min((j - (Ny - half)) / half, one));
    const T rx3 = rx * rx * rx, lx3 = lx * lx * lx, ly3 = ly * ly * ly, uy3 = uy * uy * uy;
    const T smax = (T)0.018f;
    const T sx = smax * (rx3 + lx3);
    const T sy = smax * (uy3 + ly3);
    T s = sx + sy - sx * sy;
    return std::min(s, (T)0.999f);
  }

  void stage(int st) {
    // inputs and outputs of kernel_WENO_step0/1/2
    const int in = st == 0 ? 0 : (st == 1 ? 1 : 2);
    const int out = st == 1 ? 2 : 1;
    const T* P = p[in].data();
    const T* U = u[in].data();
    const T* V = v[in].data();
    const float hf = (float)h;
#pragma omp parallel for schedule(static)
    for (int j = 3; j < Ny - 3; j++)
      for (int i = 3; i < Nx - 3; i++) {
        const size_t C = at(i, j);
        if (S[C] < hf) continue;
        T pv[4], uv[4], vv[4];
        vs(pv, P, C, 1);
        vs(uv, U, C, 1);
        const T FpP = Fp(pv[0], pv[1], uv[0], uv[1]), FpM = Fp(pv[2], pv[3], uv[2], uv[3]);
        const T FuP = Fu(pv[0], pv[1], uv[0], uv[1]), FuM = Fu(pv[2], pv[3], uv[2], uv[3]);
        vs(pv, P, C, Nx);
        vs(vv, V, C, Nx);
        const T GpP = Fp(pv[0], pv[1], vv[0], vv[1]), GpM = Fp(pv[2], pv[3], vv[2], vv[3]);
        const T GvP = Gv(pv[0], pv[1], vv[0], vv[1]), GvM = Gv(pv[2], pv[3], vv[2], vv[3]);
        const T ru = dt * ((-FuP + FuM) / h);
        const T rv = dt * ((-GvP + GvM) / h);
        const T rp = dt * ((-FpP + FpM - GpP + GpM) / h);
        T nu, nv, np;
        if (st == 0) {
          nu = u[0][C] + ru;
          nv = v[0][C] + rv;
          np = p[0][C] + rp;
        } else if (st == 1) {
          nu = (T)0.75f * u[0][C] + (T)0.25f * (u[1][C] + ru);
          nv = (T)0.75f * v[0][C] + (T)0.25f * (v[1][C] + rv);
          np = (T)0.75f * p[0][C] + (T)0.25f * (p[1][C] + rp);
        } else {
          nu = (u[0][C] + (T)2 * (u[2][C] + ru)) / (T)3;
          nv = (v[0][C] + (T)2 * (v[2][C] + rv)) / (T)3;
          np = (p[0][C] + (T)2 * (p[2][C] + rp)) / (T)3;
        }
        const T s = spml_s(i, j);
        nu -= s * nu;
        nv -= s * nv;
        np -= s * np;
        u[out][C] = nu;
        v[out][C] = nv;
        p[out][C] = np;
      }
    // periodic_BC after the stage (see the header); it copies p and v only, u's ghost rows
    // are never written
    for (int i = 3; i < Nx - 3; i++) {
      if (!colfluid[i]) continue;
      for (std::vector<T>* f : {&p[out], &v[out]}) {
        std::vector<T>& q = *f;
        q[at(i, Ny - 3)] = q[at(i, Ny - 4)];
        q[at(i, Ny - 2)] = q[at(i, Ny - 4)];
        q[at(i, Ny - 1)] = q[at(i, Ny - 5)];
        q[at(i, 2)] = q[at(i, 3)];
        q[at(i, 1)] = q[at(i, 3)];
        q[at(i, 0)] = q[at(i, 3)];
      }
    }
    boundary(st, in, out);
  }

  // cubic_interp_1d and bicubic_interp (functions.cuh:421-478)
  static T cubic(T fm1, T f0, T f1, T f2, T s) {
    const T s2 = s * s;
    const T wm1 = -s * (s - (T)2) * (s - (T)1) / (T)6;
    const T w0 = (s - (T)2) * (s - (T)1) * (s + (T)1) / (T)2;
    const T w1 = s * (-s2 + s + (T)2) / (T)2;
    const T w2 = s * (s2 - (T)1) / (T)6;
    return wm1 * fm1 + w0 * f0 + w1 * f1 + w2 * f2;
  }
  T bicubic(const T* f, T Dx, T Dy) const {
    const T gx = Dx / h, gy = Dy / h;
    const int i = (int)std::floor(gx), j = (int)std::floor(gy);
    const T sx = gx - (T)i, sy = gy - (T)j;
    T g[4];
    for (int r = 0; r < 4; r++) {
      const int jj = j - 1 + r;
      g[r] = cubic(f[at(i - 1, jj)], f[at(i, jj)], f[at(i + 1, jj)], f[at(i + 2, jj)], sx);
    }
    return cubic(g[0], g[1], g[2], g[3], sy);
  }

  // ADE_solver (functions.cuh:635-669) with the stage constants and state sets of main.cu:816-825
  T ade(int b, int m, T w_in, int st) {
    T a_, b_, c_;
    T *lf, *mf, *rf, *l1, *m1, *r1, *l2, *m2, *r2;
    if (st == 0) {
      a_ = 0; b_ = 1; c_ = 1;
      lf = phi.data(); mf = phi_old.data(); rf = phi_old.data();
      l1 = ps1.data(); m1 = ps1_old.data(); r1 = ps1_old.data();
      l2 = ps2.data(); m2 = ps2_old.data(); r2 = ps2_old.data();
    } else if (st == 1) {
      a_ = 3; b_ = 1; c_ = 4;
      lf = phi_nu.data(); mf = phi_old.data(); rf = phi.data();
      l1 = ps1_nu.data(); m1 = ps1_old.data(); r1 = ps1.data();
      l2 = ps2_nu.data(); m2 = ps2_old.data(); r2 = ps2.data();
    } else {
      a_ = 1; b_ = 2; c_ = 3;
      lf = phi.data(); mf = phi_old.data(); rf = phi_nu.data();
      l1 = ps1.data(); m1 = ps1_old.data(); r1 = ps1_nu.data();
      l2 = ps2.data(); m2 = ps2_old.data(); r2 = ps2_nu.data();
    }
    T sumA = 0, sumBC = 0;
    for (int k = 0; k < K; k++) {
      const int mm = m * K + k, s = b * K + k;
      const T Lphi = w_in - zeta[mm] * rf[s];
      T x = a_ * mf[s] + b_ * (rf[s] + dt * Lphi);
      x /= c_;
      lf[s] = x;
      sumA += A[mm] * x;
    }
    for (int l = 0; l < L; l++) {
      const int mm = m * L + l, s = b * L + l;
      const T L1 = w_in - (alpha[mm] * r1[s] + beta[mm] * r2[s]);
      const T L2 = beta[mm] * r1[s] - alpha[mm] * r2[s];
      T x1 = a_ * m1[s] + b_ * (r1[s] + dt * L1);
      x1 /= c_;
      T x2 = a_ * m2[s] + b_ * (r2[s] + dt * L2);
      x2 /= c_;
      l1[s] = x1;
      l2[s] = x2;
      sumBC += B[mm] * x1 + C[mm] * x2;
    }
    return Rinf[m] * w_in + sumA + sumBC;
  }

  // kernel_apply_BC_immersed_sdf (functions.cuh:672-783)
  void boundary(int st, int in, int out) {
    const T* Po = p[in].data();
    const T* Uo = u[in].data();
    const T* Vo = v[in].data();
    // every band node owns its ADE states and its own output node
#pragma omp parallel for schedule(static)
    for (int j = 3; j < Ny - 3; j++)
      for (int i = 3; i < Nx - 3; i++) {
        const size_t Cij = at(i, j);
        const uint8_t o = oid[Cij];
        if (o == 0 || o == 0xFF) continue;
        const T s = (T)S[Cij];
        const int b = bmap[Cij];
        const T gx = ((T)S[at(i + 1, j)] - (T)S[at(i - 1, j)]) * ((T)0.5f / h);
        const T gy = ((T)S[at(i, j + 1)] - (T)S[at(i, j - 1)]) * ((T)0.5f / h);
        T gn = std::sqrt(gx * gx + gy * gy);
        gn = std::max(gn, (T)1e-12f);
        const T nx = -gx / gn, ny = -gy / gn;
        const T Cx = (T)i * h, Cy = (T)j * h;
        const T Wx = Cx + s * nx, Wy = Cy + s * ny;
        const T l = s + h;
        const T Dx = Wx - l * nx, Dy = Wy - l * ny;
        const T pD = bicubic(Po, Dx, Dy), uD = bicubic(Uo, Dx, Dy), vD = bicubic(Vo, Dx, Dy);
        const T un = uD * nx + vD * ny;
        const T ut = -uD * ny + vD * nx;
        const T Z0 = rho * c;
        const T w_out = pD + Z0 * un;
        const T w_in = ade(b, (int)o - 1, w_out, st);
        const T p_b = (T)0.5f * (w_in + w_out);
        const T un_b = (w_out - w_in) / ((T)2 * Z0);
        const T u_b = un_b * nx - ut * ny;
        const T v_b = un_b * ny + ut * nx;
        T chi;
        if (s >= tol) chi = 0;
        else if (s <= h) chi = 1;
        else {
          const T r = (s - h) / (tol - h);
          chi = (T)1 - r * r * ((T)3 - (T)2 * r);
        }
        u[out][Cij] = ((T)1 - chi) * u[out][Cij] + chi * u_b;
        v[out][Cij] = ((T)1 - chi) * v[out][Cij] + chi * v_b;
        p[out][Cij] = ((T)1 - chi) * p[out][Cij] + chi * p_b;
      }
  }
};

template <class T>
int run(int Nx, int Ny, double h, double dt, double rho, double c, double eps, double tol, const int* pml,
        const float* S, const uint8_t* oid, int nmat, int K, int L, const double* Rinf, const double* A,
        const double* zeta, const double* B, const double* C, const double* alpha, const double* beta,
        const double* p0, const double* u0, const double* v0, int ri, int rj, int64_t nsteps, double* ir,
        double* pout, double* uout, double* vout) {
  if (Nx < 10 || Ny < 10 || nmat < 0 || K < 0 || L < 0) return -1;
  Legacy2D<T> m;
  m.Nx = Nx; m.Ny = Ny;
  m.h = (T)h; m.dt = (T)dt; m.rho = (T)rho; m.c = (T)c; m.eps = (T)eps; m.tol = (T)tol;
  m.keyN = (T)pml[0]; m.keyS = (T)pml[1]; m.keyE = (T)pml[2]; m.keyW = (T)pml[3];
  m.S = S; m.oid = oid; m.K = K; m.L = L;
  auto cp = [](const double* a, size_t n) {
    std::vector<T> r(n, (T)0);
    for (size_t q = 0; q < n && a; q++) r[q] = (T)a[q];
    return r;
  };
  m.Rinf = cp(Rinf, nmat); m.A = cp(A, (size_t)nmat * K); m.zeta = cp(zeta, (size_t)nmat * K);
  m.B = cp(B, (size_t)nmat * L); m.C = cp(C, (size_t)nmat * L);
  m.alpha = cp(alpha, (size_t)nmat * L); m.beta = cp(beta, (size_t)nmat * L);
  const size_t N = (size_t)Nx * Ny;
  for (int q = 0; q < 3; q++) {
    m.p[q].assign(N, 0); m.u[q].assign(N, 0); m.v[q].assign(N, 0);
  }
  m.p[0] = cp(p0, N); m.u[0] = cp(u0, N); m.v[0] = cp(v0, N);
  // build_boundary_map (common/filterABC.h:95-108)
  m.bmap.assign(N, -1);
  int nB = 0;
  for (size_t q = 0; q < N; q++)
    if (oid[q] != 0xFF && oid[q] != 0) {
      if ((int)oid[q] > nmat) return -1;
      m.bmap[q] = nB++;
    }
  const size_t nk = (size_t)nB * K, nl = (size_t)nB * L;
  for (auto* a : {&m.phi, &m.phi_old, &m.phi_nu}) a->assign(nk, 0);
  for (auto* a : {&m.ps1, &m.ps1_old, &m.ps1_nu, &m.ps2, &m.ps2_old, &m.ps2_nu}) a->assign(nl, 0);
  m.colfluid.assign(Nx, 0);
  for (int i = 3; i < Nx - 3; i++)
    for (int j = 3; j < Ny - 3; j++)
      if (!(S[m.at(i, j)] < (float)h)) m.colfluid[i] = 1;
  for (int64_t n = 0; n < nsteps; n++) {
    m.stage(0);
    m.stage(1);
    m.stage(2);
    m.p[0] = m.p[1]; m.u[0] = m.u[1]; m.v[0] = m.v[1];
    m.phi_old = m.phi; m.ps1_old = m.ps1; m.ps2_old = m.ps2;
    if (ir) ir[n] = (double)m.p[1][m.at(ri, rj)];
  }
  for (size_t q = 0; q < N; q++) {
    if (pout) pout[q] = (double)m.p[0][q];
    if (uout) uout[q] = (double)m.u[0][q];
    if (vout) vout[q] = (double)m.v[0][q];
  }
  return 0;
}

}  // namespace

extern "C" int orc_l2d_run(int use_float, int Nx, int Ny, double h, double dt, double rho, double c, double eps,
                           double tol, const int* pml, const float* S, const uint8_t* oid, int nmat, int K, int L,
                           const double* Rinf, const double* A, const double* zeta, const double* B,
                           const double* C, const double* alpha, const double* beta, const double* p0,
                           const double* u0, const double* v0, int ri, int rj, int64_t nsteps, double* ir,
                           double* pout, double* uout, double* vout) {
  if (use_float)
    return run<float>(Nx, Ny, h, dt, rho, c, eps, tol, pml, S, oid, nmat, K, L, Rinf, A, zeta, B, C, alpha, beta, p0,
                      u0, v0, ri, rj, nsteps, ir, pout, uout, vout);
  return run<double>(Nx, Ny, h, dt, rho, c, eps, tol, pml, S, oid, nmat, K, L, Rinf, A, zeta, B, C, alpha, beta, p0,
                     u0, v0, ri, rj, nsteps, ir, pout, uout, vout);
}
