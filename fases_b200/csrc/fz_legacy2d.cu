// fz_legacy2d.cu -- the 2D legacy scheme of the reference's `2D-solver/` (include/fz_legacy2d.h).
//
// One fused kernel per SSP-RK3 stage replaces the reference's stage kernel, its in-kernel
// ghost-row copy and its separate immersed-boundary kernel (2D-solver/core/main.cu:816-825):
//   - a 32 x 6 tile of nodes with a 3-node halo of the stage input (p, u, v) is staged in shared
//     memory; the WENO-JS stencils and the bicubic boundary probe (always within 3 nodes of the
//     band node: D = C - h n) read only from there;
//   - every node's two face values per direction and variable (V+ at i+1/2, V- at i-1/2) are
//     reconstructed once, by one thread, into shared memory (34 x 6 nodes for x, 32 x 8 for y:
//     one pass of the 256 threads each), where the reference reconstructs every face twice, once
//     from each side;
//   - fluid nodes (S >= h) get the stage update and the multiplicative sPML;
//   - the nodes of rows 3, Ny-5 and Ny-4 write the ghost rows of p and v of their column;
//   - band nodes then run their ADE stage and blend the boundary state in, from the same tile;
//   - in the last stage the receiver node records its sample.
// Buffers: U0 and U1 swap roles every step instead of the reference's U0 <- U1 copy (one copy
// after the first step makes them equal everywhere, after which the swap is exact), and the ADE
// state sets swap old/current the same way. The step is captured in CUDA graphs.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "fz.h"
#include "fz_legacy2d.h"

namespace l2d {

constexpr int TX = 32, TY = 6, HALO = 3, NT = 256;
constexpr int SX = TX + 2 * HALO, SY = TY + 2 * HALO;
constexpr int FX = TX + 2, FY = TY + 2;  // face-value columns (x) and rows (y) of a tile
constexpr uint8_t FLUID = 1, BAND = 2;
constexpr int32_t ERR_PROBE = 1;
constexpr int GRAPH_STEPS = 32;  // even: a graph starts and ends with U0 in buffer 0

template <class R>
struct Band {
  R nx, ny, sx, sy, chi;
  int32_t ib, jb;  // bicubic base node (the stencil is ib-1..ib+2, jb-1..jb+2)
  int32_t mat;
};

template <class R>
struct Args {
  int Nx, Ny;
  R h, dt, rho, c, eps;
  R keyN, keyS, keyE, keyW, half;
  const R* in[3];    // stage input p, u, v (stencils and probes)
  const R* base[3];  // U0 p, u, v (stages 1 and 2)
  R* out[3];
  const uint8_t* cls;
  const uint8_t* colfluid;
  const int32_t* bidx;  // band index of each node, -1 elsewhere
  const Band<R>* band;
  int K, L;
  const R *Rinf, *A, *zeta, *B, *C, *alpha, *beta;
  R a_ssp, b_ssp, c_ssp;
  R* phiL; const R* phiM; const R* phiR;
  R* p1L; const R* p1M; const R* p1R;
  R* p2L; const R* p2M; const R* p2R;
  int64_t rec;
  int64_t nsamples;
  double* ir;
  int64_t* step;
  int32_t* err;
};

// WENO5-JS value at face i+1/2 (IDX 1) or i-1/2 (IDX 0) of the node f points at, stride st;
// candidate and smoothness tables of 2D-solver/core/main.cu:638-651, weights of
// functions.cuh:1096-1112, the smoothness indicator in double as functions.cuh:1115-1123
template <class R, int IDX>
__device__ __forceinline__ R weno_js(const R* f, int st, R eps) {
  constexpr double crl[4][3] = {{11.0 / 6.0, -7.0 / 6.0, 1.0 / 3.0},
                                {1.0 / 3.0, 5.0 / 6.0, -1.0 / 6.0},
                                {-1.0 / 6.0, 5.0 / 6.0, 1.0 / 3.0},
                                {1.0 / 3.0, -7.0 / 6.0, 11.0 / 6.0}};
  constexpr double brl[3][3] = {{3, -4, 1}, {1, 0, -1}, {1, -4, 3}};
  constexpr double dd[3] = {3.0 / 10.0, 3.0 / 5.0, 1.0 / 10.0};
  R V[3], al[3];
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const R q0 = f[-r * st], q1 = f[(1 - r) * st], q2 = f[(2 - r) * st];
    R acc = R(0);
    acc += (R)crl[r + IDX][0] * q0;
    acc += (R)crl[r + IDX][1] * q1;
    acc += (R)crl[r + IDX][2] * q2;
    V[r] = acc;
    const R b1 = q0 - R(2) * q1 + q2;
    const R b2 = (R)brl[r][0] * q0 + (R)brl[r][1] * q1 + (R)brl[r][2] * q2;
    const R bt = (R)((13.0 * (double)b1 * (double)b1 / 12.0) + (0.25 * (double)b2 * (double)b2));
    const R aux = bt + eps;
    al[r] = (R)dd[IDX == 1 ? r : 2 - r] / (aux * aux);
  }
  R out = R(0);
#pragma unroll
  for (int r = 0; r < 3; r++) out += (al[r] / (al[0] + al[1] + al[2])) * V[r];
  return out;
}

template <class R>
__device__ __forceinline__ R cubic(R fm1, R f0, R f1, R f2, R s) {
  const R s2 = s * s;
  const R wm1 = -s * (s - R(2)) * (s - R(1)) / R(6);
  const R w0 = (s - R(2)) * (s - R(1)) * (s + R(1)) / R(2);
  const R w1 = s * (-s2 + s + R(2)) / R(2);
  const R w2 = s * (s2 - R(1)) / R(6);
  return wm1 * fm1 + w0 * f0 + w1 * f1 + w2 * f2;
}

template <class R, int STAGE>
__global__ void __launch_bounds__(NT) k_l2d_stage(const Args<R> a) {
  __shared__ R sm[3][SY][SX];
  __shared__ R xf[4][TY][FX];  // p+, p-, u+, u- of nodes i0-1 .. i0+TX
  __shared__ R yf[4][FY][TX];  // p+, p-, v+, v- of nodes j0-1 .. j0+TY
  const int t = threadIdx.x;
  const int i0 = blockIdx.x * TX + HALO, j0 = blockIdx.y * TY + HALO;
  for (int q = t; q < SX * SY; q += NT) {
    const int x = q % SX, y = q / SX;
    const int gi = i0 - HALO + x, gj = j0 - HALO + y;
    const bool ok = gi < a.Nx && gj < a.Ny;
    const size_t g = (size_t)gj * a.Nx + gi;
#pragma unroll
    for (int f = 0; f < 3; f++) sm[f][y][x] = ok ? a.in[f][g] : R(0);
  }
  __syncthreads();
  // face values: WENO_x / WENO_y of functions.cuh:1125-1176, each face once
  if (t < FX * TY) {
    const int row = t / FX, col = t % FX;  // node (i0 + col - 1, j0 + row)
    const R* fp = &sm[0][row + HALO][col + HALO - 1];
    const R* fu = &sm[1][row + HALO][col + HALO - 1];
    xf[0][row][col] = weno_js<R, 1>(fp, 1, a.eps);
    xf[1][row][col] = weno_js<R, 0>(fp, 1, a.eps);
    xf[2][row][col] = weno_js<R, 1>(fu, 1, a.eps);
    xf[3][row][col] = weno_js<R, 0>(fu, 1, a.eps);
  }
  {
    const int row = t / TX, col = t % TX;  // node (i0 + col, j0 + row - 1)
    const R* fp = &sm[0][row + HALO - 1][col + HALO];
    const R* fv = &sm[2][row + HALO - 1][col + HALO];
    yf[0][row][col] = weno_js<R, 1>(fp, SX, a.eps);
    yf[1][row][col] = weno_js<R, 0>(fp, SX, a.eps);
    yf[2][row][col] = weno_js<R, 1>(fv, SX, a.eps);
    yf[3][row][col] = weno_js<R, 0>(fv, SX, a.eps);
  }
  __syncthreads();
  if (t >= TX * TY) return;
  const int tx = t % TX, ty = t / TX;
  const int i = i0 + tx, j = j0 + ty;
  if (i >= a.Nx - 3 || j >= a.Ny - 3) return;
  const size_t C = (size_t)j * a.Nx + i;
  const uint8_t cl = a.cls[C];
  R np, nu, nv;
  if (cl & FLUID) {
    const R* sp = &sm[0][ty + HALO][tx + HALO];
    const R* su = &sm[1][ty + HALO][tx + HALO];
    const R* sv = &sm[2][ty + HALO][tx + HALO];
    const R rho = a.rho, c = a.c;
    // Godunov fluxes of functions.cuh:199-213 (the 0.5 applied in double as there) on the face
    // values of compute_Vs_x / compute_Vs_y: [0] V+ at i, [1] V- at i+1, [2] V+ at i-1, [3] V- at i
    auto Fp = [&](R pM, R pP, R uM, R uP) { return (R)(0.5 * (double)(rho * c * c * (uP + uM) - c * (pP - pM))); };
    auto Fu = [&](R pM, R pP, R uM, R uP) { return (R)(0.5 * (double)((pP + pM) / rho - c * (uP - uM))); };
    auto Gv = [&](R pM, R pP, R vM, R vP) { return (R)(0.5 * (double)((pM + pP) / rho - c * (vP - vM))); };
    R FpP, FpM, FuP, FuM, GpP, GpM, GvP, GvM;
    {
      const int x = tx + 1;
      const R p0 = xf[0][ty][x], p1 = xf[1][ty][x + 1], p2 = xf[0][ty][x - 1], p3 = xf[1][ty][x];
      const R u0 = xf[2][ty][x], u1 = xf[3][ty][x + 1], u2 = xf[2][ty][x - 1], u3 = xf[3][ty][x];
      FpP = Fp(p0, p1, u0, u1);
      FpM = Fp(p2, p3, u2, u3);
      FuP = Fu(p0, p1, u0, u1);
      FuM = Fu(p2, p3, u2, u3);
    }
    {
      const int y = ty + 1;
      const R p0 = yf[0][y][tx], p1 = yf[1][y + 1][tx], p2 = yf[0][y - 1][tx], p3 = yf[1][y][tx];
      const R v0 = yf[2][y][tx], v1 = yf[3][y + 1][tx], v2 = yf[2][y - 1][tx], v3 = yf[3][y][tx];
      GpP = Fp(p0, p1, v0, v1);
      GpM = Fp(p2, p3, v2, v3);
      GvP = Gv(p0, p1, v0, v1);
      GvM = Gv(p2, p3, v2, v3);
    }
    const R ru = a.dt * ((-FuP + FuM) / a.h);
    const R rv = a.dt * ((-GvP + GvM) / a.h);
    const R rp = a.dt * ((-FpP + FpM - GpP + GpM) / a.h);
    // kernel_WENO_step0/1/2 combinations (functions.cuh:1241-1243, 1311-1313, 1378-1380)
    if (STAGE == 0) {
      nu = *su + ru;
      nv = *sv + rv;
      np = *sp + rp;
    } else if (STAGE == 1) {
      nu = (R)0.75f * a.base[1][C] + (R)0.25f * (*su + ru);
      nv = (R)0.75f * a.base[2][C] + (R)0.25f * (*sv + rv);
      np = (R)0.75f * a.base[0][C] + (R)0.25f * (*sp + rp);
    } else {
      nu = (a.base[1][C] + R(2) * (*su + ru)) / R(3);
      nv = (a.base[2][C] + R(2) * (*sv + rv)) / R(3);
      np = (a.base[0][C] + R(2) * (*sp + rp)) / R(3);
    }
    // sPML (functions.cuh:941-965)
    const R one = R(1), zero = R(0), half = a.half;
    const R rx = a.keyE * fmax(zero, fmin((R)(i - (a.Nx - half)) / half, one));
    const R lx = a.keyW * fmax(zero, fmin((half - i) / half, one));
    const R ly = a.keyS * fmax(zero, fmin((half - j) / half, one));
    const R uy = a.keyN * fmax(zero, fmin((j - (a.Ny - half)) / half, one));
    const R smax = (R)0.018f;
    const R sx = smax * (rx * rx * rx + lx * lx * lx);
    const R sy = smax * (uy * uy * uy + ly * ly * ly);
    const R s = fmin(sx + sy - sx * sy, (R)0.999f);
    nu -= s * nu;
    nv -= s * nv;
    np -= s * np;
  } else {
    np = a.out[0][C];
    nu = a.out[1][C];
    nv = a.out[2][C];
  }
  // ghost rows of p and v (periodic_BC, functions.cuh:268-298)
  if (a.colfluid[i]) {
    const int Nx = a.Nx, Ny = a.Ny;
    if (j == 3) {
      for (int r = 0; r < 3; r++) {
        a.out[0][(size_t)r * Nx + i] = np;
        a.out[2][(size_t)r * Nx + i] = nv;
      }
    } else if (j == Ny - 4) {
      for (int r = Ny - 3; r < Ny - 1; r++) {
        a.out[0][(size_t)r * Nx + i] = np;
        a.out[2][(size_t)r * Nx + i] = nv;
      }
    } else if (j == Ny - 5) {
      a.out[0][(size_t)(Ny - 1) * Nx + i] = np;
      a.out[2][(size_t)(Ny - 1) * Nx + i] = nv;
    }
  }
  if (cl & BAND) {
    // kernel_apply_BC_immersed_sdf (functions.cuh:672-783) on the stage input in the tile
    const int b = a.bidx[C];
    const Band<R> g = a.band[b];
    const int x = g.ib - (i0 - HALO), y = g.jb - (j0 - HALO);
    R pD = R(0), uD = R(0), vD = R(0);
    if (x >= 1 && x + 2 < SX && y >= 1 && y + 2 < SY) {
      R gp[4], gu[4], gv[4];
#pragma unroll
      for (int r = 0; r < 4; r++) {
        const int yy = y - 1 + r;
        gp[r] = cubic(sm[0][yy][x - 1], sm[0][yy][x], sm[0][yy][x + 1], sm[0][yy][x + 2], g.sx);
        gu[r] = cubic(sm[1][yy][x - 1], sm[1][yy][x], sm[1][yy][x + 1], sm[1][yy][x + 2], g.sx);
        gv[r] = cubic(sm[2][yy][x - 1], sm[2][yy][x], sm[2][yy][x + 1], sm[2][yy][x + 2], g.sx);
      }
      pD = cubic(gp[0], gp[1], gp[2], gp[3], g.sy);
      uD = cubic(gu[0], gu[1], gu[2], gu[3], g.sy);
      vD = cubic(gv[0], gv[1], gv[2], gv[3], g.sy);
    } else {
      atomicOr(a.err, ERR_PROBE);
    }
    const R nx = g.nx, ny = g.ny;
    const R un = uD * nx + vD * ny;
    const R ut = -uD * ny + vD * nx;
    const R Z0 = a.rho * a.c;
    const R w_out = pD + Z0 * un;
    // ADE_solver (functions.cuh:635-669)
    const int m = g.mat;
    R sumA = R(0), sumBC = R(0);
    for (int k = 0; k < a.K; k++) {
      const int mm = m * a.K + k, s = b * a.K + k;
      const R Lphi = w_out - a.zeta[mm] * a.phiR[s];
      R v = a.a_ssp * a.phiM[s] + a.b_ssp * (a.phiR[s] + a.dt * Lphi);
      v /= a.c_ssp;
      a.phiL[s] = v;
      sumA += a.A[mm] * v;
    }
    for (int l = 0; l < a.L; l++) {
      const int mm = m * a.L + l, s = b * a.L + l;
      const R r1 = a.p1R[s], r2 = a.p2R[s];
      const R L1 = w_out - (a.alpha[mm] * r1 + a.beta[mm] * r2);
      const R L2 = a.beta[mm] * r1 - a.alpha[mm] * r2;
      R v1 = a.a_ssp * a.p1M[s] + a.b_ssp * (r1 + a.dt * L1);
      v1 /= a.c_ssp;
      R v2 = a.a_ssp * a.p2M[s] + a.b_ssp * (r2 + a.dt * L2);
      v2 /= a.c_ssp;
      a.p1L[s] = v1;
      a.p2L[s] = v2;
      sumBC += a.B[mm] * v1 + a.C[mm] * v2;
    }
    const R w_in = a.Rinf[m] * w_out + sumA + sumBC;
    const R p_b = (R)0.5f * (w_in + w_out);
    const R un_b = (w_out - w_in) / (R(2) * Z0);
    const R u_b = un_b * nx - ut * ny;
    const R v_b = un_b * ny + ut * nx;
    const R chi = g.chi;
    nu = (R(1) - chi) * nu + chi * u_b;
    nv = (R(1) - chi) * nv + chi * v_b;
    np = (R(1) - chi) * np + chi * p_b;
  }
  if (cl & (FLUID | BAND)) {
    a.out[0][C] = np;
    a.out[1][C] = nu;
    a.out[2][C] = nv;
  }
  if (STAGE == 2 && (int64_t)C == a.rec) {
    const int64_t n = *a.step;
    if (n < a.nsamples) a.ir[n] = (double)np;
    *a.step = n + 1;
  }
}

}  // namespace l2d

struct fz_l2d {
  fz_l2d_params prm{};
  int dev = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  size_t N = 0;
  bool fp64 = false;
  void* buf[3][3] = {};      // [buffer][p,u,v]; buffers 0/1 swap the U0/U1 roles, 2 is U2
  uint8_t* d_cls = nullptr;
  uint8_t* d_colfluid = nullptr;
  int32_t* d_bidx = nullptr;
  void* d_band = nullptr;
  void* d_coef[7] = {};      // Rinf, A, zeta, B, C, alpha, beta
  void* d_state[3][3] = {};  // [phi, psi1, psi2][set 0, set 1, nu]; sets 0/1 swap old/current
  double* d_ir = nullptr;
  int64_t* d_step = nullptr;
  int32_t* d_err = nullptr;
  int64_t nB = 0;
  int nmat = 0, K = 0, L = 0;
  bool geometry = false, materials = false;
  int max_oid = 0;
  int64_t rec = -1, nsamples = 0;
  int64_t steps = 0;
  int64_t rec_base = 0;    // step count when the trace last restarted
  int par = 0;             // buffer holding U0 (and state set holding the old ADE state)
  bool first_copy = true;  // U0 <- U1 once after the first step
  cudaGraphExec_t graph = nullptr;
};

namespace {

int fail(fz_l2d* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

int cuda_fail(fz_l2d* h, cudaError_t e, const char* what) {
  return fail(h, FZ_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define L2D_CUDA(h, call, what)                           \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_fail(h, e_, what); \
  } while (0)

size_t rsize(const fz_l2d* h) { return h->fp64 ? sizeof(double) : sizeof(float); }

void free_graph(fz_l2d* h) {
  if (h->graph) cudaGraphExecDestroy(h->graph);
  h->graph = nullptr;
}

template <class R>
void to_r(std::vector<unsigned char>& out, const double* a, size_t n) {
  out.assign(n * sizeof(R), 0);
  R* o = (R*)out.data();
  for (size_t q = 0; q < n; q++) o[q] = a ? (R)a[q] : R(0);
}

int upload(fz_l2d* h, void** dst, const double* src, size_t n, const char* what) {
  if (*dst) cudaFree(*dst);
  *dst = nullptr;
  const size_t bytes = std::max<size_t>(n, 1) * rsize(h);
  L2D_CUDA(h, cudaMalloc(dst, bytes), what);
  std::vector<unsigned char> tmp;
  if (h->fp64) to_r<double>(tmp, src, n); else to_r<float>(tmp, src, n);
  if (n) L2D_CUDA(h, cudaMemcpy(*dst, tmp.data(), n * rsize(h), cudaMemcpyHostToDevice), what);
  return FZ_OK;
}

// Band geometry of kernel_apply_BC_immersed_sdf (functions.cuh:686-718) and chi_layered
// (functions.cuh:534-543), in the arithmetic of the field type
template <class R>
int build_band(fz_l2d* h, const float* S, const uint8_t* oid, std::vector<int32_t>& bidx,
               std::vector<unsigned char>& out) {
  const int Nx = h->prm.Nx, Ny = h->prm.Ny;
  const R hh = (R)h->prm.h, tol = (R)h->prm.tol;
  std::vector<l2d::Band<R>> band;
  for (int j = 3; j < Ny - 3; j++)
    for (int i = 3; i < Nx - 3; i++) {
      const size_t C = (size_t)j * Nx + i;
      const uint8_t o = oid[C];
      if (o == 0 || o == 0xFF) continue;
      const R s = (R)S[C];
      const R gx = ((R)S[C + 1] - (R)S[C - 1]) * ((R)0.5f / hh);
      const R gy = ((R)S[C + Nx] - (R)S[C - Nx]) * ((R)0.5f / hh);
      R gn = std::sqrt(gx * gx + gy * gy);
      gn = std::max(gn, (R)1e-12f);
      const R nx = -gx / gn, ny = -gy / gn;
      const R Cx = (R)i * hh, Cy = (R)j * hh;
      const R Wx = Cx + s * nx, Wy = Cy + s * ny;
      const R l = s + hh;
      const R Dx = Wx - l * nx, Dy = Wy - l * ny;
      const R fx = Dx / hh, fy = Dy / hh;
      const int ib = (int)std::floor(fx), jb = (int)std::floor(fy);
      if (ib - 1 < i - 3 || ib + 2 > i + 3 || jb - 1 < j - 3 || jb + 2 > j + 3)
        return fail(h, FZ_EINVAL, "fz_l2d_load_geometry: the boundary probe of node (" + std::to_string(i) + "," +
                                      std::to_string(j) + ") leaves its 3-node neighbourhood (inconsistent S)");
      R chi;
      if (s >= tol) chi = R(0);
      else if (s <= hh) chi = R(1);
      else {
        const R r = (s - hh) / (tol - hh);
        chi = R(1) - r * r * (R(3) - R(2) * r);
      }
      l2d::Band<R> b;
      b.nx = nx; b.ny = ny;
      b.sx = fx - (R)ib; b.sy = fy - (R)jb;
      b.chi = chi;
      b.ib = ib; b.jb = jb;
      b.mat = (int32_t)o - 1;
      bidx[C] = (int32_t)band.size();
      band.push_back(b);
    }
  out.assign(band.size() * sizeof(l2d::Band<R>), 0);
  if (!band.empty()) std::memcpy(out.data(), band.data(), out.size());
  h->nB = (int64_t)band.size();
  return FZ_OK;
}

int wait(fz_l2d* h) {
  const auto t0 = std::chrono::steady_clock::now();
  int sleep_us = 20;
  for (;;) {
    const cudaError_t e = cudaStreamQuery(h->stream);
    if (e == cudaSuccess) break;
    if (e != cudaErrorNotReady) return cuda_fail(h, e, "stream");
    if (std::chrono::steady_clock::now() - t0 > std::chrono::minutes(10))
      return fail(h, FZ_ETIMEOUT, "fz_l2d: device work did not finish in time");
    std::this_thread::sleep_for(std::chrono::microseconds(sleep_us));
    sleep_us = std::min(sleep_us * 2, 2000);
  }
  int32_t kerr = 0;
  L2D_CUDA(h, cudaMemcpy(&kerr, h->d_err, sizeof(kerr), cudaMemcpyDeviceToHost), "error word D2H");
  if (kerr) return fail(h, FZ_EBOUNDS, "fz_l2d: a boundary probe left the staged tile");
  return FZ_OK;
}

template <class R>
l2d::Args<R> args(fz_l2d* h, int stage, int par) {
  l2d::Args<R> a{};
  const fz_l2d_params& p = h->prm;
  a.Nx = p.Nx; a.Ny = p.Ny;
  a.h = (R)p.h; a.dt = (R)p.dt; a.rho = (R)p.rho; a.c = (R)p.c; a.eps = (R)p.eps;
  a.keyN = (R)p.pml_n; a.keyS = (R)p.pml_s; a.keyE = (R)p.pml_e; a.keyW = (R)p.pml_w;
  a.half = (R)(int)(0.15f * (float)std::min(p.Nx, p.Ny));
  const int b0 = par, b1 = 1 - par;
  const int in = stage == 0 ? b0 : (stage == 1 ? b1 : 2);
  const int out = stage == 1 ? 2 : b1;
  for (int f = 0; f < 3; f++) {
    a.in[f] = (const R*)h->buf[in][f];
    a.base[f] = (const R*)h->buf[b0][f];
    a.out[f] = (R*)h->buf[out][f];
  }
  a.cls = h->d_cls; a.colfluid = h->d_colfluid; a.bidx = h->d_bidx; a.band = (const l2d::Band<R>*)h->d_band;
  a.K = h->K; a.L = h->L;
  a.Rinf = (const R*)h->d_coef[0]; a.A = (const R*)h->d_coef[1]; a.zeta = (const R*)h->d_coef[2];
  a.B = (const R*)h->d_coef[3]; a.C = (const R*)h->d_coef[4]; a.alpha = (const R*)h->d_coef[5];
  a.beta = (const R*)h->d_coef[6];
  // ADE state sets and SSP constants of main.cu:816-825 (left, middle, right)
  const int so = par, sc = 1 - par;
  R* st[3][3];
  for (int q = 0; q < 3; q++)
    for (int s = 0; s < 3; s++) st[q][s] = (R*)h->d_state[q][s];
  int lft, rgt;
  if (stage == 0) { a.a_ssp = R(0); a.b_ssp = R(1); a.c_ssp = R(1); lft = sc; rgt = so; }
  else if (stage == 1) { a.a_ssp = R(3); a.b_ssp = R(1); a.c_ssp = R(4); lft = 2; rgt = sc; }
  else { a.a_ssp = R(1); a.b_ssp = R(2); a.c_ssp = R(3); lft = sc; rgt = 2; }
  a.phiL = st[0][lft]; a.phiM = st[0][so]; a.phiR = st[0][rgt];
  a.p1L = st[1][lft]; a.p1M = st[1][so]; a.p1R = st[1][rgt];
  a.p2L = st[2][lft]; a.p2M = st[2][so]; a.p2R = st[2][rgt];
  a.rec = h->rec; a.nsamples = h->nsamples; a.ir = h->d_ir; a.step = h->d_step; a.err = h->d_err;
  return a;
}

template <class R>
cudaError_t enqueue_step(fz_l2d* h, int par) {
  const dim3 blk(l2d::NT);
  const dim3 grd((h->prm.Nx - 6 + l2d::TX - 1) / l2d::TX, (h->prm.Ny - 6 + l2d::TY - 1) / l2d::TY);
  l2d::k_l2d_stage<R, 0><<<grd, blk, 0, h->stream>>>(args<R>(h, 0, par));
  l2d::k_l2d_stage<R, 1><<<grd, blk, 0, h->stream>>>(args<R>(h, 1, par));
  l2d::k_l2d_stage<R, 2><<<grd, blk, 0, h->stream>>>(args<R>(h, 2, par));
  return cudaGetLastError();
}

cudaError_t step(fz_l2d* h, int par) { return h->fp64 ? enqueue_step<double>(h, par) : enqueue_step<float>(h, par); }

int ready(fz_l2d* h) {
  if (!h->geometry) return fail(h, FZ_ESTATE, "fz_l2d: load the geometry first");
  if (h->nB > 0 && !h->materials) return fail(h, FZ_ESTATE, "fz_l2d: the geometry has band cells: set the materials");
  if (h->materials && h->max_oid > h->nmat)
    return fail(h, FZ_EINVAL, "fz_l2d: the geometry names material " + std::to_string(h->max_oid) + " of " +
                                  std::to_string(h->nmat));
  return FZ_OK;
}

size_t state_count(const fz_l2d* h, int q) {
  return (size_t)std::max<int64_t>(h->nB, 1) * std::max(q == 0 ? h->K : h->L, 1);
}

int alloc_states(fz_l2d* h) {
  free_graph(h);
  for (int q = 0; q < 3; q++)
    for (int s = 0; s < 3; s++) {
      if (h->d_state[q][s]) cudaFree(h->d_state[q][s]);
      h->d_state[q][s] = nullptr;
      const size_t n = state_count(h, q);
      L2D_CUDA(h, cudaMalloc(&h->d_state[q][s], n * rsize(h)), "cudaMalloc(ADE state)");
      L2D_CUDA(h, cudaMemset(h->d_state[q][s], 0, n * rsize(h)), "ADE state reset");
    }
  return FZ_OK;
}

}  // namespace

extern "C" {

void fz_l2d_params_init(fz_l2d_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  // the reference's float arithmetic (main.cu:82, 378-392, 591) at 22 C and C_CFL = 0.2
  const float hf = 0.005f, T = 22.0f + 273.15f;
  const float cf = std::sqrt(1.4f * 287.05f * T);
  p->h = hf;
  p->c = cf;
  p->rho = 1.225f;
  p->dt = 0.2f * hf / cf;
  p->eps = 1e-7f;
  p->tol = 3.0f * hf;
  p->pml_n = 1;
  p->pml_s = 1;
  p->precision = FZ_FP32;
}

int fz_l2d_create(const fz_l2d_params* p, fz_l2d** out) {
  if (!p || !out) return FZ_EINVAL;
  *out = nullptr;
  if (p->Nx < 10 || p->Ny < 10 || !(p->h > 0) || !(p->dt > 0) || !(p->rho > 0) || !(p->c > 0) || !(p->eps > 0) ||
      !(p->tol > p->h) || (p->precision != FZ_FP32 && p->precision != FZ_FP64))
    return FZ_EINVAL;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return FZ_ENODEV;
  if (p->device < 0 || p->device >= ndev) return FZ_EINVAL;
  fz_l2d* h = new (std::nothrow) fz_l2d;
  if (!h) return FZ_ENOMEM;
  h->prm = *p;
  h->dev = p->device;
  h->fp64 = p->precision == FZ_FP64;
  h->N = (size_t)p->Nx * p->Ny;
  cudaSetDevice(h->dev);
  auto bad = [&](cudaError_t e) {
    if (e == cudaSuccess) return false;
    fz_l2d_destroy(h);
    return true;
  };
  if (bad(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking))) return FZ_ECUDA;
  for (int b = 0; b < 3; b++)
    for (int f = 0; f < 3; f++)
      if (bad(cudaMalloc(&h->buf[b][f], h->N * rsize(h))) || bad(cudaMemset(h->buf[b][f], 0, h->N * rsize(h))))
        return FZ_ENOMEM;
  if (bad(cudaMalloc(&h->d_step, sizeof(int64_t))) || bad(cudaMemset(h->d_step, 0, sizeof(int64_t))) ||
      bad(cudaMalloc(&h->d_err, sizeof(int32_t))) || bad(cudaMemset(h->d_err, 0, sizeof(int32_t))))
    return FZ_ENOMEM;
  *out = h;
  return FZ_OK;
}

int fz_l2d_destroy(fz_l2d* h) {
  if (!h) return FZ_EINVAL;
  cudaSetDevice(h->dev);
  if (h->stream) cudaStreamSynchronize(h->stream);
  free_graph(h);
  for (auto& b : h->buf)
    for (void*& f : b) cudaFree(f);
  for (auto& q : h->d_state)
    for (void*& s : q) cudaFree(s);
  for (void*& c : h->d_coef) cudaFree(c);
  cudaFree(h->d_cls); cudaFree(h->d_colfluid); cudaFree(h->d_bidx); cudaFree(h->d_band);
  cudaFree(h->d_ir); cudaFree(h->d_step); cudaFree(h->d_err);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return FZ_OK;
}

int fz_l2d_load_geometry(fz_l2d* h, const float* S, const uint8_t* oid) {
  if (!h) return FZ_EINVAL;
  if (!S || !oid) return fail(h, FZ_EINVAL, "fz_l2d_load_geometry: NULL array");
  cudaSetDevice(h->dev);
  const int Nx = h->prm.Nx, Ny = h->prm.Ny;
  const float hf = (float)h->prm.h;
  std::vector<uint8_t> cls(h->N, 0), colfluid((size_t)Nx, 0);
  std::vector<int32_t> bidx(h->N, -1);
  int max_oid = 0;
  for (int j = 3; j < Ny - 3; j++)
    for (int i = 3; i < Nx - 3; i++) {
      const size_t C = (size_t)j * Nx + i;
      if (!std::isfinite(S[C])) return fail(h, FZ_EINVAL, "fz_l2d_load_geometry: non-finite S");
      if (!(S[C] < hf)) {
        cls[C] |= l2d::FLUID;
        colfluid[(size_t)i] = 1;
      }
      if (oid[C] != 0 && oid[C] != 0xFF) {
        cls[C] |= l2d::BAND;
        max_oid = std::max(max_oid, (int)oid[C]);
      }
    }
  std::vector<unsigned char> band;
  const int rc = h->fp64 ? build_band<double>(h, S, oid, bidx, band) : build_band<float>(h, S, oid, bidx, band);
  if (rc != FZ_OK) return rc;
  free_graph(h);
  cudaFree(h->d_cls); cudaFree(h->d_colfluid); cudaFree(h->d_bidx); cudaFree(h->d_band);
  h->d_cls = nullptr; h->d_colfluid = nullptr; h->d_bidx = nullptr; h->d_band = nullptr;
  L2D_CUDA(h, cudaMalloc(&h->d_cls, h->N), "cudaMalloc(cls)");
  L2D_CUDA(h, cudaMemcpy(h->d_cls, cls.data(), h->N, cudaMemcpyHostToDevice), "cls H2D");
  L2D_CUDA(h, cudaMalloc(&h->d_colfluid, (size_t)Nx), "cudaMalloc(colfluid)");
  L2D_CUDA(h, cudaMemcpy(h->d_colfluid, colfluid.data(), (size_t)Nx, cudaMemcpyHostToDevice), "colfluid H2D");
  L2D_CUDA(h, cudaMalloc(&h->d_bidx, h->N * sizeof(int32_t)), "cudaMalloc(band index)");
  L2D_CUDA(h, cudaMemcpy(h->d_bidx, bidx.data(), h->N * sizeof(int32_t), cudaMemcpyHostToDevice), "band index H2D");
  L2D_CUDA(h, cudaMalloc(&h->d_band, std::max<size_t>(band.size(), 16)), "cudaMalloc(band)");
  if (!band.empty())
    L2D_CUDA(h, cudaMemcpy(h->d_band, band.data(), band.size(), cudaMemcpyHostToDevice), "band H2D");
  h->max_oid = max_oid;
  h->geometry = true;
  const int r2 = alloc_states(h);
  if (r2 != FZ_OK) return r2;
  return fz_l2d_set_fields(h, nullptr, nullptr, nullptr);
}

int fz_l2d_set_materials(fz_l2d* h, int nmat, int K, int L, const double* Rinf, const double* A, const double* zeta,
                         const double* B, const double* C, const double* alpha, const double* beta) {
  if (!h) return FZ_EINVAL;
  if (nmat < 1 || nmat > 254 || K < 0 || L < 0 || K > 64 || L > 64 || !Rinf || (K && (!A || !zeta)) ||
      (L && (!B || !C || !alpha || !beta)))
    return fail(h, FZ_EINVAL, "fz_l2d_set_materials: bad counts or NULL coefficient array");
  cudaSetDevice(h->dev);
  L2D_CUDA(h, cudaStreamSynchronize(h->stream), "stream");
  free_graph(h);
  const size_t nk = (size_t)nmat * K, nl = (size_t)nmat * L;
  const double* src[7] = {Rinf, A, zeta, B, C, alpha, beta};
  const size_t cnt[7] = {(size_t)nmat, nk, nk, nl, nl, nl, nl};
  for (int q = 0; q < 7; q++) {
    const int rc = upload(h, &h->d_coef[q], src[q], cnt[q], "material coefficients");
    if (rc != FZ_OK) return rc;
  }
  h->nmat = nmat;
  h->K = K;
  h->L = L;
  h->materials = true;
  const int rc = alloc_states(h);
  if (rc != FZ_OK) return rc;
  return fz_l2d_set_fields(h, nullptr, nullptr, nullptr);
}

int fz_l2d_set_fields(fz_l2d* h, const double* p, const double* u, const double* v) {
  if (!h) return FZ_EINVAL;
  cudaSetDevice(h->dev);
  L2D_CUDA(h, cudaStreamSynchronize(h->stream), "stream");
  const double* in[3] = {p, u, v};
  std::vector<unsigned char> tmp;
  for (int b = 0; b < 3; b++)
    for (int f = 0; f < 3; f++) {
      if (b == 0 && in[f]) {
        if (h->fp64) to_r<double>(tmp, in[f], h->N); else to_r<float>(tmp, in[f], h->N);
        L2D_CUDA(h, cudaMemcpy(h->buf[0][f], tmp.data(), h->N * rsize(h), cudaMemcpyHostToDevice), "fields H2D");
      } else {
        L2D_CUDA(h, cudaMemset(h->buf[b][f], 0, h->N * rsize(h)), "fields reset");
      }
    }
  for (int q = 0; q < 3; q++)
    for (int s = 0; s < 3; s++)
      if (h->d_state[q][s])
        L2D_CUDA(h, cudaMemset(h->d_state[q][s], 0, state_count(h, q) * rsize(h)), "ADE state reset");
  L2D_CUDA(h, cudaMemset(h->d_step, 0, sizeof(int64_t)), "step reset");
  if (h->d_ir && h->nsamples) L2D_CUDA(h, cudaMemset(h->d_ir, 0, h->nsamples * sizeof(double)), "trace reset");
  h->steps = 0;
  h->rec_base = 0;
  h->par = 0;
  h->first_copy = true;
  return FZ_OK;
}

int fz_l2d_set_receiver(fz_l2d* h, int i, int j, int64_t nsamples) {
  if (!h) return FZ_EINVAL;
  if (i < 3 || i >= h->prm.Nx - 3 || j < 3 || j >= h->prm.Ny - 3 || nsamples < 0)
    return fail(h, FZ_EINVAL,
                "fz_l2d_set_receiver: the receiver must be an interior node (3 <= i < Nx-3, 3 <= j < Ny-3)");
  cudaSetDevice(h->dev);
  L2D_CUDA(h, cudaStreamSynchronize(h->stream), "stream");
  free_graph(h);
  cudaFree(h->d_ir);
  h->d_ir = nullptr;
  L2D_CUDA(h, cudaMalloc(&h->d_ir, std::max<int64_t>(nsamples, 1) * sizeof(double)), "cudaMalloc(trace)");
  L2D_CUDA(h, cudaMemset(h->d_ir, 0, std::max<int64_t>(nsamples, 1) * sizeof(double)), "trace reset");
  L2D_CUDA(h, cudaMemset(h->d_step, 0, sizeof(int64_t)), "step reset");
  h->rec = (int64_t)j * h->prm.Nx + i;
  h->nsamples = nsamples;
  h->rec_base = h->steps;
  return FZ_OK;
}

int fz_l2d_run(fz_l2d* h, int64_t nsteps) {
  if (!h || nsteps < 0) return FZ_EINVAL;
  int rc = ready(h);
  if (rc != FZ_OK) return rc;
  cudaSetDevice(h->dev);
  int64_t left = nsteps;
  while (left > 0) {
    if (h->first_copy) {
      L2D_CUDA(h, step(h, h->par), "stage launch");
      // U0 <- U1 after the first step (main.cu:828-831); afterwards the buffers only swap roles
      for (int f = 0; f < 3; f++)
        L2D_CUDA(h, cudaMemcpyAsync(h->buf[h->par][f], h->buf[1 - h->par][f], h->N * rsize(h),
                                    cudaMemcpyDeviceToDevice, h->stream), "U0 <- U1");
      h->par ^= 1;
      h->first_copy = false;
      left--;
      h->steps++;
      continue;
    }
    if (h->par == 0 && left >= l2d::GRAPH_STEPS) {
      if (!h->graph) {
        cudaGraph_t g = nullptr;
        L2D_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        cudaError_t e = cudaSuccess;
        for (int s = 0; s < l2d::GRAPH_STEPS && e == cudaSuccess; s++) e = step(h, s & 1);
        const cudaError_t e2 = cudaStreamEndCapture(h->stream, &g);
        if (e == cudaSuccess) e = e2;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&h->graph, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(h, e, "step graph");
      }
      L2D_CUDA(h, cudaGraphLaunch(h->graph, h->stream), "graph launch");
      left -= l2d::GRAPH_STEPS;
      h->steps += l2d::GRAPH_STEPS;
      continue;
    }
    L2D_CUDA(h, step(h, h->par), "stage launch");
    h->par ^= 1;
    left--;
    h->steps++;
  }
  return wait(h);
}

int fz_l2d_run_timed(fz_l2d* h, int64_t nsteps, double* ms) {
  if (!h || !ms || nsteps < 0) return FZ_EINVAL;
  cudaSetDevice(h->dev);
  cudaEvent_t a = nullptr, b = nullptr;
  L2D_CUDA(h, cudaEventCreate(&a), "event");
  cudaError_t e = cudaEventCreate(&b);
  if (e != cudaSuccess) {
    cudaEventDestroy(a);
    return cuda_fail(h, e, "event");
  }
  e = cudaEventRecord(a, h->stream);
  int rc = e == cudaSuccess ? fz_l2d_run(h, nsteps) : cuda_fail(h, e, "event record");
  if (rc == FZ_OK) {
    e = cudaEventRecord(b, h->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    float x = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&x, a, b);
    if (e == cudaSuccess) *ms = x; else rc = cuda_fail(h, e, "event timing");
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return rc;
}

int64_t fz_l2d_step_count(const fz_l2d* h) { return h ? h->steps : -1; }

int64_t fz_l2d_band_cells(const fz_l2d* h) { return h ? h->nB : -1; }

int64_t fz_l2d_samples(const fz_l2d* h) { return h ? std::min(h->nsamples, h->steps - h->rec_base) : -1; }

int fz_l2d_get_ir(fz_l2d* h, double* out, int64_t n) {
  if (!h || !out || n < 0) return FZ_EINVAL;
  if (n > fz_l2d_samples(h)) return fail(h, FZ_EINVAL, "fz_l2d_get_ir: more samples asked for than recorded");
  if (n == 0) return FZ_OK;
  cudaSetDevice(h->dev);
  const int rc = wait(h);
  if (rc != FZ_OK) return rc;
  L2D_CUDA(h, cudaMemcpy(out, h->d_ir, n * sizeof(double), cudaMemcpyDeviceToHost), "trace D2H");
  return FZ_OK;
}

int fz_l2d_get_fields(fz_l2d* h, double* p, double* u, double* v) {
  if (!h) return FZ_EINVAL;
  cudaSetDevice(h->dev);
  const int rc = wait(h);
  if (rc != FZ_OK) return rc;
  double* out[3] = {p, u, v};
  std::vector<unsigned char> tmp(h->N * rsize(h));
  for (int f = 0; f < 3; f++) {
    if (!out[f]) continue;
    L2D_CUDA(h, cudaMemcpy(tmp.data(), h->buf[h->par][f], tmp.size(), cudaMemcpyDeviceToHost), "fields D2H");
    for (size_t q = 0; q < h->N; q++)
      out[f][q] = h->fp64 ? ((const double*)tmp.data())[q] : (double)((const float*)tmp.data())[q];
  }
  return FZ_OK;
}

int fz_l2d_last_error(const fz_l2d* h, char* buf, size_t cap) {
  if (!h || !buf || cap == 0) return FZ_EINVAL;
  std::snprintf(buf, cap, "%s", h->err.c_str());
  return FZ_OK;
}

}  // extern "C"
