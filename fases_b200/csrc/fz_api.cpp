// fz_api.cpp -- C ABI of the stepper (include/fz.h): handle lifetime, geometry and band setup,
// materials, sources, receivers, the step loop with CUDA graphs, bounded waits and readback.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "fz_internal.h"
#include "fz_kernels.h"

using fz::XOFF;
using fz::GHOST;

namespace {
thread_local std::string g_err;
}

namespace fzi {
int set_error(fz_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  g_err = msg;
  return code;
}
int set_global_error(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
int cuda_fail(fz_handle* h, cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  return set_error(h, (e == cudaErrorMemoryAllocation) ? FZ_ENOMEM : FZ_ECUDA, m);
}
}  // namespace fzi

using fzi::cuda_fail;
using fzi::set_error;

#define FZ_CUDA(h, call, what)                       \
  do {                                               \
    cudaError_t e__ = (call);                        \
    if (e__ != cudaSuccess) return cuda_fail(h, e__, what); \
  } while (0)

namespace {

template <class T>
void dfree(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

int64_t dev_index(const fz_handle* h, int i, int j, int k) {
  return (int64_t)XOFF + i + h->Sx * ((int64_t)j + (int64_t)h->Ny * k);
}

int64_t ref_index(const fz_handle* h, int i, int j, int k) {
  return (int64_t)i + (int64_t)h->Nx * ((int64_t)j + (int64_t)h->Ny * k);
}

void free_graphs(fz_handle* h) {
  h->launch_gen++;
  for (auto& g : h->graph) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
}

void free_device(fz_handle* h) {
  free_graphs(h);
  for (auto& set : h->U)
    for (auto& f : set) dfree(f);
  dfree(h->d_cls);
  for (auto& p : h->d_pml_coef) dfree(p);
  for (auto& p : h->d_psi) dfree(p);
  dfree(h->d_brec);
  dfree(h->d_bgeo);
  dfree(h->d_bnrm);
  for (auto& set : h->d_ade)
    for (auto& p : set) dfree(p);
  dfree(h->d_mat);
  dfree(h->d_src_cell);
  dfree(h->d_src_coef);
  dfree(h->d_src_freq);
  dfree(h->d_us);
  dfree(h->d_rec_cell);
  dfree(h->d_ir);
  dfree(h->d_vel);
  dfree(h->d_slices);
  h->sl_on = false;
}

// cuTensorMapEncodeTiled, fetched from the driver at run time (no link-time libcuda dependency).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

// 3-D map over one device array (Sx x Ny x Nz*nb elements of esz bytes) with bx x by x 1 boxes;
// reads outside the allocation fill with zeros.
int make_map(fz_handle* h, CUtensorMap* map, void* base, size_t esz, CUtensorMapDataType type, int bx, int by) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return set_error(h, FZ_ECUDA, "cuTensorMapEncodeTiled not available from the driver");
  const cuuint64_t dims[3] = {(cuuint64_t)h->Sx, (cuuint64_t)h->Ny, (cuuint64_t)h->Nz * h->nb};
  const cuuint64_t strides[2] = {(cuuint64_t)h->Sx * esz, (cuuint64_t)h->plane * esz};
  const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = enc(map, type, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(h, FZ_ECUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return FZ_OK;
}

int make_field_maps(fz_handle* h) {
  const CUtensorMapDataType t = h->fp64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  for (int s = 0; s < 3; s++) {
    for (int f = 0; f < 3; f++) {
      int rc = make_map(h, &h->halo_map[s][f], h->U[s][f], h->rsize, t, fz::PW, fz::PH);
      if (rc != FZ_OK) return rc;
    }
    for (int f = 0; f < 4; f++) {
      int rc = make_map(h, &h->own_map[s][f], h->U[s][f], h->rsize, t, fz::TX, fz::TY);
      if (rc != FZ_OK) return rc;
    }
  }
  return make_map(h, &h->cls_map, h->d_cls, 1, CU_TENSOR_MAP_DATA_TYPE_UINT8, fz::TX, fz::TY);
}

// Per-axis cPML coefficient table, restated from functions3D.cuh:689-723 (evaluated once here in
// FP64 instead of powf/expf/logf per cell and stage), with the profile constants taken from
// fz_params. The entries are carried as values with their derivatives with respect to
// (pml_R0, pml_kappa_max, pml_alpha_max), which the adjoint uses for the cPML gradient.
struct D3 {
  double v, g[3];
};
D3 dconst(double v) { return D3{v, {0.0, 0.0, 0.0}}; }
D3 operator+(D3 a, D3 b) { return D3{a.v + b.v, {a.g[0] + b.g[0], a.g[1] + b.g[1], a.g[2] + b.g[2]}}; }
D3 operator-(D3 a, D3 b) { return D3{a.v - b.v, {a.g[0] - b.g[0], a.g[1] - b.g[1], a.g[2] - b.g[2]}}; }
D3 operator*(D3 a, D3 b) {
  D3 r{a.v * b.v, {}};
  for (int q = 0; q < 3; q++) r.g[q] = a.g[q] * b.v + a.v * b.g[q];
  return r;
}
D3 operator/(D3 a, D3 b) {
  D3 r{a.v / b.v, {}};
  for (int q = 0; q < 3; q++) r.g[q] = (a.g[q] * b.v - a.v * b.g[q]) / (b.v * b.v);
  return r;
}
D3 dexp(D3 a) {
  D3 r{std::exp(a.v), {}};
  for (int q = 0; q < 3; q++) r.g[q] = r.v * a.g[q];
  return r;
}
}  // namespace

namespace fzi {
void pml_entry(const fz_params& p, int N, int lo, int hi, int i, PmlEntry* out) {
  const int d = p.pml_cells, ng = GHOST;
  const double m = p.pml_order;
  // pref = (m+1) c ln(1/R0) / (2 d h); d pref / d R0 = -(m+1) c / (2 d h R0)
  const D3 pref{0.5 * p.c * (m + 1.0) * std::log(1.0 / p.pml_R0) / ((double)d * p.h),
                {-0.5 * p.c * (m + 1.0) / ((double)d * p.h * p.pml_R0), 0.0, 0.0}};
  const D3 kappa_max{p.pml_kappa_max, {0.0, 1.0, 0.0}};
  const D3 alpha_max{p.pml_alpha_max, {0.0, 0.0, 1.0}};
  const D3 alpha_min = dconst(0.1) * alpha_max;
  const double xm = std::min(1.0, std::max(0.0, ((double)(ng + d) - i) / d));
  const double xp = std::min(1.0, std::max(0.0, (i - ((double)(N - 1 - ng) - d)) / d));
  const D3 sig = dconst(lo) * pref * dconst(std::pow(xm, m)) + dconst(hi) * pref * dconst(std::pow(xp, m));
  const double dep = lo * xm + hi * xp;
  const D3 kap = dconst(1.0) + (kappa_max - dconst(1.0)) * dconst(std::pow(dep, m));
  const D3 alp = alpha_min + (alpha_max - alpha_min) * dconst(1.0 - dep);
  const bool in = (lo && i >= ng && i < ng + d) || (hi && i >= N - ng - d && i <= N - 1 - ng);
  out->tile = in ? ((i < ng + d) ? (i - ng) : (i - (N - ng - d) + d)) : -1;
  const D3 kinv1 = dconst(1.0) / kap - dconst(1.0);
  const D3 b = dexp(dconst(0.0) - (alp + sig / kap) * dconst(p.dt));
  const D3 ca = (sig.v > 0.0) ? (sig / (kap * (sig + kap * alp))) * (b - dconst(1.0)) : dconst(0.0);
  const D3* e[3] = {&kinv1, &b, &ca};
  for (int q = 0; q < 3; q++) {
    out->v[q] = e[q]->v;
    for (int r = 0; r < 3; r++) out->d[q][r] = e[q]->g[r];
  }
}
}  // namespace fzi

namespace {

template <class R>
std::vector<fz::PmlCoef<R>> pml_table(int N, int lo, int hi, const fz_params& p) {
  std::vector<fz::PmlCoef<R>> t((size_t)N);
  for (int i = 0; i < N; i++) {
    fzi::PmlEntry e;
    fzi::pml_entry(p, N, lo, hi, i, &e);
    fz::PmlCoef<R> c;
    c.tile = e.tile;
    c.kinv1 = (R)e.v[0];
    c.b = (R)e.v[1];
    c.ca = (R)e.v[2];
    t[(size_t)i] = c;
  }
  return t;
}

template <class R>
int upload_pml(fz_handle* h) {
  const fz_params& p = h->prm;
  // axis x: L (lo) / R (hi); y: B (lo) / F (hi); z: D (lo) / U (hi)
  const int lo[3] = {p.pml[3] != 0, p.pml[5] != 0, p.pml[1] != 0};
  const int hi[3] = {p.pml[2] != 0, p.pml[4] != 0, p.pml[0] != 0};
  const int n[3] = {h->Nx, h->Ny, h->Nz};
  typedef typename fz::Pair<R>::T P;
  const int64_t d2 = 2 * (int64_t)p.pml_cells;
  const int64_t nb = h->nb;
  const int64_t tile_n[3] = {d2 * h->Ny * h->Nz * nb, (int64_t)h->Nx * d2 * h->Nz * nb,
                             (int64_t)h->Nx * h->Ny * d2 * nb};
  for (int a = 0; a < 3; a++) {
    auto t = pml_table<R>(n[a], lo[a], hi[a], p);
    if (a == 2 && nb > 1) {
      // batch members stack along z: one z table per member, its psi tiles offset by the member
      const size_t n1 = t.size();
      t.resize(n1 * (size_t)nb);
      for (int64_t m = 1; m < nb; m++)
        for (size_t q = 0; q < n1; q++) {
          fz::PmlCoef<R> c = t[q];
          if (c.tile >= 0) c.tile += (int32_t)(m * d2);
          t[(size_t)m * n1 + q] = c;
        }
    }
    FZ_CUDA(h, cudaMalloc(&h->d_pml_coef[a], t.size() * sizeof(t[0])), "cudaMalloc(pml table)");
    FZ_CUDA(h, cudaMemcpy(h->d_pml_coef[a], t.data(), t.size() * sizeof(t[0]), cudaMemcpyHostToDevice),
            "cudaMemcpy(pml table)");
    if (lo[a] || hi[a]) {
      FZ_CUDA(h, cudaMalloc(&h->d_psi[a], (size_t)tile_n[a] * sizeof(P)), "cudaMalloc(psi)");
      FZ_CUDA(h, cudaMemset(h->d_psi[a], 0, (size_t)tile_n[a] * sizeof(P)), "cudaMemset(psi)");
    }
  }
  return FZ_OK;
}

// Immersed band list (functions3D.cuh:462-512 evaluated once per cell instead of per stage).
// Band cells: interior cells [3, N-3)^3 with oid not in {0, 0xFF} (the BC kernel's condition,
// functions3D.cuh:464-478, with bmap >= 0 <=> oid not in {0, 0xFF}, common/filterABC.h:99-105).
template <class R>
int build_band(fz_handle* h) {
  const int Nx = h->Nx, Ny = h->Ny, Nz = h->Nz;
  const double hh = h->prm.h, tol = h->prm.tol_cells * h->prm.h;
  const float* S = h->S_host.data();
  const uint8_t* oid = h->oid_host.data();
  std::vector<int64_t> cell, corner;
  std::vector<R> geo, nrm;
  std::vector<int32_t> mat;
  h->band_cell_ref.clear();
  auto Sat = [&](int i, int j, int k) { return (double)S[ref_index(h, i, j, k)]; };
  // one list per z plane, built in parallel and joined in plane order (the build_boundary_map
  // order of common/filterABC.h:95-108)
  struct Plane {
    std::vector<int64_t> cell, corner, ref;
    std::vector<R> geo, nrm;
    std::vector<int32_t> mat;
  };
  std::vector<Plane> planes((size_t)Nz);
#pragma omp parallel for schedule(dynamic, 1)
  for (int k = GHOST; k < Nz - GHOST; k++) {
    Plane& P = planes[(size_t)k];
    for (int j = GHOST; j < Ny - GHOST; j++)
      for (int i = GHOST; i < Nx - GHOST; i++) {
        const int64_t rc = ref_index(h, i, j, k);
        const uint8_t o = oid[rc];
        if (o == 0 || o == 0xFF) continue;
        const double s = S[rc];
        const double gx = (Sat(i + 1, j, k) - Sat(i - 1, j, k)) * (0.5 / hh);
        const double gy = (Sat(i, j + 1, k) - Sat(i, j - 1, k)) * (0.5 / hh);
        const double gz = (Sat(i, j, k + 1) - Sat(i, j, k - 1)) * (0.5 / hh);
        const double gn = std::max(std::sqrt(gx * gx + gy * gy + gz * gz), 1e-12);
        const double nx = -gx / gn, ny = -gy / gn, nz = -gz / gn;
        const double Cx = (i + 0.5) * hh, Cy = (j + 0.5) * hh, Cz = (k + 0.5) * hh;
        const double Wx = Cx + s * nx, Wy = Cy + s * ny, Wz = Cz + s * nz;
        const double l = s + 2.0 * hh;
        const double Dx = Wx - l * nx, Dy = Wy - l * ny, Dz = Wz - l * nz;
        const double fx = Dx / hh - 0.5, fy = Dy / hh - 0.5, fzz = Dz / hh - 0.5;
        int bi = (int)std::floor(fx), bj = (int)std::floor(fy), bk = (int)std::floor(fzz);
        bi = std::max(0, std::min(bi, Nx - 2));
        bj = std::max(0, std::min(bj, Ny - 2));
        bk = std::max(0, std::min(bk, Nz - 2));
        double chi;
        if (s >= tol) chi = 0.0;
        else if (s <= hh) chi = 1.0;
        else {
          const double r = (s - hh) / (tol - hh);
          chi = 1.0 - r * r * (3.0 - 2.0 * r);
        }
        P.cell.push_back(dev_index(h, i, j, k));
        P.corner.push_back(dev_index(h, bi, bj, bk));
        P.geo.push_back((R)(fx - bi));
        P.geo.push_back((R)(fy - bj));
        P.geo.push_back((R)(fzz - bk));
        P.geo.push_back((R)chi);
        P.nrm.push_back((R)nx);
        P.nrm.push_back((R)ny);
        P.nrm.push_back((R)nz);
        P.nrm.push_back((R)0);
        P.mat.push_back((int32_t)o - 1);
        P.ref.push_back(rc);
      }
  }
  for (const Plane& P : planes) {
    cell.insert(cell.end(), P.cell.begin(), P.cell.end());
    corner.insert(corner.end(), P.corner.begin(), P.corner.end());
    geo.insert(geo.end(), P.geo.begin(), P.geo.end());
    nrm.insert(nrm.end(), P.nrm.begin(), P.nrm.end());
    mat.insert(mat.end(), P.mat.begin(), P.mat.end());
    h->band_cell_ref.insert(h->band_cell_ref.end(), P.ref.begin(), P.ref.end());
  }
  h->nB1 = (int64_t)cell.size();
  h->nB = h->nB1 * h->nb;
  h->band_mat = mat;
  if (h->nB == 0) return FZ_OK;
  // batch members: the same band cells in every member's field set (and their own ADE states)
  for (int m = 1; m < h->nb; m++)
    for (int64_t b = 0; b < h->nB1; b++) {
      cell.push_back(cell[(size_t)b] + (int64_t)m * h->ncell_dev);
      corner.push_back(corner[(size_t)b] + (int64_t)m * h->ncell_dev);
      for (int q = 0; q < 4; q++) {
        geo.push_back(geo[(size_t)(4 * b + q)]);
        nrm.push_back(nrm[(size_t)(4 * b + q)]);
      }
      mat.push_back(mat[(size_t)b]);
    }
  for (int64_t c : cell) h->cls_host[(size_t)c] |= fz::CLS_BAND;
  FZ_CUDA(h, cudaMemcpy(h->d_cls, h->cls_host.data(), h->cls_host.size(), cudaMemcpyHostToDevice), "cls H2D");
  std::vector<int4> rec((size_t)h->nB);
  for (size_t b = 0; b < rec.size(); b++) {
    const uint64_t c = (uint64_t)cell[b];
    rec[b].x = (int)(uint32_t)(c & 0xffffffffu);
    rec[b].y = (int)(uint32_t)(c >> 32);
    rec[b].z = (int)(corner[b] - cell[b]);  // within a few rows and planes: fits 32 bits
    rec[b].w = mat[b];
  }
  FZ_CUDA(h, cudaMalloc(&h->d_brec, rec.size() * sizeof(int4)), "cudaMalloc(band)");
  FZ_CUDA(h, cudaMalloc(&h->d_bgeo, geo.size() * sizeof(R)), "cudaMalloc(band)");
  FZ_CUDA(h, cudaMalloc(&h->d_bnrm, nrm.size() * sizeof(R)), "cudaMalloc(band)");
  FZ_CUDA(h, cudaMemcpy(h->d_brec, rec.data(), rec.size() * sizeof(int4), cudaMemcpyHostToDevice), "band H2D");
  FZ_CUDA(h, cudaMemcpy(h->d_bgeo, geo.data(), geo.size() * sizeof(R), cudaMemcpyHostToDevice), "band H2D");
  FZ_CUDA(h, cudaMemcpy(h->d_bnrm, nrm.data(), nrm.size() * sizeof(R), cudaMemcpyHostToDevice), "band H2D");
  return FZ_OK;
}

template <class R>
int finalize(fz_handle* h) {
  if (h->finalized) return FZ_OK;
  if (!h->have_geometry) return set_error(h, FZ_ESTATE, "fz_run before fz_load_geometry_raw");
  // materials: every band cell must name a loaded material (the reference indexes R_inf[oid-1]
  // without a check, main3D.cu:579 + functions3D.cuh:525)
  for (size_t b = 0; b < h->band_mat.size(); b++)
    if (h->band_mat[b] >= h->nMat)
      return set_error(h, FZ_EINVAL,
                       "band cell " + std::to_string(h->band_cell_ref[b]) + " has material id " +
                           std::to_string(h->band_mat[b] + 1) + " but only " + std::to_string(h->nMat) +
                           " materials are set");
  const int nm = std::max(1, h->nMat);
  if (h->Rinf.empty()) {
    h->K = 1;
    h->L = 1;
    h->Rinf.assign(nm, 0.0);
    h->A.assign(nm, 0.0); h->zeta.assign(nm, 0.0);
    h->B.assign(nm, 0.0); h->C.assign(nm, 0.0); h->alpha.assign(nm, 0.0); h->beta.assign(nm, 0.0);
  }
  std::vector<double> packed;
  for (auto* v : {&h->Rinf, &h->A, &h->zeta, &h->B, &h->C, &h->alpha, &h->beta})
    packed.insert(packed.end(), v->begin(), v->end());
  FZ_CUDA(h, cudaMalloc(&h->d_mat, packed.size() * 8), "cudaMalloc(materials)");
  FZ_CUDA(h, cudaMemcpy(h->d_mat, packed.data(), packed.size() * 8, cudaMemcpyHostToDevice), "materials H2D");
  // ADE states (3 rotating sets, main3D.cu:683-709), zeroed
  if (h->nB > 0) {
    const size_t nk = (size_t)h->nB * h->K, nl = (size_t)h->nB * h->L;
    for (int s = 0; s < 3; s++) {
      FZ_CUDA(h, cudaMalloc(&h->d_ade[s][0], nk * 8), "cudaMalloc(ADE)");
      FZ_CUDA(h, cudaMalloc(&h->d_ade[s][1], nl * 8), "cudaMalloc(ADE)");
      FZ_CUDA(h, cudaMalloc(&h->d_ade[s][2], nl * 8), "cudaMalloc(ADE)");
      FZ_CUDA(h, cudaMemset(h->d_ade[s][0], 0, nk * 8), "cudaMemset(ADE)");
      FZ_CUDA(h, cudaMemset(h->d_ade[s][1], 0, nl * 8), "cudaMemset(ADE)");
      FZ_CUDA(h, cudaMemset(h->d_ade[s][2], 0, nl * 8), "cudaMemset(ADE)");
    }
  }
  // sources
  h->nsrc_dev = 0;
  if (h->nsrc > 0) {
    std::vector<int64_t> cells;
    std::vector<R> coef, freq;
    const double As = 6.0 * h->prm.h * h->prm.h;
    for (int s = 0; s < h->nsrc; s++) {
      const int i = h->src_ijk[3 * s], j = h->src_ijk[3 * s + 1], k = h->src_ijk[3 * s + 2];
      const int mem = h->src_member.empty() ? -1 : h->src_member[s];
      for (int m = 0; m < h->nb; m++) {
        if (mem >= 0 && mem != m) continue;
        const int64_t g = dev_index(h, i, j, k) + (int64_t)m * h->ncell_dev;
        cells.push_back(g);
        coef.push_back((R)(h->prm.dt * h->prm.c * h->prm.c * h->src_val[s] * h->prm.rho * As /
                           (h->prm.h * h->prm.h * h->prm.h)));
        freq.push_back((R)(h->src_freq.empty() ? 0.0 : h->src_freq[s]));
        h->cls_host[g] |= fz::CLS_SOURCE;
      }
    }
    h->nsrc_dev = (int)cells.size();
    FZ_CUDA(h, cudaMalloc(&h->d_src_cell, cells.size() * 8), "cudaMalloc(src)");
    FZ_CUDA(h, cudaMalloc(&h->d_src_coef, coef.size() * sizeof(R)), "cudaMalloc(src)");
    FZ_CUDA(h, cudaMalloc(&h->d_src_freq, freq.size() * sizeof(R)), "cudaMalloc(src)");
    FZ_CUDA(h, cudaMemcpy(h->d_src_cell, cells.data(), cells.size() * 8, cudaMemcpyHostToDevice), "src H2D");
    FZ_CUDA(h, cudaMemcpy(h->d_src_coef, coef.data(), coef.size() * sizeof(R), cudaMemcpyHostToDevice), "src H2D");
    FZ_CUDA(h, cudaMemcpy(h->d_src_freq, freq.data(), freq.size() * sizeof(R), cudaMemcpyHostToDevice), "src H2D");
    if (!h->u_s.empty()) {
      std::vector<R> us(h->u_s.begin(), h->u_s.end());
      h->n_us = (int64_t)us.size();
      FZ_CUDA(h, cudaMalloc(&h->d_us, us.size() * sizeof(R)), "cudaMalloc(u_s)");
      FZ_CUDA(h, cudaMemcpy(h->d_us, us.data(), us.size() * sizeof(R), cudaMemcpyHostToDevice), "u_s H2D");
    }
    FZ_CUDA(h, cudaMemcpy(h->d_cls, h->cls_host.data(), h->cls_host.size(), cudaMemcpyHostToDevice), "cls H2D");
  }
  // receivers
  if (h->nrec > 0) {
    std::vector<int64_t> cells;
    for (int m = 0; m < h->nb; m++)  // traces [member][receiver][step]
      for (int r = 0; r < h->nrec; r++)
        cells.push_back(dev_index(h, h->rec_ijk[3 * r], h->rec_ijk[3 * r + 1], h->rec_ijk[3 * r + 2]) +
                        (int64_t)m * h->ncell_dev);
    FZ_CUDA(h, cudaMalloc(&h->d_rec_cell, cells.size() * 8), "cudaMalloc(rec)");
    FZ_CUDA(h, cudaMemcpy(h->d_rec_cell, cells.data(), cells.size() * 8, cudaMemcpyHostToDevice), "rec H2D");
    const size_t n = (size_t)h->nrec * h->nb * (size_t)std::max<int64_t>(1, h->rec_cap);
    FZ_CUDA(h, cudaMalloc(&h->d_ir, n * 8), "cudaMalloc(ir)");
    FZ_CUDA(h, cudaMalloc(&h->d_vel, n * 3 * 8), "cudaMalloc(vel)");
    FZ_CUDA(h, cudaMemset(h->d_ir, 0, n * 8), "cudaMemset(ir)");
    FZ_CUDA(h, cudaMemset(h->d_vel, 0, n * 3 * 8), "cudaMemset(vel)");
  }
  // launch geometry: z chunks so that the grid fills the GPU several times over
  int occ = 1;
  FZ_CUDA(h, fz::stage_occupancy<R>(&occ), "occupancy");
  occ = std::max(1, occ);
  h->stage_occ = occ;
  const int ntx = (h->Nx - 2 * GHOST + fz::TX - 1) / fz::TX;
  const int nty = (h->Ny - 2 * GHOST + fz::TY - 1) / fz::TY;
  const int nzi = h->Nz - 2 * GHOST;
  const int64_t slots = (int64_t)h->nsm * occ;
  // Pick the z-chunk count that best fills whole waves of CTA slots, charging each chunk about
  // 1.5 planes of start-up work (two extra z centres and the TMA ring fill).
  int best = 1;
  double best_eff = -1.0;
  for (int nk = 1; nk <= std::max(1, nzi / 8); nk++) {
    const int chunk = (nzi + nk - 1) / nk;
    const int nk_eff = (nzi + chunk - 1) / chunk;
    const int64_t items = (int64_t)ntx * nty * nk_eff * h->nb;
    const int64_t waves = (items + slots - 1) / slots;
    const double eff = ((double)items / (double)(waves * slots)) * ((double)chunk / (chunk + 1.5));
    if (eff > best_eff + 1e-9) {
      best_eff = eff;
      best = nk;
    }
  }
  h->kz_heuristic = (nzi + best - 1) / best;
  h->finalized = true;
  fzi::set_kz_chunk(h, h->kz_chunk > 0 ? h->kz_chunk : 0);
  return FZ_OK;
}

template <class R>
fz::StageArgs<R> stage_args(fz_handle* h, int stage) {
  typedef typename fz::Pair<R>::T P;
  fz::StageArgs<R> a;
  std::memset(&a, 0, sizeof(a));
  R* const* u0 = (R* const*)h->U[h->i0];
  R* const* u1 = (R* const*)h->U[h->i1];
  R* const* u2 = (R* const*)h->U[h->i2];
  R* const* in = (stage == 0) ? u0 : (stage == 1) ? u1 : u2;
  R* const* out = (stage == 1) ? u2 : u1;
  a.pi = in[0]; a.ui = in[1]; a.vi = in[2]; a.wi = in[3];
  a.pb = u0[0]; a.ub = u0[1]; a.vb = u0[2]; a.wb = u0[3];
  a.po = out[0]; a.uo = out[1]; a.vo = out[2]; a.wo = out[3];
  a.cls = h->d_cls;
  a.Nx = h->Nx; a.Ny = h->Ny; a.Nz = h->Nz;
  a.Sx = h->Sx; a.plane = h->plane;
  a.kz_chunk = h->kz_chunk;
  a.zchunks = h->zchunks;
  a.zoff[0] = 0;
  for (int c = 0; c < h->zchunks && c < fz::FZ_MAX_ZCHUNKS; c++) a.zoff[c + 1] = a.zoff[c] + h->zsizes[(size_t)c];
  const fz_params& p = h->prm;
  a.dt_h = (R)(p.dt / p.h);
  a.frc2 = (R)(0.5 * p.rho * p.c * p.c);
  a.firho = (R)(0.5 / p.rho);
  a.fc = (R)(0.5 * p.c);
  a.inv_h = (R)(1.0 / p.h);
  const double w = (stage == 0) ? 1.0 : (stage == 1) ? 0.25 : 2.0 / 3.0;
  a.wdt = (R)(w * p.dt);
  a.pml_on = h->pml_on ? 1 : 0;
  a.pml_d2 = 2 * p.pml_cells;
  a.pcx = (const fz::PmlCoef<R>*)h->d_pml_coef[0];
  a.pcy = (const fz::PmlCoef<R>*)h->d_pml_coef[1];
  a.pcz = (const fz::PmlCoef<R>*)h->d_pml_coef[2];
  a.psix = (P*)h->d_psi[0];
  a.psiy = (P*)h->d_psi[1];
  a.psiz = (P*)h->d_psi[2];
  a.nsrc = h->nsrc_dev;
  a.src_cell = h->d_src_cell;
  a.src_coef = (const R*)h->d_src_coef;
  a.src_freq = (const R*)h->d_src_freq;
  a.u_s = (const R*)h->d_us;
  a.n_us = h->n_us;
  a.src_opt = h->src_opt;
  a.src_w = (R)w;
  a.nn_mul = 2;
  a.nn_add = (stage == 0) ? 0 : (stage == 1) ? 2 : 1;  // main3D.cu:1288, 1296, 1304
  a.half_dt = (R)(0.5 * p.dt);
  a.step = h->d_step;
  a.err = h->d_err;
  a.nfield = h->ncell_dev * h->nb;
  {
    const int64_t d2 = 2 * (int64_t)p.pml_cells;
    a.npsi[0] = h->d_psi[0] ? d2 * h->Ny * h->Nz * h->nb : 0;
    a.npsi[1] = h->d_psi[1] ? (int64_t)h->Nx * d2 * h->Nz * h->nb : 0;
    a.npsi[2] = h->d_psi[2] ? (int64_t)h->Nx * h->Ny * d2 * h->nb : 0;
    a.npc[0] = h->Nx;
    a.npc[1] = h->Ny;
    a.npc[2] = (int64_t)h->Nz * h->nb;
  }
  a.test_skip_plane = h->test_skip_plane;
  return a;
}

template <class R>
fz::BandArgs<R> band_args(fz_handle* h, int stage) {
  fz::BandArgs<R> b;
  std::memset(&b, 0, sizeof(b));
  R* const* u0 = (R* const*)h->U[h->i0];
  R* const* u1 = (R* const*)h->U[h->i1];
  R* const* u2 = (R* const*)h->U[h->i2];
  R* const* in = (stage == 0) ? u0 : (stage == 1) ? u1 : u2;
  R* const* out = (stage == 1) ? u2 : u1;
  b.nB = h->nB;
  b.rec = h->d_brec;
  b.geo = (const R*)h->d_bgeo; b.nrm = (const R*)h->d_bnrm;
  b.pi = in[0]; b.ui = in[1]; b.vi = in[2]; b.wi = in[3];
  b.po = out[0]; b.uo = out[1]; b.vo = out[2]; b.wo = out[3];
  b.Sx = h->Sx; b.plane = h->plane;
  b.err = h->d_err;
  b.nfield = h->ncell_dev * h->nb;
  b.Z0 = h->prm.rho * h->prm.c;
  b.dt = h->prm.dt;
  // ADE state roles (left, middle, right) of the stage, main3D.cu:1290-1306
  int L_, M_, R_;
  if (stage == 0) { L_ = h->ph_cur; M_ = h->ph_old; R_ = h->ph_old; }
  else if (stage == 1) { L_ = h->ph_nu; M_ = h->ph_old; R_ = h->ph_cur; }
  else { L_ = h->ph_cur; M_ = h->ph_old; R_ = h->ph_nu; }
  b.phL = h->d_ade[L_][0]; b.phM = h->d_ade[M_][0]; b.phR = h->d_ade[R_][0];
  b.s1L = h->d_ade[L_][1]; b.s1M = h->d_ade[M_][1]; b.s1R = h->d_ade[R_][1];
  b.s2L = h->d_ade[L_][2]; b.s2M = h->d_ade[M_][2]; b.s2R = h->d_ade[R_][2];
  b.K = h->K; b.L = h->L;
  const int nm = std::max(1, h->nMat);
  const double* m = h->d_mat;
  b.Rinf = m; m += nm;
  b.A = m; m += (size_t)nm * h->K;
  b.zeta = m; m += (size_t)nm * h->K;
  b.B = m; m += (size_t)nm * h->L;
  b.C = m; m += (size_t)nm * h->L;
  b.alpha = m; m += (size_t)nm * h->L;
  b.beta = m;
  return b;
}

struct Timer {
  fz_handle* h;
  int kind;
  cudaEvent_t a = nullptr, b = nullptr;
  Timer(fz_handle* h_, int k) : h(h_), kind(k) {
    if (!h->profiling) return;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, h->stream);
  }
  ~Timer() {
    if (!h->profiling) return;
    cudaEventRecord(b, h->stream);
    h->timings.push_back({kind, a, b});
  }
};

template <class R>
cudaError_t enqueue_stage_kernel(fz_handle* h, int st) {
  const int in_set = (st == 0) ? h->i0 : (st == 1) ? h->i1 : h->i2;
  fz::StageMaps m;
  m.p = h->halo_map[in_set][0];
  m.u = h->halo_map[in_set][1];
  m.v = h->halo_map[in_set][2];
  m.bp = h->own_map[h->i0][0];
  m.bu = h->own_map[h->i0][1];
  m.bv = h->own_map[h->i0][2];
  m.bw = h->own_map[h->i0][3];
  m.cls = h->cls_map;
  return fz::launch_stage<R>(st, h->prm.two_d != 0, stage_args<R>(h, st), m, h->stage_grid, h->stream);
}

// Stage st of the current step: the stage kernel, then the immersed band (main3D.cu:1286-1306).
template <class R>
cudaError_t enqueue_stage(fz_handle* h, int st) {
  cudaError_t e;
  {
    Timer t(h, st);
    e = enqueue_stage_kernel<R>(h, st);
    if (e != cudaSuccess) return e;
  }
  if (h->nB > 0) {
    Timer t(h, 3);
    e = fz::launch_band<R>(st, band_args<R>(h, st), h->stream);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// End of a step: receiver gather, device step counter, buffer rotation (main3D.cu:1312-1319,
// 1399-1414).
template <class R>
cudaError_t enqueue_finish(fz_handle* h) {
  cudaError_t e;
  {
    Timer t(h, 4);
    R* const* u1 = (R* const*)h->U[h->i1];
    e = fz::launch_receivers<R>(u1[0], u1[1], u1[2], u1[3], h->d_rec_cell, h->nrec * h->nb, h->d_ir, h->d_vel,
                                h->rec_cap, h->d_step, h->d_err, h->ncell_dev * h->nb, h->stream);
    if (e != cudaSuccess) return e;
    if (h->sl_on) {
      e = fz::launch_slices<R>(u1[0], u1[1], u1[2], u1[3], h->Nx, h->Ny, h->Nz, h->Sx, h->sl_i, h->sl_j, h->sl_k,
                               h->d_step, h->sl_step, h->sl_cap, h->d_slices, h->nsm, h->stream);
      if (e != cudaSuccess) return e;
    }
  }
  std::swap(h->i0, h->i1);
  std::swap(h->ph_old, h->ph_cur);
  return cudaSuccess;
}

// One time step (main3D.cu:1280-1319 + receivers 1399-1414).
template <class R>
cudaError_t enqueue_step(fz_handle* h) {
  for (int st = 0; st < 3; st++) {
    const cudaError_t e = enqueue_stage<R>(h, st);
    if (e != cudaSuccess) return e;
  }
  return enqueue_finish<R>(h);
}

// Captures and instantiates the graph of G steps for the current buffer parity (h->i0), unless it
// exists. Capture advances the host-side rotation by G (even) steps: back where it started.
template <class R>
int ensure_graph(fz_handle* h) {
  const int G = h->graph_steps;
  const int par = h->i0;  // buffer assignment repeats every 2 steps
  if (h->graph[par]) return FZ_OK;
  cudaGraph_t g = nullptr;
  FZ_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
  cudaError_t e = cudaSuccess;
  for (int s = 0; s < G && e == cudaSuccess; s++) e = enqueue_step<R>(h);
  cudaError_t e2 = cudaStreamEndCapture(h->stream, &g);
  if (e != cudaSuccess) return cuda_fail(h, e, "capture step");
  if (e2 != cudaSuccess) return cuda_fail(h, e2, "end capture");
  e = cudaGraphInstantiate(&h->graph[par], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_fail(h, e, "graph instantiate");
  FZ_CUDA(h, cudaGraphUpload(h->graph[par], h->stream), "graph upload");
  return FZ_OK;
}

bool graphs_on(const fz_handle* h) { return !h->profiling && h->graph_steps > 0 && (h->graph_steps % 2) == 0; }

// Finalises the set-up and instantiates the step graphs of both buffer parities without running
// a step: the parity is flipped on the host only (the field-set and ADE-set roles swap together
// every step) and flipped back.
template <class R>
int prepare_graphs(fz_handle* h) {
  int rc = finalize<R>(h);
  if (rc != FZ_OK || !graphs_on(h)) return rc;
  for (int flip = 0; flip < 2; flip++) {
    rc = ensure_graph<R>(h);
    std::swap(h->i0, h->i1);
    std::swap(h->ph_old, h->ph_cur);
    if (rc != FZ_OK) {
      if (flip == 0) {
        std::swap(h->i0, h->i1);
        std::swap(h->ph_old, h->ph_cur);
      }
      return rc;
    }
  }
  return FZ_OK;
}

template <class R>
int run_steps(fz_handle* h, int64_t nsteps) {
  int rc = finalize<R>(h);
  if (rc != FZ_OK) return rc;
  int64_t done = 0;
  const int G = h->graph_steps;
  if (graphs_on(h)) {
    while (nsteps - done >= G) {
      const int par = h->i0;
      rc = ensure_graph<R>(h);
      if (rc != FZ_OK) return rc;
      FZ_CUDA(h, cudaGraphLaunch(h->graph[par], h->stream), "graph launch");
      done += G;
      h->steps_enqueued += G;
    }
  }
  for (; done < nsteps; done++) {
    cudaError_t e = enqueue_step<R>(h);
    if (e != cudaSuccess) return cuda_fail(h, e, "step launch");
    h->steps_enqueued += 1;
  }
  return FZ_OK;
}

template <class R>
int load_geometry(fz_handle* h, const float* S, const uint8_t* oid, int Nx, int Ny, int Nz) {
  free_device(h);
  h->finalized = false;
  h->kz_chunk = 0;  // a new grid starts from the heuristic tile depth
  h->stage_grid = dim3(0, 0, 0);
  h->Nx = Nx; h->Ny = Ny; h->Nz = Nz;
  h->Sx = ((int64_t)Nx + XOFF + 31) / 32 * 32;
  h->plane = h->Sx * Ny;
  h->ncell_dev = h->plane * Nz;
  h->nb = std::max(1, h->prm.batch);
  if (h->Lx == 0) { h->Lx = Nx * h->prm.h; h->Ly = Ny * h->prm.h; h->Lz = Nz * h->prm.h; }
  const size_t N = (size_t)Nx * Ny * Nz;
  h->S_host.assign(S, S + N);
  h->oid_host.assign(oid, oid + N);
  const size_t bytes = (size_t)h->ncell_dev * h->nb * sizeof(R);
  for (int s = 0; s < 3; s++)
    for (int f = 0; f < 4; f++) {
      FZ_CUDA(h, cudaMalloc(&h->U[s][f], bytes), "cudaMalloc(fields)");
      FZ_CUDA(h, cudaMemset(h->U[s][f], 0, bytes), "cudaMemset(fields)");
    }
  // cell classes: update where the stage kernels would not return early (functions3D.cuh:1091-1097)
  h->cls_host.assign((size_t)h->ncell_dev, 0);
  int64_t nup = 0;
  const float hf = (float)h->prm.h;
#pragma omp parallel for reduction(+ : nup) schedule(static)
  for (int k = GHOST; k < Nz - GHOST; k++)
    for (int j = GHOST; j < Ny - GHOST; j++)
      for (int i = GHOST; i < Nx - GHOST; i++)
        if (!(S[ref_index(h, i, j, k)] < hf)) {
          h->cls_host[(size_t)dev_index(h, i, j, k)] = fz::CLS_UPDATE;
          nup++;
        }
  h->n_update = nup;
  // one copy of the class bytes per batch member, so that the stage kernels index them like the fields
  h->cls_host.resize((size_t)h->ncell_dev * h->nb);
  for (int m = 1; m < h->nb; m++)
    std::copy(h->cls_host.begin(), h->cls_host.begin() + h->ncell_dev, h->cls_host.begin() + m * h->ncell_dev);
  FZ_CUDA(h, cudaMalloc(&h->d_cls, h->cls_host.size()), "cudaMalloc(cls)");
  FZ_CUDA(h, cudaMemcpy(h->d_cls, h->cls_host.data(), h->cls_host.size(), cudaMemcpyHostToDevice), "cls H2D");
  {
    int rc = make_field_maps(h);
    if (rc != FZ_OK) return rc;
  }
  h->pml_on = false;
  for (int f = 0; f < 6; f++) h->pml_on = h->pml_on || (h->prm.pml[f] != 0);
  int rc = upload_pml<R>(h);
  if (rc != FZ_OK) return rc;
  rc = build_band<R>(h);
  if (rc != FZ_OK) return rc;
  h->i0 = 0; h->i1 = 1; h->i2 = 2;
  h->ph_old = 0; h->ph_cur = 1; h->ph_nu = 2;
  FZ_CUDA(h, cudaMemset(h->d_step, 0, sizeof(int64_t)), "reset step");
  h->steps_enqueued = 0;
  h->have_geometry = true;
  return FZ_OK;
}

template <class R>
int get_fields(fz_handle* h, double* p, double* u, double* v, double* w) {
  const size_t rowb = (size_t)h->Nx * sizeof(R);
  const size_t N = (size_t)h->Nx * h->Ny * h->Nz;
  std::vector<R> tmp(N);
  double* outs[4] = {p, u, v, w};
  for (int f = 0; f < 4; f++) {
    if (!outs[f]) continue;
    for (int m = 0; m < h->nb; m++) {
      const R* src = (const R*)h->U[h->i0][f] + XOFF + (size_t)m * h->ncell_dev;
      FZ_CUDA(h, cudaMemcpy2D(tmp.data(), rowb, src, (size_t)h->Sx * sizeof(R), rowb,
                              (size_t)h->Ny * h->Nz, cudaMemcpyDeviceToHost), "fields D2H");
      double* o = outs[f] + (size_t)m * N;
      const R* t = tmp.data();
#pragma omp parallel for schedule(static)
      for (int64_t c = 0; c < (int64_t)N; c++) o[c] = (double)t[c];
    }
  }
  return FZ_OK;
}

template <class R>
int set_fields(fz_handle* h, const double* p, const double* u, const double* v, const double* w) {
  const size_t rowb = (size_t)h->Nx * sizeof(R);
  const size_t N = (size_t)h->Nx * h->Ny * h->Nz;
  std::unique_ptr<R[]> tmp(new (std::nothrow) R[N]);
  if (!tmp) return set_error(h, FZ_ENOMEM, "fz_set_fields: out of host memory");
  const double* ins[4] = {p, u, v, w};
  for (int f = 0; f < 4; f++) {
    if (!ins[f]) {
      FZ_CUDA(h, cudaMemset(h->U[h->i0][f], 0, (size_t)h->ncell_dev * h->nb * sizeof(R)), "fields zero");
      continue;
    }
    for (int m = 0; m < h->nb; m++) {
      R* dst = (R*)h->U[h->i0][f] + XOFF + (size_t)m * h->ncell_dev;
      const double* in = ins[f] + (size_t)m * N;
      R* t = tmp.get();
#pragma omp parallel for schedule(static)
      for (int64_t c = 0; c < (int64_t)N; c++) t[c] = (R)in[c];
      FZ_CUDA(h, cudaMemcpy2D(dst, (size_t)h->Sx * sizeof(R), tmp.get(), rowb, rowb,
                              (size_t)h->Ny * h->Nz, cudaMemcpyHostToDevice), "fields H2D");
    }
  }
  return FZ_OK;
}

template <class R>
int energy(fz_handle* h, double* E) {
  FZ_CUDA(h, cudaMemsetAsync(h->d_scratch, 0, sizeof(double), h->stream), "energy reset");
  R* const* u0 = (R* const*)h->U[h->i0];
  const double rc2 = h->prm.rho * h->prm.c * h->prm.c;
  FZ_CUDA(h, fz::launch_energy<R>(u0[0], u0[1], u0[2], u0[3], h->ncell_dev * h->nb, 1.0 / rc2, h->prm.rho,
                                  h->d_scratch, h->nsm, h->stream), "energy launch");
  int rc = fz_sync(h, 0);
  if (rc != FZ_OK) return rc;
  FZ_CUDA(h, cudaMemcpy(E, h->d_scratch, sizeof(double), cudaMemcpyDeviceToHost), "energy D2H");
  return FZ_OK;
}

bool check_handle(fz_handle* h) { return h != nullptr; }

}  // namespace

namespace fzi {
int prepare(fz_handle* h) {
  cudaSetDevice(h->device);
  return h->fp64 ? finalize<double>(h) : finalize<float>(h);
}
cudaError_t enqueue(fz_handle* h) { return h->fp64 ? enqueue_step<double>(h) : enqueue_step<float>(h); }
cudaError_t enqueue_stage(fz_handle* h, int st) {
  return h->fp64 ? ::enqueue_stage<double>(h, st) : ::enqueue_stage<float>(h, st);
}
int bind_field_set(fz_handle* h, int set, void* const* f) {
  h->launch_gen++;
  const CUtensorMapDataType t = h->fp64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  for (int q = 0; q < 4; q++) h->U[set][q] = f[q];
  for (int q = 0; q < 3; q++) {
    const int rc = make_map(h, &h->halo_map[set][q], h->U[set][q], h->rsize, t, fz::PW, fz::PH);
    if (rc != FZ_OK) return rc;
  }
  for (int q = 0; q < 4; q++) {
    const int rc = make_map(h, &h->own_map[set][q], h->U[set][q], h->rsize, t, fz::TX, fz::TY);
    if (rc != FZ_OK) return rc;
  }
  return FZ_OK;
}
cudaError_t enqueue_stage_kernel(fz_handle* h, int st) {
  return h->fp64 ? ::enqueue_stage_kernel<double>(h, st) : ::enqueue_stage_kernel<float>(h, st);
}
int set_z_sizes(fz_handle* h, const std::vector<int>& sizes) {
  const int nzi = h->Nz - 2 * GHOST;
  int sum = 0;
  for (int c : sizes) {
    if (c < 1) return set_error(h, FZ_EINVAL, "z chunk of fewer than one plane");
    sum += c;
  }
  if (sizes.empty() || (int)sizes.size() > fz::FZ_MAX_ZCHUNKS || sum != nzi)
    return set_error(h, FZ_EINVAL, "z chunks must cover the interior planes in at most " +
                                       std::to_string(fz::FZ_MAX_ZCHUNKS) + " pieces");
  const int ntx = (h->Nx - 2 * GHOST + fz::TX - 1) / fz::TX;
  const int nty = (h->Ny - 2 * GHOST + fz::TY - 1) / fz::TY;
  const dim3 grid((unsigned)ntx, (unsigned)nty, (unsigned)(sizes.size() * h->nb));
  const bool same = sizes == h->zsizes && grid.x == h->stage_grid.x && grid.y == h->stage_grid.y &&
                    grid.z == h->stage_grid.z;
  h->zsizes = sizes;
  h->zchunks = (int)sizes.size();
  h->kz_chunk = *std::max_element(sizes.begin(), sizes.end());
  h->stage_grid = grid;
  if (same) return FZ_OK;
  h->launch_gen++;
  for (auto& g : h->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  return FZ_OK;
}

void set_kz_chunk(fz_handle* h, int kz_chunk) {
  const int nzi = h->Nz - 2 * GHOST;
  int c = std::max(1, std::min(nzi, kz_chunk > 0 ? kz_chunk : h->kz_heuristic));
  c = std::max(c, (nzi + fz::FZ_MAX_ZCHUNKS - 1) / fz::FZ_MAX_ZCHUNKS);
  std::vector<int> sizes;
  for (int z = 0; z < nzi; z += c) sizes.push_back(std::min(c, nzi - z));
  set_z_sizes(h, sizes);
}

std::vector<int> guided_z_sizes(fz_handle* h, int depth) {
  const int nzi = h->Nz - 2 * GHOST;
  const int D = std::max(1, std::min(nzi, depth > 0 ? depth : h->kz_heuristic));
  const int ntx = (h->Nx - 2 * GHOST + fz::TX - 1) / fz::TX;
  const int nty = (h->Ny - 2 * GHOST + fz::TY - 1) / fz::TY;
  const int rows = std::max(1, (h->nsm * h->stage_occ) / std::max(1, ntx * nty));  // chunk rows per wave
  const int d2 = std::max(1, D / 2), d4 = std::max(1, D / 4);
  const int tail2 = rows * d2, tail4 = rows * d4;
  std::vector<int> sizes;
  int left = nzi;
  while (left > tail2 + tail4 && left > D) {
    sizes.push_back(D);
    left -= D;
  }
  while (left > tail4 && left > d2) {
    sizes.push_back(d2);
    left -= d2;
  }
  while (left > 0) {
    const int c = std::min(d4, left);
    sizes.push_back(c);
    left -= c;
  }
  if (sizes.size() > 1 && 2 * sizes.back() < d4) {  // a sliver at the end joins the chunk before it
    const int c = sizes.back();
    sizes.pop_back();
    sizes.back() += c;
  }
  if ((int)sizes.size() > fz::FZ_MAX_ZCHUNKS) {  // too fine: uniform chunks instead
    sizes.clear();
    const int c = std::max(D, (nzi + fz::FZ_MAX_ZCHUNKS - 1) / fz::FZ_MAX_ZCHUNKS);
    for (int z = 0; z < nzi; z += c) sizes.push_back(std::min(c, nzi - z));
  }
  return sizes;
}
cudaError_t enqueue_finish(fz_handle* h) { return h->fp64 ? ::enqueue_finish<double>(h) : ::enqueue_finish<float>(h); }

template <class R>
void stage_desc(fz_handle* h, int st, fz::StageArgs<R>* a, fz::StageMaps* m) {
  const int in_set = (st == 0) ? h->i0 : (st == 1) ? h->i1 : h->i2;
  m->p = h->halo_map[in_set][0];
  m->u = h->halo_map[in_set][1];
  m->v = h->halo_map[in_set][2];
  m->bp = h->own_map[h->i0][0];
  m->bu = h->own_map[h->i0][1];
  m->bv = h->own_map[h->i0][2];
  m->bw = h->own_map[h->i0][3];
  m->cls = h->cls_map;
  *a = stage_args<R>(h, st);
}
template <class R>
void band_desc(fz_handle* h, int st, fz::BandArgs<R>* b) {
  *b = band_args<R>(h, st);
}
template <class R>
void rec_desc(fz_handle* h, fz::RecArgs<R>* r) {
  R* const* u1 = (R* const*)h->U[h->i1];
  r->p = u1[0];
  r->u = u1[1];
  r->v = u1[2];
  r->w = u1[3];
  r->rcell = h->d_rec_cell;
  r->nrec = h->nrec * h->nb;
  r->ir = h->d_ir;
  r->vel = h->d_vel;
  r->cap = h->rec_cap;
  r->step = h->d_step;
  r->err = h->d_err;
  r->nfield = h->ncell_dev * h->nb;
}
void rotate(fz_handle* h) {
  std::swap(h->i0, h->i1);
  std::swap(h->ph_old, h->ph_cur);
}
template void stage_desc<float>(fz_handle*, int, fz::StageArgs<float>*, fz::StageMaps*);
template void stage_desc<double>(fz_handle*, int, fz::StageArgs<double>*, fz::StageMaps*);
template void band_desc<float>(fz_handle*, int, fz::BandArgs<float>*);
template void band_desc<double>(fz_handle*, int, fz::BandArgs<double>*);
template void rec_desc<float>(fz_handle*, fz::RecArgs<float>*);
template void rec_desc<double>(fz_handle*, fz::RecArgs<double>*);
}  // namespace fzi

// ==========================================================================================
// C ABI
// ==========================================================================================
extern "C" {

int fz_params_init(fz_params* p) {
  if (!p) return fzi::set_global_error(FZ_EINVAL, "fz_params_init: NULL");
  std::memset(p, 0, sizeof(*p));
  p->abi_version = FZ_ABI_VERSION;
  p->precision = FZ_FP32;
  p->device = 0;
  p->pml_cells = 20;
  p->h = 0.02;
  // main3D.cu:450-456 at 20 degC, in the reference's float arithmetic
  const float Temp = 20.0f + 273.15f;
  p->c = (double)std::sqrt(1.4f * 287.05f * Temp);
  p->rho = (double)1.225f;
  p->dt = 0.5 * p->h / p->c;
  p->tol_cells = 3.0;
  p->pml_R0 = 1e-7;  // functions3D.cuh:692-719
  p->pml_kappa_max = 5.0;
  p->pml_alpha_max = M_PI * 20.0;
  p->pml_order = 2.0;
  return FZ_OK;
}

int fz_create(const fz_params* p, fz_handle** out) {
  if (!p || !out) return fzi::set_global_error(FZ_EINVAL, "fz_create: NULL argument");
  *out = nullptr;
  if (p->abi_version != FZ_ABI_VERSION)
    return fzi::set_global_error(FZ_EINVAL, "fz_create: abi_version mismatch");
  if (p->batch < 0 || p->batch > 4096)
    return fzi::set_global_error(FZ_EINVAL, "fz_create: batch must be in [0, 4096]");
  if (p->two_d && (p->pml[0] || p->pml[1]))
    return fzi::set_global_error(FZ_EINVAL, "fz_create: a planar (two_d) solve has no z faces: U_PML and D_PML must be 0");
  if (!(p->h > 0) || !(p->c > 0) || !(p->rho > 0) || !(p->dt > 0) || p->pml_cells < 1 ||
      (p->precision != FZ_FP32 && p->precision != FZ_FP64) || !(p->tol_cells > 1.0))
    return fzi::set_global_error(FZ_EINVAL, "fz_create: invalid parameter (h, c, rho, dt > 0; pml_cells >= 1; "
                                            "precision FZ_FP32/FZ_FP64; tol_cells > 1)");
  if (!(p->pml_R0 > 0 && p->pml_R0 < 1) || !(p->pml_kappa_max >= 1) || !(p->pml_alpha_max >= 0) ||
      !(p->pml_order > 0))
    return fzi::set_global_error(FZ_EINVAL, "fz_create: invalid cPML profile (0 < pml_R0 < 1, pml_kappa_max >= 1, "
                                            "pml_alpha_max >= 0, pml_order > 0)");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev <= 0)
    return fzi::set_global_error(FZ_ENODEV, std::string("no CUDA device: ") + cudaGetErrorString(e));
  if (p->device < 0 || p->device >= ndev) return fzi::set_global_error(FZ_ENODEV, "fz_create: bad device ordinal");
  fz_handle* h = new (std::nothrow) fz_handle();
  if (!h) return fzi::set_global_error(FZ_ENOMEM, "fz_create: out of host memory");
  h->prm = *p;
  h->device = p->device;
  h->fp64 = (p->precision == FZ_FP64);
  h->rsize = h->fp64 ? 8 : 4;
  e = cudaSetDevice(h->device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, h->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = h->fp64 ? fz::stage_setup<double>() : fz::stage_setup<float>();
  if (e == cudaSuccess) e = cudaMalloc(&h->d_step, sizeof(int64_t));
  if (e == cudaSuccess) e = cudaMemset(h->d_step, 0, sizeof(int64_t));
  if (e == cudaSuccess) e = cudaMalloc(&h->d_scratch, 64);
  if (e == cudaSuccess) e = cudaMalloc(&h->d_err, sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMemset(h->d_err, 0, sizeof(int32_t));
  if (e != cudaSuccess) {
    int rc = fzi::set_global_error(FZ_ECUDA, std::string("fz_create: ") + cudaGetErrorString(e));
    fz_destroy(h);
    return rc;
  }
  *out = h;
  return FZ_OK;
}

void fz_destroy(fz_handle* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (auto& t : h->timings) {
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
  }
  free_device(h);
  dfree(h->d_step);
  dfree(h->d_scratch);
  dfree(h->d_err);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

int fz_load_geometry_raw(fz_handle* h, const float* S, const uint8_t* oid, int32_t Nx, int32_t Ny,
                         int32_t Nz) {
  if (!check_handle(h)) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  if (!S || !oid) return set_error(h, FZ_EINVAL, "fz_load_geometry_raw: NULL array");
  const int minn = 2 * GHOST + 1;
  if (Nx < minn || Ny < minn || Nz < minn)
    return set_error(h, FZ_EINVAL, "fz_load_geometry_raw: grid must be at least 7 cells per axis");
  if (h->prm.two_d && Nz != minn)
    return set_error(h, FZ_EINVAL, "fz_load_geometry_raw: a planar (two_d) grid has Nz = 7 (one plane plus ghosts)");
  if (h->prm.pml_cells * 2 + 2 * GHOST > std::min(Nx, std::min(Ny, Nz)) &&
      (h->prm.pml[0] || h->prm.pml[1] || h->prm.pml[2] || h->prm.pml[3] || h->prm.pml[4] || h->prm.pml[5]))
    ;  // narrow domains with overlapping PML bands follow the reference's index rule
  cudaSetDevice(h->device);
  return h->fp64 ? load_geometry<double>(h, S, oid, Nx, Ny, Nz) : load_geometry<float>(h, S, oid, Nx, Ny, Nz);
}

int fz_set_materials(fz_handle* h, int32_t nMat, int32_t K, int32_t L, const double* Rinf, const double* A,
                     const double* zeta, const double* B, const double* C, const double* alpha,
                     const double* beta) {
  if (!check_handle(h)) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  if (h->finalized) return set_error(h, FZ_ESTATE, "fz_set_materials after the first fz_run");
  if (nMat < 0 || nMat > 254 || K < 0 || L < 0) return set_error(h, FZ_EINVAL, "fz_set_materials: bad sizes");
  if (nMat > 0 && !Rinf) return set_error(h, FZ_EINVAL, "fz_set_materials: NULL Rinf");
  if (K > 0 && nMat > 0 && (!A || !zeta)) return set_error(h, FZ_EINVAL, "fz_set_materials: NULL A/zeta");
  if (L > 0 && nMat > 0 && (!B || !C || !alpha || !beta))
    return set_error(h, FZ_EINVAL, "fz_set_materials: NULL B/C/alpha/beta");
  // K_m, L_m >= 1 as main3D.cu:602-603; missing poles are zero-filled as read_fit_file leaves them
  const int Kc = std::max(1, K), Lc = std::max(1, L), nm = std::max(1, nMat);
  h->nMat = nMat; h->K = Kc; h->L = Lc;
  h->Rinf.assign(nm, 0.0);
  h->A.assign((size_t)nm * Kc, 0.0); h->zeta.assign((size_t)nm * Kc, 0.0);
  h->B.assign((size_t)nm * Lc, 0.0); h->C.assign((size_t)nm * Lc, 0.0);
  h->alpha.assign((size_t)nm * Lc, 0.0); h->beta.assign((size_t)nm * Lc, 0.0);
  for (int m = 0; m < nMat; m++) {
    h->Rinf[m] = Rinf[m];
    for (int k = 0; k < K; k++) {
      h->A[(size_t)m * Kc + k] = A[(size_t)m * K + k];
      h->zeta[(size_t)m * Kc + k] = zeta[(size_t)m * K + k];
    }
    for (int l = 0; l < L; l++) {
      const size_t d = (size_t)m * Lc + l, s = (size_t)m * L + l;
      h->B[d] = B[s]; h->C[d] = C[s]; h->alpha[d] = alpha[s]; h->beta[d] = beta[s];
    }
  }
  h->have_materials = true;
  return FZ_OK;
}

int fz_set_sources(fz_handle* h, int32_t n, const int32_t* cell_ijk, const double* sval, int32_t src_opt,
                   const double* freq, const double* u_s, int64_t n_us) {
  if (!check_handle(h)) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  if (h->finalized) return set_error(h, FZ_ESTATE, "fz_set_sources after the first fz_run");
  if (!h->have_geometry) return set_error(h, FZ_ESTATE, "fz_set_sources before fz_load_geometry_raw");
  if (n < 0 || (n > 0 && (!cell_ijk || !sval))) return set_error(h, FZ_EINVAL, "fz_set_sources: bad arguments");
  if (src_opt < 0 || src_opt > 2) return set_error(h, FZ_EINVAL, "fz_set_sources: src_opt must be 0, 1 or 2");
  if (n > 0 && src_opt == 2 && !freq) return set_error(h, FZ_EINVAL, "fz_set_sources: sine sources need freq");
  if (n > 0 && src_opt != 2 && (!u_s || n_us < 1))
    return set_error(h, FZ_EINVAL, "fz_set_sources: PCS/Ricker sources need u_s");
  for (int s = 0; s < n; s++) {
    const int i = cell_ijk[3 * s], j = cell_ijk[3 * s + 1], k = cell_ijk[3 * s + 2];
    if (i < 0 || i >= h->Nx || j < 0 || j >= h->Ny || k < 0 || k >= h->Nz)
      return set_error(h, FZ_EINVAL, "fz_set_sources: source cell outside the grid");
  }
  h->nsrc = n;
  h->src_ijk.assign(cell_ijk, cell_ijk + 3 * (size_t)n);
  h->src_val.assign(sval, sval + n);
  h->src_freq.assign((size_t)n, 0.0);
  if (freq) h->src_freq.assign(freq, freq + n);
  h->src_opt = src_opt;
  h->src_member.clear();  // every source in every batch member until fz_set_source_members
  h->u_s.clear();
  if (u_s && n_us > 0) h->u_s.assign(u_s, u_s + n_us);
  return FZ_OK;
}

int fz_set_source_members(fz_handle* h, int32_t n, const int32_t* member) {
  if (!check_handle(h)) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  if (h->finalized) return set_error(h, FZ_ESTATE, "fz_set_source_members after the first fz_run");
  if (n != h->nsrc || (n > 0 && !member))
    return set_error(h, FZ_EINVAL, "fz_set_source_members: need one member index per source of fz_set_sources");
  const int nb = std::max(1, h->prm.batch);
  for (int s = 0; s < n; s++)
    if (member[s] < -1 || member[s] >= nb)
      return set_error(h, FZ_EINVAL, "fz_set_source_members: member index outside [-1, batch)");
  h->src_member.assign(member, member + n);
  return FZ_OK;
}

int fz_set_receivers(fz_handle* h, int32_t n, const int32_t* cell_ijk, int64_t capacity_steps) {
  if (!check_handle(h)) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  if (h->finalized) return set_error(h, FZ_ESTATE, "fz_set_receivers after the first fz_run");
  if (!h->have_geometry) return set_error(h, FZ_ESTATE, "fz_set_receivers before fz_load_geometry_raw");
  if (n < 0 || (n > 0 && !cell_ijk) || capacity_steps < 0)
    return set_error(h, FZ_EINVAL, "fz_set_receivers: bad arguments");
  for (int r = 0; r < n; r++) {
    const int i = cell_ijk[3 * r], j = cell_ijk[3 * r + 1], k = cell_ijk[3 * r + 2];
    // main3D.cu:942-944: a receiver outside the domain stops the run
    if (i < 0 || i >= h->Nx || j < 0 || j >= h->Ny || k < 0 || k >= h->Nz)
      return set_error(h, FZ_EINVAL, "fz_set_receivers: receiver outside the domain");
  }
  h->nrec = n;
  h->rec_ijk.assign(cell_ijk, cell_ijk + 3 * (size_t)n);
  h->rec_cap = capacity_steps;
  return FZ_OK;
}

int fz_set_slices(fz_handle* h, int32_t i0, int32_t j0, int32_t k0, int64_t anim_step, int64_t max_frames) {
  if (!check_handle(h)) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  if (!h->have_geometry) return set_error(h, FZ_ESTATE, "fz_set_slices before fz_load_geometry_raw");
  if (h->steps_enqueued != 0 || h->nb != 1)
    return set_error(h, FZ_ESTATE, "fz_set_slices: set before the first step, on a single-member solve");
  if (i0 < 0 || i0 >= h->Nx || j0 < 0 || j0 >= h->Ny || k0 < 0 || k0 >= h->Nz || anim_step < 1 || max_frames < 0)
    return set_error(h, FZ_EINVAL, "fz_set_slices: planes inside the grid, anim_step >= 1, max_frames >= 0");
  cudaSetDevice(h->device);
  dfree(h->d_slices);
  h->sl_on = false;
  if (max_frames == 0) return FZ_OK;
  const int64_t frame = 3 * ((int64_t)h->Ny * h->Nz + (int64_t)h->Nx * h->Nz + (int64_t)h->Nx * h->Ny);
  FZ_CUDA(h, cudaMalloc(&h->d_slices, (size_t)frame * max_frames * sizeof(float)), "cudaMalloc(slices)");
  h->sl_i = i0; h->sl_j = j0; h->sl_k = k0;
  h->sl_step = anim_step;
  h->sl_cap = max_frames;
  h->sl_frame = frame;
  h->sl_on = true;
  free_graphs(h);  // captured steps must include the slice launch
  return FZ_OK;
}

int fz_get_slices(fz_handle* h, float* out, int64_t cap, int64_t* frames) {
  if (!check_handle(h)) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  int rc = fz_sync(h, 0);
  if (rc != FZ_OK) return rc;
  int64_t n = 0;
  FZ_CUDA(h, cudaMemcpy(&n, h->d_step, sizeof(int64_t), cudaMemcpyDeviceToHost), "step D2H");
  const int64_t nf = h->sl_on ? std::min(h->sl_cap, n > 0 ? (n - 1) / h->sl_step + 1 : 0) : 0;
  if (frames) *frames = nf;
  if (!out) return FZ_OK;
  if (cap < nf * h->sl_frame) return set_error(h, FZ_EINVAL, "fz_get_slices: buffer too small");
  if (nf > 0)
    FZ_CUDA(h, cudaMemcpy(out, h->d_slices, (size_t)(nf * h->sl_frame) * sizeof(float), cudaMemcpyDeviceToHost),
            "slices D2H");
  return FZ_OK;
}

int fz_set_fields(fz_handle* h, const double* p, const double* u, const double* v, const double* w) {
  if (!check_handle(h)) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  if (!h->have_geometry) return set_error(h, FZ_ESTATE, "fz_set_fields before fz_load_geometry_raw");
  int rc = fz_sync(h, 0);
  // a blown-up state, or one a kernel's bounded wait left invalid, is what this call replaces; a
  // host-side timeout (work still running) is not
  if (rc == FZ_ETIMEOUT && cudaStreamQuery(h->stream) != cudaSuccess) return rc;
  if (rc != FZ_OK && rc != FZ_ENONFINITE && rc != FZ_ETIMEOUT) return rc;
  cudaSetDevice(h->device);
  // a new initial state, as a fresh solver has it: the two other field sets zero (cells the stage
  // kernels skip keep their values from set to set), quiescent ADE and cPML auxiliary states and
  // a clean health word
  FZ_CUDA(h, cudaMemset(h->d_err, 0, sizeof(int32_t)), "error word reset");
  for (int q : {h->i1, h->i2})
    for (int f = 0; f < 4; f++)
      FZ_CUDA(h, cudaMemset(h->U[q][f], 0, (size_t)h->ncell_dev * h->nb * h->rsize), "field set reset");
  if (h->nB > 0)
    for (int q = 0; q < 3; q++)
      for (int a = 0; a < 3; a++)
        if (h->d_ade[q][a]) {
          const size_t n = (size_t)h->nB * (a == 0 ? h->K : h->L) * 8;
          FZ_CUDA(h, cudaMemset(h->d_ade[q][a], 0, n), "ADE reset");
        }
  {
    const int64_t d2 = 2 * (int64_t)h->prm.pml_cells;
    const int64_t tile_n[3] = {d2 * h->Ny * h->Nz * h->nb, (int64_t)h->Nx * d2 * h->Nz * h->nb,
                               (int64_t)h->Nx * h->Ny * d2 * h->nb};
    for (int a = 0; a < 3; a++)
      if (h->d_psi[a]) FZ_CUDA(h, cudaMemset(h->d_psi[a], 0, (size_t)tile_n[a] * 2 * h->rsize), "psi reset");
  }
  return h->fp64 ? set_fields<double>(h, p, u, v, w) : set_fields<float>(h, p, u, v, w);
}

// ---- checkpoint / resume -------------------------------------------------------------------
// Layout of a saved state: StateHeader, then the field sets in rotation roles (U0, U1, U2; 4
// fields each), the ADE sets in roles (old, cur, nu; phi, psi1, psi2), the cPML psi tiles, the
// receiver traces and velocities, the animation frames.
namespace {
struct StateHeader {
  char magic[8];
  int32_t precision, nb, Nx, Ny, Nz, K, L, nrec, slices, pml_cells;
  int64_t nB, rec_cap, step, sl_cap, psi_bytes[3];
  uint64_t physics;  // hash of what the update arithmetic depends on beyond the shapes
};

// FNV-1a (64 bit) over byte ranges.
struct Fnv {
  uint64_t h = 1469598103934665603ull;
  void add(const void* p, size_t n) {
    const unsigned char* b = (const unsigned char*)p;
    for (size_t i = 0; i < n; i++) h = (h ^ b[i]) * 1099511628211ull;
  }
};
#define FNV_VAL(f, x) (f).add(&(x), sizeof(x))
#define FNV_VEC(f, v)                                                   \
  do {                                                                  \
    const uint64_t n__ = (uint64_t)(v).size();                          \
    (f).add(&n__, sizeof(n__));                                         \
    if (n__) (f).add((v).data(), (size_t)n__ * sizeof((v)[0]));         \
  } while (0)

// The parameters a saved state was stepped with: grid spacing, speed of sound, density, time step,
// blending band, cPML faces, thickness and profile, the geometry, every material coefficient and
// the sources. A state saved under other physics must not continue here.
uint64_t physics_hash(const fz_handle* h) {
  Fnv f;
  const fz_params& p = h->prm;
  for (double x : {p.h, p.c, p.rho, p.dt, p.tol_cells, p.pml_R0, p.pml_kappa_max, p.pml_alpha_max, p.pml_order})
    FNV_VAL(f, x);
  FNV_VAL(f, p.pml);
  FNV_VAL(f, p.pml_cells);
  FNV_VAL(f, p.two_d);
  FNV_VEC(f, h->S_host);
  FNV_VEC(f, h->oid_host);
  FNV_VAL(f, h->nMat);
  for (const std::vector<double>* v : {&h->Rinf, &h->A, &h->zeta, &h->B, &h->C, &h->alpha, &h->beta}) FNV_VEC(f, *v);
  FNV_VEC(f, h->src_ijk);
  FNV_VEC(f, h->src_val);
  FNV_VEC(f, h->src_freq);
  FNV_VEC(f, h->u_s);
  FNV_VAL(f, h->src_opt);
  FNV_VEC(f, h->src_member);
  return f.h;
}

struct StatePart {
  void* dev;
  size_t bytes;
};

std::vector<StatePart> state_parts(fz_handle* h) {
  std::vector<StatePart> v;
  const size_t fb = (size_t)h->ncell_dev * h->nb * h->rsize;
  for (int role : {h->i0, h->i1, h->i2})
    for (int f = 0; f < 4; f++) v.push_back({h->U[role][f], fb});
  const size_t ab[3] = {(size_t)h->K * h->nB * 8, (size_t)h->L * h->nB * 8, (size_t)h->L * h->nB * 8};
  for (int role : {h->ph_old, h->ph_cur, h->ph_nu})
    for (int q = 0; q < 3; q++)
      if (h->nB > 0) v.push_back({h->d_ade[role][q], ab[q]});
  const int64_t d2 = 2 * (int64_t)h->prm.pml_cells;
  const int64_t tile_n[3] = {d2 * h->Ny * h->Nz * h->nb, (int64_t)h->Nx * d2 * h->Nz * h->nb,
                             (int64_t)h->Nx * h->Ny * d2 * h->nb};
  for (int a = 0; a < 3; a++)
    if (h->d_psi[a]) v.push_back({h->d_psi[a], (size_t)tile_n[a] * 2 * h->rsize});
  if (h->nrec > 0) {
    const size_t n = (size_t)h->nrec * h->nb * (size_t)std::max<int64_t>(1, h->rec_cap);
    v.push_back({h->d_ir, n * 8});
    v.push_back({h->d_vel, n * 3 * 8});
  }
  if (h->sl_on) v.push_back({h->d_slices, (size_t)(h->sl_frame * h->sl_cap) * sizeof(float)});
  return v;
}

void state_header(fz_handle* h, StateHeader& hd) {
  std::memset(&hd, 0, sizeof(hd));
  std::memcpy(hd.magic, "FZSTATE2", 8);
  hd.precision = h->prm.precision;
  hd.pml_cells = h->prm.pml_cells;
  hd.physics = physics_hash(h);
  hd.nb = h->nb; hd.Nx = h->Nx; hd.Ny = h->Ny; hd.Nz = h->Nz; hd.K = h->K; hd.L = h->L;
  hd.nrec = h->nrec; hd.slices = h->sl_on ? 1 : 0;
  hd.nB = h->nB; hd.rec_cap = h->rec_cap; hd.sl_cap = h->sl_on ? h->sl_cap : 0;
  for (int a = 0; a < 3; a++) hd.psi_bytes[a] = h->d_psi[a] ? 1 : 0;
}
}  // namespace

int fz_state_bytes(fz_handle* h, int64_t* bytes) {
  if (!check_handle(h) || !bytes) return fzi::set_global_error(FZ_EINVAL, "fz_state_bytes: NULL argument");
  if (!h->have_geometry) return set_error(h, FZ_ESTATE, "fz_state_bytes before fz_load_geometry_raw");
  int rc = fzi::prepare(h);
  if (rc != FZ_OK) return rc;
  int64_t n = (int64_t)sizeof(StateHeader);
  for (const auto& p : state_parts(h)) n += (int64_t)p.bytes;
  *bytes = n;
  return FZ_OK;
}

int fz_state_save(fz_handle* h, void* buf, int64_t cap) {
  fz_range nvtx_range("fz_state_save");
  int64_t need = 0;
  int rc = fz_state_bytes(h, &need);
  if (rc != FZ_OK) return rc;
  if (!buf || cap < need) return set_error(h, FZ_EINVAL, "fz_state_save: buffer needs " + std::to_string(need) + " bytes");
  rc = fz_sync(h, 0);
  if (rc != FZ_OK) return rc;
  StateHeader hd;
  state_header(h, hd);
  FZ_CUDA(h, cudaMemcpy(&hd.step, h->d_step, sizeof(int64_t), cudaMemcpyDeviceToHost), "step D2H");
  char* o = (char*)buf;
  std::memcpy(o, &hd, sizeof(hd));
  o += sizeof(hd);
  for (const auto& p : state_parts(h)) {
    FZ_CUDA(h, cudaMemcpy(o, p.dev, p.bytes, cudaMemcpyDeviceToHost), "state D2H");
    o += p.bytes;
  }
  return FZ_OK;
}

int fz_state_load(fz_handle* h, const void* buf, int64_t len) {
  fz_range nvtx_range("fz_state_load");
  int64_t need = 0;
  int rc = fz_state_bytes(h, &need);
  if (rc != FZ_OK) return rc;
  if (!buf || len < need) return set_error(h, FZ_EINVAL, "fz_state_load: state of the wrong size for this solver");
  rc = fz_sync(h, 0);
  if (rc != FZ_OK) return rc;
  StateHeader mine, hd;
  state_header(h, mine);
  std::memcpy(&hd, buf, sizeof(hd));
  const int64_t step = hd.step;
  hd.step = 0;
  if (std::memcmp(mine.magic, hd.magic, sizeof(hd.magic)) != 0)
    return set_error(h, FZ_EINVAL, "fz_state_load: not a state of this library version");
  const uint64_t their_physics = hd.physics;
  hd.physics = mine.physics;
  if (std::memcmp(&mine, &hd, sizeof(hd)) != 0)
    return set_error(h, FZ_EINVAL, "fz_state_load: the state was saved by a solver of another configuration "
                                   "(grid, precision, batch, band, poles, receivers, cPML or slices differ)");
  if (their_physics != mine.physics)
    return set_error(h, FZ_EINVAL, "fz_state_load: the state was saved by a solver with other physics "
                                   "(h, c, rho, dt, geometry, materials, cPML profile or sources differ)");
  const char* o = (const char*)buf + sizeof(hd);
  for (const auto& p : state_parts(h)) {
    FZ_CUDA(h, cudaMemcpy(p.dev, o, p.bytes, cudaMemcpyHostToDevice), "state H2D");
    o += p.bytes;
  }
  FZ_CUDA(h, cudaMemcpy(h->d_step, &step, sizeof(step), cudaMemcpyHostToDevice), "step H2D");
  FZ_CUDA(h, cudaMemset(h->d_err, 0, sizeof(int32_t)), "error word reset");
  h->steps_enqueued = step;
  return FZ_OK;
}

int fz_check_health(fz_handle* h, int64_t* nonfinite) {
  if (!check_handle(h)) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  if (!h->have_geometry) return set_error(h, FZ_ESTATE, "fz_check_health before fz_load_geometry_raw");
  cudaSetDevice(h->device);
  unsigned long long* d = (unsigned long long*)h->d_scratch;  // 64-byte per-handle scratch
  FZ_CUDA(h, cudaMemsetAsync(d, 0, sizeof(*d), h->stream), "health reset");
  const int64_t n = h->ncell_dev * h->nb;
  cudaError_t e = h->fp64 ? fz::launch_count_nonfinite<double>((const double*)h->U[h->i0][0], (const double*)h->U[h->i0][1],
                                                               (const double*)h->U[h->i0][2], (const double*)h->U[h->i0][3],
                                                               n, d, h->nsm, h->stream)
                          : fz::launch_count_nonfinite<float>((const float*)h->U[h->i0][0], (const float*)h->U[h->i0][1],
                                                              (const float*)h->U[h->i0][2], (const float*)h->U[h->i0][3],
                                                              n, d, h->nsm, h->stream);
  if (e != cudaSuccess) return cuda_fail(h, e, "health launch");
  int rc = fz_sync(h, 0);
  unsigned long long cnt = 0;
  FZ_CUDA(h, cudaMemcpy(&cnt, d, sizeof(cnt), cudaMemcpyDeviceToHost), "health D2H");
  if (nonfinite) *nonfinite = (int64_t)cnt;
  if (cnt > 0) return set_error(h, FZ_ENONFINITE, std::to_string(cnt) + " non-finite values in the current state");
  return rc;
}

int fz_run(fz_handle* h, int64_t nsteps) {
  fz_range nvtx_range("fz_run");
  if (!check_handle(h)) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  if (nsteps < 0) return set_error(h, FZ_EINVAL, "fz_run: negative step count");
  cudaSetDevice(h->device);
  return h->fp64 ? run_steps<double>(h, nsteps) : run_steps<float>(h, nsteps);
}

#ifdef FZ_WAIT_TEST
// Wait-test build only: the stage kernels never issue the tile of plane `plane` of each z chunk
// (-1: every tile is issued), so their bounded wait for it runs out.
extern "C" int fz_test_skip_plane(fz_handle* h, int32_t plane) {
  if (!check_handle(h)) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  h->test_skip_plane = plane;
  free_graphs(h);  // captured launches carry the old value
  return FZ_OK;
}
#endif

int fz_prepare(fz_handle* h) {
  fz_range nvtx_range("fz_prepare");
  if (!check_handle(h)) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  cudaSetDevice(h->device);
  int rc = h->fp64 ? prepare_graphs<double>(h) : prepare_graphs<float>(h);
  if (rc == FZ_OK) rc = fz_sync(h, 0);
  return rc;
}

int fz_run_progress(fz_handle* h, int64_t nsteps, int32_t every_percent, fz_progress_fn cb, void* user) {
  fz_range nvtx_range("fz_run_progress");
  if (!check_handle(h)) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  if (nsteps < 0 || every_percent < 1 || every_percent > 100)
    return set_error(h, FZ_EINVAL, "fz_run_progress: nsteps >= 0 and every_percent in [1, 100]");
  const int64_t slice = std::max<int64_t>(1, nsteps * every_percent / 100);
  int64_t done = 0;
  while (done < nsteps) {
    const int64_t n = std::min(slice, nsteps - done);
    int rc = fz_run(h, n);
    if (rc == FZ_OK) rc = fz_sync(h, 0);
    if (rc != FZ_OK) return rc;
    done += n;
    if (cb && cb(done, nsteps, user) != 0) break;
  }
  return FZ_OK;
}

int fz_run_timed(fz_handle* h, int64_t nsteps, double* ms) {
  if (!check_handle(h) || !ms) return fzi::set_global_error(FZ_EINVAL, "NULL argument");
  cudaSetDevice(h->device);
  int rc = fz_sync(h, 0);
  if (rc != FZ_OK) return rc;
  cudaEvent_t a = nullptr, b = nullptr;
  FZ_CUDA(h, cudaEventCreate(&a), "event");
  cudaError_t e = cudaEventCreate(&b);
  if (e != cudaSuccess) { cudaEventDestroy(a); return cuda_fail(h, e, "event"); }
  e = cudaEventRecord(a, h->stream);
  rc = (e == cudaSuccess) ? fz_run(h, nsteps) : cuda_fail(h, e, "event record");
  if (rc == FZ_OK) {
    e = cudaEventRecord(b, h->stream);
    rc = (e == cudaSuccess) ? fz_sync(h, 0) : cuda_fail(h, e, "event record");
  }
  if (rc == FZ_OK) {
    float x = 0.f;
    e = cudaEventElapsedTime(&x, a, b);
    if (e == cudaSuccess) *ms = x; else rc = cuda_fail(h, e, "event elapsed");
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return rc;
}

int fz_sync(fz_handle* h, int64_t timeout_ms) {
  if (!check_handle(h)) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  if (timeout_ms <= 0) timeout_ms = 600000;
  cudaSetDevice(h->device);
  const auto t0 = std::chrono::steady_clock::now();
  int sleep_us = 20;
  for (;;) {
    cudaError_t e = cudaStreamQuery(h->stream);
    if (e == cudaSuccess) {
      int32_t kerr = 0;
      e = cudaMemcpy(&kerr, h->d_err, sizeof(kerr), cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) return cuda_fail(h, e, "error word D2H");
      if (kerr & fz::KERR_TMA_TIMEOUT)
        return set_error(h, FZ_ETIMEOUT, "a kernel's bounded wait gave up (code " + std::to_string(kerr) +
                                             "); results of this run are invalid");
      if (kerr & fz::KERR_NONFINITE)
        return set_error(h, FZ_ENONFINITE, "a receiver sampled NaN or Inf: the solution blew up (check the "
                                               "materials' passivity, the CFL number and the initial fields)");
      if (kerr & fz::KERR_BOUNDS)
        return set_error(h, FZ_EBOUNDS, "the bounds-checked build caught an index outside its array (error word " +
                                             std::to_string(kerr) + ")");
      if (kerr != 0) return set_error(h, FZ_ECUDA, "device error word " + std::to_string(kerr));
      return FZ_OK;
    }
    if (e != cudaErrorNotReady) return cuda_fail(h, e, "stream");
    const auto ms =
        std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0).count();
    if (ms > timeout_ms) return set_error(h, FZ_ETIMEOUT, "fz_sync: device work did not finish in time");
    std::this_thread::sleep_for(std::chrono::microseconds(sleep_us));
    sleep_us = std::min(sleep_us * 2, 2000);
  }
}

int fz_steps_done(fz_handle* h, int64_t* n) {
  if (!check_handle(h) || !n) return fzi::set_global_error(FZ_EINVAL, "NULL argument");
  int rc = fz_sync(h, 0);
  if (rc != FZ_OK) return rc;
  FZ_CUDA(h, cudaMemcpy(n, h->d_step, sizeof(int64_t), cudaMemcpyDeviceToHost), "step D2H");
  return FZ_OK;
}

static int get_samples(fz_handle* h, double* out64, float* out32, int64_t cap, bool vel) {
  if (!check_handle(h)) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  int rc = fz_sync(h, 0);
  if (rc != FZ_OK) return rc;
  int64_t n = 0;
  FZ_CUDA(h, cudaMemcpy(&n, h->d_step, sizeof(int64_t), cudaMemcpyDeviceToHost), "step D2H");
  n = std::min(n, h->rec_cap);
  const int comp = vel ? 3 : 1;
  const int rows = h->nrec * h->nb;  // [member][receiver]
  const int64_t need = (int64_t)rows * n * comp;
  if (cap < need) return set_error(h, FZ_EINVAL, "output buffer too small: need " + std::to_string(need));
  if (need == 0) return FZ_OK;
  std::vector<double> tmp((size_t)rows * h->rec_cap * comp);
  FZ_CUDA(h, cudaMemcpy(tmp.data(), vel ? h->d_vel : h->d_ir, tmp.size() * 8, cudaMemcpyDeviceToHost), "IR D2H");
  for (int r = 0; r < rows; r++)
    for (int64_t t = 0; t < n * comp; t++) {
      const double x = tmp[(size_t)r * h->rec_cap * comp + t];
      const size_t o = (size_t)r * n * comp + t;
      if (out64) out64[o] = x;
      if (out32) out32[o] = (float)x;
    }
  return FZ_OK;
}

int fz_get_ir(fz_handle* h, float* out, int64_t cap) { return get_samples(h, nullptr, out, cap, false); }
int fz_get_ir64(fz_handle* h, double* out, int64_t cap) { return get_samples(h, out, nullptr, cap, false); }
int fz_get_vel(fz_handle* h, float* out, int64_t cap) { return get_samples(h, nullptr, out, cap, true); }

int fz_get_fields(fz_handle* h, double* p, double* u, double* v, double* w) {
  if (!check_handle(h)) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  if (!h->have_geometry) return set_error(h, FZ_ESTATE, "fz_get_fields before fz_load_geometry_raw");
  int rc = fz_sync(h, 0);
  if (rc != FZ_OK) return rc;
  return h->fp64 ? get_fields<double>(h, p, u, v, w) : get_fields<float>(h, p, u, v, w);
}

int fz_energy(fz_handle* h, double* E) {
  if (!check_handle(h) || !E) return fzi::set_global_error(FZ_EINVAL, "NULL argument");
  if (!h->have_geometry) return set_error(h, FZ_ESTATE, "fz_energy before fz_load_geometry_raw");
  cudaSetDevice(h->device);
  return h->fp64 ? energy<double>(h, E) : energy<float>(h, E);
}

int fz_info(fz_handle* h, int32_t* dims, int64_t* n_band, int64_t* n_update) {
  if (!check_handle(h)) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  if (dims) { dims[0] = h->Nx; dims[1] = h->Ny; dims[2] = h->Nz; }
  if (n_band) *n_band = h->nB1;  // band cells of one batch member
  if (n_update) *n_update = h->n_update;
  return FZ_OK;
}

int fz_profile_enable(fz_handle* h, int32_t on) {
  if (!check_handle(h)) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  h->profiling = (on != 0);
  return FZ_OK;
}

int fz_profile_read(fz_handle* h, double* ms, int64_t* launches, int32_t nkinds) {
  if (!check_handle(h)) return fzi::set_global_error(FZ_EINVAL, "NULL handle");
  int rc = fz_sync(h, 0);
  if (rc != FZ_OK) return rc;
  for (auto& t : h->timings) {
    float x = 0.f;
    if (cudaEventElapsedTime(&x, t.a, t.b) == cudaSuccess && t.kind >= 0 && t.kind < 8) {
      h->prof_ms[t.kind] += x;
      h->prof_n[t.kind] += 1;
    }
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
  }
  h->timings.clear();
  for (int k = 0; k < nkinds && k < 8; k++) {
    if (ms) ms[k] = h->prof_ms[k];
    if (launches) launches[k] = h->prof_n[k];
  }
  for (int k = 0; k < 8; k++) { h->prof_ms[k] = 0; h->prof_n[k] = 0; }
  return FZ_OK;
}

int fz_device_memory(int32_t device, int64_t* free_bytes, int64_t* total_bytes) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return fzi::set_global_error(FZ_ENODEV, "fz_device_memory: no such CUDA device");
  cudaSetDevice(device);
  size_t f = 0, t = 0;
  const cudaError_t e = cudaMemGetInfo(&f, &t);
  if (e != cudaSuccess) return fzi::set_global_error(FZ_ECUDA, std::string("cudaMemGetInfo: ") + cudaGetErrorString(e));
  if (free_bytes) *free_bytes = (int64_t)f;
  if (total_bytes) *total_bytes = (int64_t)t;
  return FZ_OK;
}

int fz_last_error(fz_handle* h, char* buf, size_t cap) {
  if (!buf || cap == 0) return FZ_EINVAL;
  const std::string& s = h ? h->err : g_err;
  std::snprintf(buf, cap, "%s", s.c_str());
  return FZ_OK;
}

int fz_global_error(char* buf, size_t cap) {
  if (!buf || cap == 0) return FZ_EINVAL;
  std::snprintf(buf, cap, "%s", g_err.c_str());
  return FZ_OK;
}

}  // extern "C"
