// fz_geometry.cu -- scene geometry from an OBJ file on the GPU: the signed distance S (positive in
// air) and the material id map oid of the padded grid, as the reference builds them before its
// time loop (3D-solver/include/parsing3D.h: OBJ reader 150-288, narrow-band distance 389-452 and
// 574-661, grid sizing 815-910, material ids 955-1154; main3D.cu:300-428 for the scene cache).
//
// B200 layout of the work, same results:
//  - distance: every triangle's 8h-expanded bounding box of voxel centres is cut into blocks of
//    4096 voxels, one CTA each, instead of one thread walking a whole wall's box; |d| lands by an
//    atomic min on the float bits (non-negative floats order like unsigned integers), so the
//    result does not depend on the order;
//  - sign: one thread per x row casts the +x parity ray, testing only triangles whose y-z bounds
//    (slightly widened) contain the ray;
//  - material id: one thread per band voxel finds the nearest triangle to the foot point,
//    skipping triangles whose bounding box is provably farther than the best so far.
// The point-triangle distance (Ericson, Real-Time Collision Detection, 5.1.5) and the ray-triangle
// test (Moller & Trumbore 1997) are written with the same operation order as the reference's, so
// that the single-precision results match.
#include <cuda_runtime.h>
#include <float.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/fz.h"
#include "fz_internal.h"

namespace {

struct V3 {
  float x, y, z;
};
__host__ __device__ __forceinline__ V3 mk(float x, float y, float z) { return V3{x, y, z}; }
__host__ __device__ __forceinline__ V3 vsub(const V3& a, const V3& b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ V3 vadd(const V3& a, const V3& b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ V3 vscale(const V3& a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ float vdot(const V3& a, const V3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ V3 vcross(const V3& a, const V3& b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

struct Tri3 {
  V3 a, b, c;
  int group;
};

// Squared distance from p to triangle abc: the Voronoi-region walk of Ericson's closest-point
// routine (vertex regions, edge regions, face).
__device__ __forceinline__ float tri_dist2(const V3& p, const V3& a, const V3& b, const V3& c) {
  const V3 ab = vsub(b, a), ac = vsub(c, a), ap = vsub(p, a);
  const float d1 = vdot(ab, ap), d2 = vdot(ac, ap);
  if (d1 <= 0.f && d2 <= 0.f) return vdot(ap, ap);
  const V3 bp = vsub(p, b);
  const float d3 = vdot(ab, bp), d4 = vdot(ac, bp);
  if (d3 >= 0.f && d4 <= d3) return vdot(bp, bp);
  const float vc = d1 * d4 - d3 * d2;
  if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
    const float v = d1 / (d1 - d3);
    const V3 q = vsub(p, vadd(a, vscale(ab, v)));
    return vdot(q, q);
  }
  const V3 cp = vsub(p, c);
  const float d5 = vdot(ab, cp), d6 = vdot(ac, cp);
  if (d6 >= 0.f && d5 <= d6) return vdot(cp, cp);
  const float vb = d5 * d2 - d1 * d6;
  if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
    const float w = d2 / (d2 - d6);
    const V3 q = vsub(p, vadd(a, vscale(ac, w)));
    return vdot(q, q);
  }
  const float va = d3 * d6 - d5 * d4;
  if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
    const float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    const V3 q = vsub(p, vadd(b, vscale(vsub(c, b), w)));
    return vdot(q, q);
  }
  const float inv = 1.f / (va + vb + vc);
  const float v = vb * inv, w = vc * inv;
  const V3 q = vsub(p, vadd(a, vadd(vscale(ab, v), vscale(ac, w))));
  return vdot(q, q);
}

// Moller-Trumbore, edge-inclusive: hit at parameter t > tmin.
__device__ __forceinline__ bool ray_hit(const V3& o, const V3& d, const V3& a, const V3& b, const V3& c, float tmin,
                                        float& t_out) {
  const V3 e1 = vsub(b, a), e2 = vsub(c, a);
  const V3 pv = vcross(d, e2);
  const float det = vdot(e1, pv);
  if (det > -1e-8f && det < 1e-8f) return false;
  const float inv = 1.f / det;
  const V3 tv = vsub(o, a);
  const float u = vdot(tv, pv) * inv;
  if (u < 0.f || u > 1.f) return false;
  const V3 qv = vcross(tv, e1);
  const float v = vdot(d, qv) * inv;
  if (v < 0.f || u + v > 1.f) return false;
  const float t = vdot(e2, qv) * inv;
  if (t > tmin) {
    t_out = t;
    return true;
  }
  return false;
}

struct GridG {
  int Nx, Ny, Nz;
  float h;
};

// block b of the distance scatter: triangle tri[b], voxels [first[b], first[b] + 4096) of its box
constexpr int SCATTER_CHUNK = 4096;

__global__ void k_fill(unsigned* a, int64_t n, unsigned v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) a[i] = v;
}

__global__ void __launch_bounds__(256) k_dist_scatter(unsigned* __restrict__ absu, const Tri3* __restrict__ tris,
                                                      const int4* __restrict__ box_lo, const int4* __restrict__ box_n,
                                                      const int* __restrict__ btri, const int64_t* __restrict__ bfirst,
                                                      GridG g) {
  const int t = btri[blockIdx.x];
  const int64_t first = bfirst[blockIdx.x];
  const Tri3 tr = tris[t];
  const int4 lo = box_lo[t], nn = box_n[t];
  const int64_t total = (int64_t)nn.x * nn.y * nn.z;
  const int64_t end = min(first + (int64_t)SCATTER_CHUNK, total);
  const float h = g.h;
  for (int64_t v = first + threadIdx.x; v < end; v += blockDim.x) {
    const int i = lo.x + (int)(v % nn.x);
    const int64_t r = v / nn.x;
    const int j = lo.y + (int)(r % nn.y);
    const int k = lo.z + (int)(r / nn.y);
    const V3 p = mk(0.0f + (i + 0.5f) * h, 0.0f + (j + 0.5f) * h, 0.0f + (k + 0.5f) * h);
    const float d = sqrtf(tri_dist2(p, tr.a, tr.b, tr.c));
    atomicMin(&absu[(size_t)k * g.Ny * g.Nx + (size_t)j * g.Nx + i], __float_as_uint(d));
  }
}

constexpr int ROW_CAP = 64;  // crossings kept per row; more -> per-voxel parity rays

// One thread per (j, k) row: parity of +x crossings ahead of each voxel centre; odd = inside air.
__global__ void k_sign_rows(const unsigned* __restrict__ absu, float* __restrict__ S, const Tri3* __restrict__ tris,
                            const float4* __restrict__ yz, int ntri, GridG g) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= g.Ny || k >= g.Nz) return;
  const float h = g.h, tmin = 1e-6f;
  // the ray sits a fraction of a cell off the row centre, so that it does not graze the edges
  // shared by axis-aligned wall triangles (an edge-inclusive test would count both)
  const float y0 = 0.0f + (j + 0.5f) * h + 0.0137f * h, z0 = 0.0f + (k + 0.5f) * h + 0.0091f * h;
  const V3 o = mk(0.0f, y0, z0), dir = mk(1.f, 0.f, 0.f);
  float xs[ROW_CAP];
  int nc = 0;
  bool overflow = false;
  for (int t = 0; t < ntri && !overflow; ++t) {
    const float4 b = yz[t];  // widened y-z bounds: a hit needs (y0, z0) inside them
    if (y0 < b.x || y0 > b.y || z0 < b.z || z0 > b.w) continue;
    const Tri3 tr = tris[t];
    float tt;
    if (ray_hit(o, dir, tr.a, tr.b, tr.c, 0.0f, tt)) {
      if (nc < ROW_CAP)
        xs[nc++] = o.x + tt;
      else
        overflow = true;
    }
  }
  const size_t row = (size_t)k * g.Ny * g.Nx + (size_t)j * g.Nx;
  if (!overflow) {
    for (int a = 1; a < nc; ++a) {  // insertion sort
      const float key = xs[a];
      int b = a - 1;
      while (b >= 0 && xs[b] > key) {
        xs[b + 1] = xs[b];
        --b;
      }
      xs[b + 1] = key;
    }
    for (int i = 0; i < g.Nx; ++i) {
      const float xc = 0.0f + (i + 0.5f) * h;
      int ahead = 0;
      for (int q = nc - 1; q >= 0; --q) {
        if (xs[q] > xc + tmin)
          ++ahead;
        else
          break;
      }
      const float d = __uint_as_float(absu[row + i]);
      S[row + i] = (ahead & 1) ? d : -d;
    }
  } else {
    for (int i = 0; i < g.Nx; ++i) {
      const float xc = 0.0f + (i + 0.5f) * h;
      const V3 p = mk(xc, y0, z0);
      int hits = 0;
      for (int t = 0; t < ntri; ++t) {
        const float4 b = yz[t];
        if (y0 < b.x || y0 > b.y || z0 < b.z || z0 > b.w) continue;
        const Tri3 tr = tris[t];
        float tt;
        if (ray_hit(p, dir, tr.a, tr.b, tr.c, tmin, tt)) ++hits;
      }
      const float d = __uint_as_float(absu[row + i]);
      S[row + i] = (hits & 1) ? d : -d;
    }
  }
}

// Material id of band voxels (0 <= S <= tol, grid interior): the group of the triangle nearest to
// the foot point C - S n, n = grad S / |grad S|; the first of equally near triangles wins.
__global__ void k_oid(const float* __restrict__ S, uint8_t* __restrict__ oid, const Tri3* __restrict__ tris,
                      const float4* __restrict__ blo, const float4* __restrict__ bhi, int ntri,
                      const int* __restrict__ gid2lid, int max_gid, GridG g, float tol) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i < 1 || j < 1 || k < 1 || i >= g.Nx - 1 || j >= g.Ny - 1 || k >= g.Nz - 1) return;
  const size_t pl = (size_t)g.Ny * g.Nx;
  const size_t idx = (size_t)k * pl + (size_t)j * g.Nx + i;
  const float s = S[idx];
  if (!(s >= 0.0f && fabsf(s) <= tol)) return;
  const float h = g.h;
  const float gx = (S[idx + 1] - S[idx - 1]) / (2.0f * h);
  const float gy = (S[idx + g.Nx] - S[idx - g.Nx]) / (2.0f * h);
  const float gz = (S[idx + pl] - S[idx - pl]) / (2.0f * h);
  const float gn2 = gx * gx + gy * gy + gz * gz;
  if (gn2 <= 1e-24f) return;
  const float inv = 1.0f / sqrtf(gn2);
  const V3 n = mk(gx * inv, gy * inv, gz * inv);
  const V3 C = mk(0.0f + (i + 0.5f) * h, 0.0f + (j + 0.5f) * h, 0.0f + (k + 0.5f) * h);
  const V3 W = mk(C.x - s * n.x, C.y - s * n.y, C.z - s * n.z);
  float best = FLT_MAX;
  int gid = -1;
  for (int t = 0; t < ntri; ++t) {
    // squared distance to the triangle's bounding box: a lower bound of the distance to it (the
    // margin keeps the skip safe against rounding in either computation)
    const float4 lo = blo[t], hi = bhi[t];
    const float ex = fmaxf(fmaxf(lo.x - W.x, W.x - hi.x), 0.f);
    const float ey = fmaxf(fmaxf(lo.y - W.y, W.y - hi.y), 0.f);
    const float ez = fmaxf(fmaxf(lo.z - W.z, W.z - hi.z), 0.f);
    const float lb = ex * ex + ey * ey + ez * ez;
    if (lb > best * 1.0001f + 1e-30f) continue;
    const Tri3 tr = tris[t];
    const float dd = tri_dist2(W, tr.a, tr.b, tr.c);
    if (dd < best) {
      best = dd;
      gid = tr.group;
    }
  }
  if (gid < 0 || gid > max_gid) return;
  const int lid = gid2lid[gid];
  if (lid >= 0 && lid <= 254) oid[idx] = (uint8_t)lid;
}

struct Mesh {
  std::vector<V3> verts;
  std::vector<int> tv;  // 3 vertex indices per triangle
  std::vector<int> tg;  // group per triangle
  std::vector<std::string> groups;
};

// OBJ reader with the reference's grouping rules (parsing3D.h:167-288): a group is created at its
// first face, "o"/"g" lines name it by their second token if there are two or more ("g Mesh1
// ceiling Model" -> ceiling), repeated names reuse the group, faces are fanned into triangles,
// vertex indices may be negative (relative) and may carry /vt/vn parts.
int read_mesh(const std::string& path, Mesh& m, std::string& err) {
  std::ifstream in(path);
  if (!in) {
    err = "Could not open OBJ: " + path;
    return FZ_EIO;
  }
  std::unordered_map<std::string, int> ids;
  std::string cur = "unnamed";
  bool named = false;
  int cur_id = -1;
  std::string line;
  auto ws = [](char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n'; };
  while (std::getline(in, line)) {
    size_t a = 0, b = line.size();
    while (a < b && ws(line[a])) a++;
    while (b > a && ws(line[b - 1])) b--;
    line = line.substr(a, b - a);
    if (line.empty() || line[0] == '#') continue;
    if (line.rfind("v ", 0) == 0) {
      std::istringstream ss(line.substr(2));
      float x, y, z;
      if (ss >> x >> y >> z) m.verts.push_back(mk(x, y, z));
    } else if (line.rfind("o ", 0) == 0 || line.rfind("g ", 0) == 0) {
      std::istringstream ss(line.substr(2));
      std::vector<std::string> parts;
      std::string tok;
      while (ss >> tok) parts.push_back(tok);
      const std::string nm = parts.size() >= 2 ? parts[1] : (parts.size() == 1 ? parts[0] : "unnamed");
      if (!named || nm != cur) {
        cur = nm;
        named = true;
        cur_id = -1;
      }
    } else if (line.rfind("f ", 0) == 0) {
      std::istringstream ss(line.substr(2));
      std::vector<int> face;
      std::string tok;
      while (ss >> tok) {
        const size_t sl = tok.find('/');
        const std::string s0 = (sl == std::string::npos) ? tok : tok.substr(0, sl);
        int vi = s0.empty() ? 0 : std::atoi(s0.c_str());
        const int nv = (int)m.verts.size();
        if (vi > 0)
          vi -= 1;
        else if (vi < 0)
          vi += nv;
        else {
          err = "Invalid face index token: '" + tok + "'";
          return FZ_EPARSE;
        }
        if (vi < 0 || vi >= nv) {
          err = "Invalid face index token: '" + tok + "'";
          return FZ_EPARSE;
        }
        face.push_back(vi);
      }
      if (face.size() < 3) continue;
      if (cur_id < 0) {
        const std::string nm = named ? cur : std::string("unnamed");
        auto it = ids.find(nm);
        if (it != ids.end()) {
          cur_id = it->second;
        } else {
          cur_id = (int)m.groups.size();
          ids[nm] = cur_id;
          m.groups.push_back(nm);
        }
      }
      for (size_t q = 1; q + 1 < face.size(); ++q) {
        m.tv.push_back(face[0]);
        m.tv.push_back(face[q]);
        m.tv.push_back(face[q + 1]);
        m.tg.push_back(cur_id);
      }
    }
  }
  if (m.verts.empty() || m.tg.empty()) {
    err = "OBJ contained no vertices or no faces.";
    return FZ_EPARSE;
  }
  return FZ_OK;
}

// Grid of the scene (parsing3D.h:682-690, 815-845, 880-910): vertices shifted so that their minimum
// corner sits at 3h; the domain is [0, max + 3h] per axis, N = ceil(L / h).
void scene_grid(const Mesh& m, float h, std::vector<V3>& tv, int dims[3], float L[3]) {
  V3 mn = m.verts[0], mx = m.verts[0];
  for (const V3& v : m.verts) {
    mn = mk(std::min(mn.x, v.x), std::min(mn.y, v.y), std::min(mn.z, v.z));
    mx = mk(std::max(mx.x, v.x), std::max(mx.y, v.y), std::max(mx.z, v.z));
  }
  const float pad = 3 * h;
  const V3 shift = mk(-mn.x + pad, -mn.y + pad, -mn.z + pad);
  tv.resize(m.verts.size());
  V3 tmx = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
  for (size_t q = 0; q < m.verts.size(); q++) {
    const V3& v = m.verts[q];
    tv[q] = mk((v.x + shift.x) * 1.f, (v.y + shift.y) * 1.f, (v.z + shift.z) * 1.f);
    tmx = mk(std::max(tmx.x, tv[q].x), std::max(tmx.y, tv[q].y), std::max(tmx.z, tv[q].z));
  }
  L[0] = tmx.x + pad;
  L[1] = tmx.y + pad;
  L[2] = tmx.z + pad;
  for (int a = 0; a < 3; a++) dims[a] = (int)std::ceil((double)L[a] / (double)h);
}

template <class T>
struct DBuf {
  T* p = nullptr;
  ~DBuf() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(size_t n) { return cudaMalloc((void**)&p, std::max<size_t>(n, 1) * sizeof(T)); }
};

#define FZ_GCHK(call, what)                                                                             \
  do {                                                                                                  \
    cudaError_t e__ = (call);                                                                           \
    if (e__ != cudaSuccess)                                                                             \
      return fzi::set_global_error(FZ_ECUDA, std::string(what) + ": " + cudaGetErrorString(e__));      \
  } while (0)

int build(const char* obj_path, double hd, double tol_cells, int device, float* S_out, uint8_t* oid_out, int64_t cap,
          int dims[3], float L[3]) {
  Mesh m;
  std::string err;
  int rc = read_mesh(obj_path, m, err);
  if (rc != FZ_OK) return fzi::set_global_error(rc, err);
  const float h = (float)hd;
  std::vector<V3> tvx;
  scene_grid(m, h, tvx, dims, L);
  const int Nx = dims[0], Ny = dims[1], Nz = dims[2];
  if (Nx < 2 || Ny < 2 || Nz < 2) return fzi::set_global_error(FZ_EINVAL, "degenerate grid (domain too small for h)");
  const int64_t N = (int64_t)Nx * Ny * Nz;
  if (!S_out && !oid_out) return FZ_OK;  // dimensions only
  if (!S_out || !oid_out || cap < N)
    return fzi::set_global_error(FZ_EINVAL, "fz_build_scene: S and oid need " + std::to_string(N) + " cells each");
  const int ntri = (int)m.tg.size();
  std::vector<Tri3> tris((size_t)ntri);
  std::vector<float4> yz((size_t)ntri), blo((size_t)ntri), bhi((size_t)ntri);
  std::vector<int4> box_lo((size_t)ntri), box_n((size_t)ntri);
  const float band = 8.f * h;
  std::vector<int> btri;
  std::vector<int64_t> bfirst;
  for (int t = 0; t < ntri; t++) {
    Tri3 tr;
    tr.a = tvx[(size_t)m.tv[3 * t]];
    tr.b = tvx[(size_t)m.tv[3 * t + 1]];
    tr.c = tvx[(size_t)m.tv[3 * t + 2]];
    tr.group = m.tg[(size_t)t];
    tris[(size_t)t] = tr;
    const float lx = std::min(tr.a.x, std::min(tr.b.x, tr.c.x)), hx = std::max(tr.a.x, std::max(tr.b.x, tr.c.x));
    const float ly = std::min(tr.a.y, std::min(tr.b.y, tr.c.y)), hy = std::max(tr.a.y, std::max(tr.b.y, tr.c.y));
    const float lz = std::min(tr.a.z, std::min(tr.b.z, tr.c.z)), hz = std::max(tr.a.z, std::max(tr.b.z, tr.c.z));
    blo[(size_t)t] = make_float4(lx, ly, lz, 0.f);
    bhi[(size_t)t] = make_float4(hx, hy, hz, 0.f);
    const float wy = 1e-5f * (hy - ly) + 1e-6f * h, wz = 1e-5f * (hz - lz) + 1e-6f * h;
    yz[(size_t)t] = make_float4(ly - wy, hy + wy, lz - wz, hz + wz);
    // the voxel-centre box of the 8h-expanded triangle box (parsing3D.h:410-416)
    int i0 = (int)std::floor((lx - band - 0.0f) / h - 0.5f), i1 = (int)std::ceil((hx + band - 0.0f) / h - 0.5f);
    int j0 = (int)std::floor((ly - band - 0.0f) / h - 0.5f), j1 = (int)std::ceil((hy + band - 0.0f) / h - 0.5f);
    int k0 = (int)std::floor((lz - band - 0.0f) / h - 0.5f), k1 = (int)std::ceil((hz + band - 0.0f) / h - 0.5f);
    i0 = std::max(i0, 0); j0 = std::max(j0, 0); k0 = std::max(k0, 0);
    i1 = std::min(i1, Nx - 1); j1 = std::min(j1, Ny - 1); k1 = std::min(k1, Nz - 1);
    const int nx = std::max(0, i1 - i0 + 1), ny = std::max(0, j1 - j0 + 1), nz = std::max(0, k1 - k0 + 1);
    box_lo[(size_t)t] = make_int4(i0, j0, k0, 0);
    box_n[(size_t)t] = make_int4(nx, ny, nz, 0);
    const int64_t tot = (int64_t)nx * ny * nz;
    for (int64_t f = 0; f < tot; f += SCATTER_CHUNK) {
      btri.push_back(t);
      bfirst.push_back(f);
    }
  }
  // material ids in order of first appearance of each group id (parsing3D.h:1004-1012)
  int max_gid = -1;
  for (int gq : m.tg) max_gid = std::max(max_gid, gq);
  std::vector<int> present((size_t)max_gid + 1, 0), gid2lid((size_t)max_gid + 1, -1);
  for (int gq : m.tg) present[(size_t)gq] = 1;
  int lid = 0;
  for (int gq = 0; gq <= max_gid; gq++)
    if (present[(size_t)gq] && lid <= 254) gid2lid[(size_t)gq] = 1 + lid++;

  if (device >= 0) FZ_GCHK(cudaSetDevice(device), "cudaSetDevice");
  cudaStream_t s = nullptr;
  FZ_GCHK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
  struct SG {
    cudaStream_t s;
    ~SG() { cudaStreamDestroy(s); }
  } sg{s};
  DBuf<Tri3> d_tris;
  DBuf<float4> d_yz, d_blo, d_bhi;
  DBuf<int4> d_box_lo, d_box_n;
  DBuf<int> d_btri, d_map;
  DBuf<int64_t> d_bfirst;
  DBuf<unsigned> d_abs;
  DBuf<float> d_S;
  DBuf<uint8_t> d_oid;
  FZ_GCHK(d_tris.alloc(ntri), "cudaMalloc");
  FZ_GCHK(d_yz.alloc(ntri), "cudaMalloc");
  FZ_GCHK(d_blo.alloc(ntri), "cudaMalloc");
  FZ_GCHK(d_bhi.alloc(ntri), "cudaMalloc");
  FZ_GCHK(d_box_lo.alloc(ntri), "cudaMalloc");
  FZ_GCHK(d_box_n.alloc(ntri), "cudaMalloc");
  FZ_GCHK(d_btri.alloc(btri.size()), "cudaMalloc");
  FZ_GCHK(d_bfirst.alloc(bfirst.size()), "cudaMalloc");
  FZ_GCHK(d_map.alloc(gid2lid.size()), "cudaMalloc");
  FZ_GCHK(d_abs.alloc((size_t)N), "cudaMalloc");
  FZ_GCHK(d_S.alloc((size_t)N), "cudaMalloc");
  FZ_GCHK(d_oid.alloc((size_t)N), "cudaMalloc");
  auto up = [&](void* d, const void* hsrc, size_t bytes) {
    return bytes ? cudaMemcpyAsync(d, hsrc, bytes, cudaMemcpyHostToDevice, s) : cudaSuccess;
  };
  FZ_GCHK(up(d_tris.p, tris.data(), tris.size() * sizeof(Tri3)), "H2D");
  FZ_GCHK(up(d_yz.p, yz.data(), yz.size() * sizeof(float4)), "H2D");
  FZ_GCHK(up(d_blo.p, blo.data(), blo.size() * sizeof(float4)), "H2D");
  FZ_GCHK(up(d_bhi.p, bhi.data(), bhi.size() * sizeof(float4)), "H2D");
  FZ_GCHK(up(d_box_lo.p, box_lo.data(), box_lo.size() * sizeof(int4)), "H2D");
  FZ_GCHK(up(d_box_n.p, box_n.data(), box_n.size() * sizeof(int4)), "H2D");
  FZ_GCHK(up(d_btri.p, btri.data(), btri.size() * sizeof(int)), "H2D");
  FZ_GCHK(up(d_bfirst.p, bfirst.data(), bfirst.size() * sizeof(int64_t)), "H2D");
  FZ_GCHK(up(d_map.p, gid2lid.data(), gid2lid.size() * sizeof(int)), "H2D");
  const GridG g{Nx, Ny, Nz, h};
  unsigned band_bits;
  std::memcpy(&band_bits, &band, sizeof(band_bits));
  k_fill<<<1184, 256, 0, s>>>(d_abs.p, N, band_bits);
  FZ_GCHK(cudaGetLastError(), "distance init");
  if (!btri.empty()) {
    k_dist_scatter<<<(unsigned)btri.size(), 256, 0, s>>>(d_abs.p, d_tris.p, d_box_lo.p, d_box_n.p, d_btri.p,
                                                          d_bfirst.p, g);
    FZ_GCHK(cudaGetLastError(), "distance scatter");
  }
  {
    const dim3 tp(32, 4), gr((unsigned)((Ny + 31) / 32), (unsigned)((Nz + 3) / 4));
    k_sign_rows<<<gr, tp, 0, s>>>(d_abs.p, d_S.p, d_tris.p, d_yz.p, ntri, g);
    FZ_GCHK(cudaGetLastError(), "sign rows");
  }
  FZ_GCHK(cudaMemsetAsync(d_oid.p, 0xFF, (size_t)N, s), "memset");
  {
    const dim3 tp(32, 8), gr((unsigned)((Nx + 31) / 32), (unsigned)((Ny + 7) / 8), (unsigned)Nz);
    const float tol = (float)tol_cells * h;  // main3D.cu:224: tol = 3.0f * h
    k_oid<<<gr, tp, 0, s>>>(d_S.p, d_oid.p, d_tris.p, d_blo.p, d_bhi.p, ntri, d_map.p, max_gid, g, tol);
    FZ_GCHK(cudaGetLastError(), "material ids");
  }
  FZ_GCHK(cudaMemcpyAsync(S_out, d_S.p, (size_t)N * sizeof(float), cudaMemcpyDeviceToHost, s), "D2H");
  FZ_GCHK(cudaMemcpyAsync(oid_out, d_oid.p, (size_t)N, cudaMemcpyDeviceToHost, s), "D2H");
  FZ_GCHK(cudaStreamSynchronize(s), "geometry build");
  return FZ_OK;
}

}  // namespace

namespace fzi {
// Layer (group) names of an OBJ in material order, the grouping of the geometry builder.
int obj_groups(const std::string& path, std::vector<std::string>& names, std::string& err) {
  Mesh m;
  const int rc = read_mesh(path, m, err);
  if (rc == FZ_OK) names = m.groups;
  return rc;
}
}  // namespace fzi

extern "C" {

int fz_scene_dims(const char* obj_path, double h, int32_t* dims, double* L) {
  if (!obj_path || !dims || !(h > 0)) return fzi::set_global_error(FZ_EINVAL, "fz_scene_dims: bad arguments");
  int d[3];
  float Lf[3];
  const int rc = build(obj_path, h, 3.0, -1, nullptr, nullptr, 0, d, Lf);
  if (rc != FZ_OK) return rc;
  for (int a = 0; a < 3; a++) {
    dims[a] = d[a];
    if (L) L[a] = Lf[a];
  }
  return FZ_OK;
}

int fz_build_scene(const char* obj_path, double h, double tol_cells, int32_t device, float* S, uint8_t* oid,
                   int64_t cap) {
  fz_range nvtx_range("fz_build_scene");
  if (!obj_path || !(h > 0) || !(tol_cells > 0) || !S || !oid)
    return fzi::set_global_error(FZ_EINVAL, "fz_build_scene: bad arguments");
  int d[3];
  float Lf[3];
  return build(obj_path, h, tol_cells, device, S, oid, cap, d, Lf);
}

}  // extern "C"
