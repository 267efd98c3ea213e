// fz_project.cpp -- the reference's project files: positional config.txt, poles.txt, .fit
// material files, src.txt / rec.txt, OBJ layer names, the S.bin/oid.bin scene cache; and the
// output files IR/VEL/header.txt/pre_header.txt/p_ref.bin that common/*.py consume.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "fz_internal.h"

using fzi::set_error;
using fzi::set_global_error;

namespace {

bool file_exists(const std::string& p) {
  std::ifstream f(p);
  return f.good();
}

std::string dirname_of(const std::string& p) {
  const size_t s = p.find_last_of('/');
  return (s == std::string::npos) ? std::string(".") : p.substr(0, s);
}

std::string basename_of(const std::string& p) {
  const size_t s = p.find_last_of('/');
  return (s == std::string::npos) ? p : p.substr(s + 1);
}

// config.txt, 3D rule (main3D.cu:115-127): '#' starts a comment; a line contributes its first
// number; lines without a number are skipped. Values are floats.
bool read_config(const std::string& path, std::vector<float>& out) {
  std::ifstream f(path);
  if (!f.is_open()) return false;
  std::string line;
  while (std::getline(f, line)) {
    const size_t h = line.find('#');
    if (h != std::string::npos) line.erase(h);
    std::istringstream iss(line);
    float v;
    if (iss >> v) out.push_back(v);
  }
  return true;
}

// Skips whitespace and full-line '#' comments (common/filterABC.h:7-22).
void skip_to_data(std::istream& in) {
  for (;;) {
    in >> std::ws;
    const int c = in.peek();
    if (c == '#') {
      std::string dummy;
      std::getline(in, dummy);
      continue;
    }
    break;
  }
}

// One .fit file (common/filterABC.h:31-90): R_inf; K L; K rows "A zeta"; L rows "B C alpha beta".
// Values are stored as the reference stores them (float). Missing poles stay zero.
int read_fit(const std::string& fn, int m, int Km, int Lm, std::vector<double>& Rinf, std::vector<double>& A,
             std::vector<double>& zeta, std::vector<double>& B, std::vector<double>& C,
             std::vector<double>& alpha, std::vector<double>& beta, std::string& err) {
  std::ifstream in(fn);
  if (!in.is_open()) {
    err = "Cannot open file: " + fn;
    return FZ_EIO;
  }
  float r = 0.f;
  int K = 0, L = 0;
  skip_to_data(in);
  if (!(in >> r)) { err = "Parse failed while reading R_inf from file: " + fn; return FZ_EPARSE; }
  Rinf[m] = r;
  skip_to_data(in);
  if (!(in >> K >> L)) { err = "Parse failed while reading K L from file: " + fn; return FZ_EPARSE; }
  if (K < 0 || K > Km) {
    err = "Invalid K_local=" + std::to_string(K) + " (K_m=" + std::to_string(Km) + ") in file: " + fn;
    return FZ_EPARSE;
  }
  if (L < 0 || L > Lm) {
    err = "Invalid L_local=" + std::to_string(L) + " (L_m=" + std::to_string(Lm) + ") in file: " + fn;
    return FZ_EPARSE;
  }
  skip_to_data(in);
  for (int k = 0; k < K; k++) {
    float a, z;
    if (!(in >> a >> z)) { err = "Parse failed while reading A_k zeta_k row " + std::to_string(k) + " from file: " + fn; return FZ_EPARSE; }
    A[(size_t)m * Km + k] = a;
    zeta[(size_t)m * Km + k] = z;
  }
  skip_to_data(in);
  for (int l = 0; l < L; l++) {
    float b, c, al, be;
    if (!(in >> b >> c >> al >> be)) {
      err = "Parse failed while reading B_l C_l alpha_l beta_l row " + std::to_string(l) + " from file: " + fn;
      return FZ_EPARSE;
    }
    const size_t o = (size_t)m * Lm + l;
    B[o] = b; C[o] = c; alpha[o] = al; beta[o] = be;
  }
  return FZ_OK;
}

// OBJ layer (group) names in material order (3D-solver/include/parsing3D.h:169-288): o/g lines
// set a pending name ("g Mesh1 ceiling Model" -> "ceiling"); a layer is created at its first face
// and reused when the name repeats. Layer m (0-based) is material m, oid m+1.
int read_obj_layers(const std::string& path, std::vector<std::string>& names, std::string& err) {
  std::ifstream in(path);
  if (!in) { err = "Could not open OBJ: " + path; return FZ_EIO; }
  std::unordered_map<std::string, int> ids;
  std::string cur = "unnamed";
  bool have = false, pending = true;
  std::string line;
  auto trim = [](std::string& s) {
    while (!s.empty() && std::strchr(" \t\r\n", s.front())) s.erase(s.begin());
    while (!s.empty() && std::strchr(" \t\r\n", s.back())) s.pop_back();
  };
  while (std::getline(in, line)) {
    trim(line);
    if (line.empty() || line[0] == '#') continue;
    if (line.rfind("o ", 0) == 0 || line.rfind("g ", 0) == 0) {
      std::istringstream ss(line);
      std::string tag, tok;
      ss >> tag;
      std::vector<std::string> parts;
      while (ss >> tok) parts.push_back(tok);
      std::string nm = parts.size() >= 2 ? parts[1] : (parts.size() == 1 ? parts[0] : "unnamed");
      if (!have || nm != cur) { cur = nm; have = true; pending = true; }
    } else if (line.rfind("f ", 0) == 0) {
      std::istringstream ss(line);
      std::string tag, tok;
      ss >> tag;
      int nv = 0;
      while (ss >> tok) nv++;
      if (nv < 3) continue;
      if (pending) {
        const std::string nm = have ? cur : std::string("unnamed");
        if (!ids.count(nm)) { ids[nm] = (int)names.size(); names.push_back(nm); }
        pending = false;
      }
    }
  }
  return FZ_OK;
}

}  // namespace

extern "C" {

int fz_source_waveform(int32_t src_opt, double glob_f, double f_cutoff, double dt, int64_t Nt, double h,
                       double rho, double* u_s, double* p_ref, double* p_peak) {
  if (Nt < 1 || !(dt > 0) || !(h > 0)) return set_global_error(FZ_EINVAL, "fz_source_waveform: bad arguments");
  const int64_t n = 2 * Nt + 1;
  std::vector<double> us((size_t)n, 0.0);
  const double dth = 0.5 * dt;
  if (src_opt == FZ_SRC_PCS) {
    // Physically constrained source (Sheaffer, van Walstijn & Fazenda 2012), main3D.cu:971-1035:
    // Gaussian force through the bilinear-transformed mass-spring-damper (M = 0.025 kg, Q = 1).
    if (!(glob_f > 0) || !(f_cutoff > 0)) return set_global_error(FZ_EINVAL, "fz_source_waveform: PCS needs f0, f_cutoff > 0");
    const double Q = 1.0, w0 = 2.0 * M_PI * glob_f;
    const double bs = w0 / std::tan(0.5 * w0 * dth);
    const double M = 0.025, Rs = w0 * M / Q, Ks = M * w0 * w0;
    const double den = M * bs * bs + Rs * bs + Ks;
    const double b0 = bs / den, b2 = -b0;
    const double a1 = 2.0 * (Ks - M * bs * bs) / den, a2 = 1.0 - 2.0 * Rs * bs / den;
    const double sig = 0.425 / f_cutoff;
    const int ts = (int)std::ceil(8.5 * sig / dth);
    std::vector<double> F((size_t)n);
    for (int64_t t = 0; t < n; t++) {
      const double td = (double)(t - ts) * dth;
      F[(size_t)t] = std::exp(-td * td / (2.0 * sig * sig));
    }
    for (int64_t t = 2; t < n; t++)
      us[(size_t)t] = b0 * F[(size_t)t] + b2 * F[(size_t)t - 2] - a1 * us[(size_t)t - 1] - a2 * us[(size_t)t - 2];
  } else if (src_opt == FZ_SRC_RICKER) {
    // Antiderivative of a Ricker wavelet, peak frequency glob_f (main3D.cu:1036-1059).
    if (!(glob_f > 0)) return set_global_error(FZ_EINVAL, "fz_source_waveform: Ricker needs f0 > 0");
    const double sig = 1.0 / (std::sqrt(2.0) * M_PI * glob_f);
    const double ts = (int)std::ceil(5.0 * sig / dth);
    for (int64_t t = 0; t < n; t++) {
      const double x = ((double)t - ts) * dth / sig;
      us[(size_t)t] = x * std::exp(-0.5 * x * x);
    }
  } else {
    return set_global_error(FZ_EINVAL, "fz_source_waveform: src_opt must be PCS (0) or Ricker (1)");
  }
  // radiated pulse at 1 m per unit strength (main3D.cu:1081-1090)
  const double As = 6.0 * h * h;
  double peak = 0.0;
  std::vector<double> pr((size_t)n, 0.0);
  for (int64_t t = 1; t < n - 1; t++) {
    const double dq = As * (us[(size_t)t + 1] - us[(size_t)t - 1]) / (2.0 * dth);
    pr[(size_t)t] = rho * dq / (4.0 * M_PI);
    peak = std::max(peak, std::fabs(pr[(size_t)t]));
  }
  if (u_s) std::copy(us.begin(), us.end(), u_s);
  if (p_ref) std::copy(pr.begin(), pr.end(), p_ref);
  if (p_peak) *p_peak = peak;
  return FZ_OK;
}

int fz_write_outputs(fz_handle* h, const char* output_dir, int32_t src_idx, const char* scene_name) {
  if (!h || !output_dir) return set_global_error(FZ_EINVAL, "fz_write_outputs: NULL argument");
  int64_t n = 0;
  int rc = fz_steps_done(h, &n);
  if (rc != FZ_OK) return rc;
  n = std::min(n, h->rec_cap);
  const std::string dir(output_dir);
  // batch member m writes the traces of source index src_idx + m
  const int rows = h->nrec * h->nb;
  std::vector<float> ir((size_t)rows * n), vel((size_t)rows * n * 3);
  if (rows > 0 && n > 0) {
    rc = fz_get_ir(h, ir.data(), (int64_t)ir.size());
    if (rc != FZ_OK) return rc;
    rc = fz_get_vel(h, vel.data(), (int64_t)vel.size());
    if (rc != FZ_OK) return rc;
  }
  // IR<rec>_<src>.bin: float32 p per step; VEL<rec>_<src>.bin: float32 (u,v,w) per step
  // (main3D.cu:1251-1256, 1403-1412)
  for (int r = 0; r < rows; r++) {
    const std::string tag = std::to_string(r % h->nrec) + "_" + std::to_string(src_idx + r / h->nrec) + ".bin";
    const std::string f1 = dir + "/IR" + tag;
    const std::string f2 = dir + "/VEL" + tag;
    FILE* a = std::fopen(f1.c_str(), "wb");
    FILE* b = std::fopen(f2.c_str(), "wb");
    if (!a || !b) {
      if (a) std::fclose(a);
      if (b) std::fclose(b);
      return set_error(h, FZ_EIO, "cannot write " + f1);
    }
    std::fwrite(ir.data() + (size_t)r * n, sizeof(float), (size_t)n, a);
    std::fwrite(vel.data() + (size_t)r * n * 3, sizeof(float), (size_t)n * 3, b);
    std::fclose(a);
    std::fclose(b);
  }
  // animation slices (main3D.cu:1206-1235, 1337-1393): pressure{X,Y,Z}.bin and the in-plane unit
  // energy-flow components I{y,z}_X, I{x,z}_Y, I{x,y}_Z, one frame after another
  int64_t pbin = 0, anim_step = 1;
  if (h->sl_on) {
    int64_t nf = 0;
    rc = fz_get_slices(h, nullptr, 0, &nf);
    if (rc != FZ_OK) return rc;
    std::vector<float> fr((size_t)(nf * h->sl_frame));
    if (nf > 0) {
      rc = fz_get_slices(h, fr.data(), (int64_t)fr.size(), &nf);
      if (rc != FZ_OK) return rc;
    }
    const int64_t nX = (int64_t)h->Ny * h->Nz, nY = (int64_t)h->Nx * h->Nz, nZ = (int64_t)h->Nx * h->Ny;
    const int64_t tot = nX + nY + nZ;
    // file, offset in the frame, plane size
    const struct { const char* name; int64_t off, len; } files[9] = {
        {"pressureX.bin", 0, nX},          {"pressureY.bin", nX, nY},          {"pressureZ.bin", nX + nY, nZ},
        {"Iy_X.bin", tot, nX},             {"Iz_X.bin", tot + nX, nX},         {"Ix_Y.bin", tot + 2 * nX, nY},
        {"Iz_Y.bin", tot + 2 * nX + nY, nY}, {"Ix_Z.bin", tot + 2 * nX + 2 * nY, nZ},
        {"Iy_Z.bin", tot + 2 * nX + 2 * nY + nZ, nZ}};
    for (const auto& fl : files) {
      const std::string fn = dir + "/" + fl.name;
      FILE* fo = std::fopen(fn.c_str(), "wb");
      if (!fo) return set_error(h, FZ_EIO, "cannot write " + fn);
      for (int64_t q = 0; q < nf; q++) std::fwrite(fr.data() + q * h->sl_frame + fl.off, sizeof(float), (size_t)fl.len, fo);
      std::fclose(fo);
    }
    pbin = nf;
    anim_step = h->sl_step;
  } else {
    const int64_t frames = std::max<int64_t>(1, std::min<int64_t>(300, n));
    anim_step = std::max<int64_t>(1, n / frames);
  }
  // header.txt (main3D.cu:1441-1449): Nx Ny Nz Nt Lx Ly Lz pbin anim_step dt scene h tol/h
  const std::string hdr = dir + "/header.txt";
  FILE* f = std::fopen(hdr.c_str(), "w");
  if (!f) return set_error(h, FZ_EIO, "cannot write " + hdr);
  const std::string scene = scene_name ? std::string(scene_name) : h->scene_name;
  std::fprintf(f, "%d %d %d %d %f %f %f %d %d %f %s %f %d\n", h->Nx, h->Ny, h->Nz, (int)n, (float)h->Lx,
               (float)h->Ly, (float)h->Lz, (int)pbin, (int)anim_step, (float)h->prm.dt, scene.c_str(),
               (float)h->prm.h, (int)(h->prm.tol_cells * h->prm.h / h->prm.h));
  std::fclose(f);
  return FZ_OK;
}

int fz_load_project(const char* scene_path, const char* config_path, const char* src_path, const char* rec_path,
                    int32_t precision, int32_t device, fz_handle** out, int64_t* n_steps_out) {
  fz_range nvtx_range("fz_load_project");
  if (!scene_path || !config_path || !src_path || !rec_path || !out)
    return set_global_error(FZ_EINVAL, "fz_load_project: NULL argument");
  *out = nullptr;
  const std::string cfg_path(config_path);
  // project layout (main3D.cu:77-87)
  const std::string cfg_dir = dirname_of(cfg_path);
  std::string root = ".";
  if (basename_of(cfg_path) == "config.txt" && basename_of(cfg_dir) == "config") root = dirname_of(cfg_dir);
  const std::string poles_path = cfg_dir + "/poles.txt";
  const std::string fit_dir = root + "/input/fit";
  const std::string out_dir = root + "/output";

  std::vector<float> conf;
  if (!read_config(cfg_path, conf)) return set_global_error(FZ_EIO, "cannot open config: " + cfg_path);
  if (conf.size() < 12)
    return set_global_error(FZ_EPARSE, "config.txt needs at least 12 values (h, t_max, f, T, CFL, poles, 6 PML keys)");
  // scalars exactly as main3D.cu computes them (float arithmetic)
  const float h = conf[0], t_max = conf[1], f_in = conf[2];
  float f_x = f_in;
  const float oct[8] = {63.f, 125.f, 250.f, 500.f, 1000.f, 2000.f, 4000.f, 8000.f};
  for (int b = 0; b < 8; b++) {
    const float hi = oct[b] * 1.41421356f;
    if (f_in <= hi) { f_x = hi; break; }
  }
  const float f_cutoff = 2.0f * f_x;
  const float rho = 1.225f;
  const float Temp = conf[3] + 273.15f;
  const float c = std::sqrt(1.4f * 287.05f * Temp);
  const float CFL = conf[4];
  const float dt = CFL * h / c;
  const int64_t Nt = (int64_t)(t_max / dt) + 1;
  const int src_opt = (conf.size() > 15) ? (int)conf[15] : 0;
  const float glob_f = (conf.size() > 16) ? conf[16] : (src_opt == 0 ? 25.0f : 0.5f * f_cutoff);

  fz_params p;
  fz_params_init(&p);
  p.precision = precision;
  p.device = device;
  p.h = h;
  p.c = c;
  p.rho = rho;
  p.dt = dt;
  // U D R L F B = config lines 7..12 (main3D.cu:155-160)
  for (int f = 0; f < 6; f++) p.pml[f] = (conf[6 + f] != 0.0f) ? 1 : 0;

  // scene cache (main3D.cu:334-428): output/S.bin and output/oid.bin, valid while the first line of
  // output/scene_cache.txt carries the key "<scene path> <scene mtime> <h> <tol>" (the path made
  // absolute and normal, main3D.cu:66-72); otherwise the geometry is built from the OBJ on the
  // device and the cache is rewritten, dims and domain size on its second line
  namespace fs = std::filesystem;
  fs::path sp(scene_path);
  if (sp.is_relative()) sp = fs::current_path() / sp;
  sp = sp.lexically_normal();
  const float tol = 3.0f * h;
  std::error_code fec;
  std::ostringstream key_s;
  key_s << sp.string() << " " << fs::last_write_time(sp, fec).time_since_epoch().count() << " " << h << " " << tol;
  const std::string cache_key = key_s.str();
  std::string key;
  int Nx = 0, Ny = 0, Nz = 0;
  float Lx = 0, Ly = 0, Lz = 0;
  std::vector<float> S;
  std::vector<uint8_t> oid;
  bool cached = false;
  {
    std::ifstream ck(out_dir + "/scene_cache.txt");
    cached = std::getline(ck, key) && key == cache_key && (ck >> Nx >> Ny >> Nz >> Lx >> Ly >> Lz);
  }
  if (cached) {
    const size_t N = (size_t)Nx * Ny * Nz;
    S.resize(N);
    oid.resize(N);
    FILE* fS = std::fopen((out_dir + "/S.bin").c_str(), "rb");
    FILE* fO = std::fopen((out_dir + "/oid.bin").c_str(), "rb");
    cached = fS && fO && std::fread(S.data(), 4, N, fS) == N && std::fread(oid.data(), 1, N, fO) == N;
    if (fS) std::fclose(fS);
    if (fO) std::fclose(fO);
  }
  if (!cached) {
    int32_t dims[3];
    double Ld[3];
    int rc = fz_scene_dims(sp.string().c_str(), h, dims, Ld);
    if (rc != FZ_OK) return rc;
    Nx = dims[0]; Ny = dims[1]; Nz = dims[2];
    Lx = (float)Ld[0]; Ly = (float)Ld[1]; Lz = (float)Ld[2];
    const size_t N = (size_t)Nx * Ny * Nz;
    S.assign(N, 0.f);
    oid.assign(N, 0xFF);
    rc = fz_build_scene(sp.string().c_str(), h, 3.0, device, S.data(), oid.data(), (int64_t)N);
    if (rc != FZ_OK) return rc;
    fs::create_directories(out_dir, fec);
    FILE* fS = std::fopen((out_dir + "/S.bin").c_str(), "wb");
    FILE* fO = std::fopen((out_dir + "/oid.bin").c_str(), "wb");
    const bool ok = fS && fO && std::fwrite(S.data(), 4, N, fS) == N && std::fwrite(oid.data(), 1, N, fO) == N;
    if (fS) std::fclose(fS);
    if (fO) std::fclose(fO);
    if (ok) {  // stamp the cache only after both arrays are written
      std::ofstream(out_dir + "/scene_cache.txt", std::ios::trunc)
          << cache_key << "\n" << Nx << " " << Ny << " " << Nz << " " << Lx << " " << Ly << " " << Lz << "\n";
    }
  }
  // materials: poles.txt (main3D.cu:592-603), layer names from the OBJ, one .fit per layer except
  // BoundingBox-like layers (main3D.cu:624-634)
  int Km = 0, Lm = 0;
  {
    std::ifstream pf(poles_path);
    if (!pf.is_open() || !(pf >> Km >> Lm)) return set_global_error(FZ_EIO, "cannot read poles file: " + poles_path);
    Km = std::max(1, Km);
    Lm = std::max(1, Lm);
  }
  std::vector<std::string> layers;
  std::string err;
  int rc = read_obj_layers(scene_path, layers, err);
  if (rc != FZ_OK) return set_global_error(rc, err);
  const int nMat = (int)layers.size();
  const int nm = std::max(1, nMat);
  std::vector<double> Rinf(nm, 0.0), A((size_t)nm * Km, 0.0), zeta((size_t)nm * Km, 0.0), B((size_t)nm * Lm, 0.0),
      C((size_t)nm * Lm, 0.0), al((size_t)nm * Lm, 0.0), be((size_t)nm * Lm, 0.0);
  for (int m = 0; m < nMat; m++) {
    const std::string& nmn = layers[(size_t)m];
    if (nmn.find("ounding") != std::string::npos || nmn.find("oundary") != std::string::npos) continue;
    rc = read_fit(fit_dir + "/" + nmn + ".fit", m, Km, Lm, Rinf, A, zeta, B, C, al, be, err);
    if (rc != FZ_OK) return set_global_error(rc, err);
  }
  // sources (main3D.cu:861-906) and receivers (928-959)
  std::vector<int32_t> sijk, rijk;
  std::vector<float> spress, sfreq;
  {
    std::ifstream sf(src_path);
    if (!sf.is_open()) return set_global_error(FZ_EIO, std::string("Failed to open sources: ") + src_path);
    std::string line;
    while (std::getline(sf, line)) {
      if (line.empty() || line[0] == '#') continue;
      std::istringstream iss(line);
      float x, y, z, s, f0;
      if (iss >> x >> y >> z >> s) {
        if (!(iss >> f0)) f0 = 0.5f * f_cutoff;
        const int i = (int)(x / h) + 3, j = (int)(y / h) + 3, k = (int)(z / h) + 3;
        if (i >= 0 && i < Nx && j >= 0 && j < Ny && k >= 0 && k < Nz) {
          sijk.push_back(i); sijk.push_back(j); sijk.push_back(k);
          spress.push_back((float)(2e-5 * (double)powf(10.0f, (float)(s / 20.0))));
          sfreq.push_back(f0);
        }
      }
    }
  }
  {
    std::ifstream rf(rec_path);
    if (!rf.is_open()) return set_global_error(FZ_EIO, std::string("Failed to open receivers: ") + rec_path);
    std::string line;
    while (std::getline(rf, line)) {
      if (line.empty() || line[0] == '#') continue;
      std::istringstream iss(line);
      float x, y, z;
      if (iss >> x >> y >> z) {
        const int i = (int)(x / h) + 3, j = (int)(y / h) + 3, k = (int)(z / h) + 3;
        if (!(i >= 0 && i < Nx && j >= 0 && j < Ny && k >= 0 && k < Nz))
          return set_global_error(FZ_EINVAL, "Receiver(s) outside domain");
        rijk.push_back(i); rijk.push_back(j); rijk.push_back(k);
      }
    }
  }
  const int nsrc = (int)spress.size();
  // waveform and scaling (main3D.cu:963-1124)
  std::vector<double> us((size_t)(2 * Nt + 1), 0.0), pref((size_t)(2 * Nt + 1), 0.0);
  const double As = 6.0 * (double)h * (double)h;
  if (src_opt == 2) {
    for (int s = 0; s < nsrc; s++) {
      const double pk = (double)rho * As * (double)sfreq[(size_t)s] / 2.0;
      if (pk > 0.0) spress[(size_t)s] /= (float)pk;
    }
  } else {
    double peak = 0.0;
    rc = fz_source_waveform(src_opt, glob_f, f_cutoff, dt, Nt, h, rho, us.data(), pref.data(), &peak);
    if (rc != FZ_OK) return rc;
    for (int s = 0; s < nsrc; s++) spress[(size_t)s] /= (float)peak;
    if (nsrc > 0) {
      std::vector<double> tmp(pref.size());
      for (size_t t = 0; t < pref.size(); t++) tmp[t] = pref[t] * (double)spress[0] / 1.0;
      FILE* fp = std::fopen((cfg_dir + "/p_ref.bin").c_str(), "wb");
      if (!fp) return set_global_error(FZ_EIO, "cannot write p_ref.bin");
      std::fwrite(tmp.data(), sizeof(double), tmp.size(), fp);
      std::fclose(fp);
    }
  }
  // waveform as the reference stores it on the device (float, main3D.cu:1122)
  for (auto& x : us) x = (double)(float)x;
  // pre_header.txt (main3D.cu:527-532)
  {
    FILE* ph = std::fopen((out_dir + "/pre_header.txt").c_str(), "w");
    if (ph) {
      std::fprintf(ph, "%d %d %d %f %d\n", Nx, Ny, Nz, h, (int)(3.0f * h / h));
      std::fclose(ph);
    }
  }
  fz_handle* H = nullptr;
  rc = fz_create(&p, &H);
  if (rc != FZ_OK) return rc;
  H->Lx = Lx; H->Ly = Ly; H->Lz = Lz;
  H->scene_name = sp.string();  // header.txt carries the absolute scene path (main3D.cu:1445)
  rc = fz_load_geometry_raw(H, S.data(), oid.data(), Nx, Ny, Nz);
  std::vector<double> sv(spress.begin(), spress.end()), sfr(sfreq.begin(), sfreq.end());
  if (rc == FZ_OK) rc = fz_set_materials(H, nMat, Km, Lm, Rinf.data(), A.data(), zeta.data(), B.data(), C.data(), al.data(), be.data());
  if (rc == FZ_OK)
    rc = fz_set_sources(H, nsrc, sijk.data(), sv.data(), src_opt, sfr.data(), src_opt == 2 ? nullptr : us.data(),
                        src_opt == 2 ? 0 : (int64_t)us.size());
  if (rc == FZ_OK) rc = fz_set_receivers(H, (int)(rijk.size() / 3), rijk.data(), Nt);
  // animation slices (main3D.cu:1152-1199): planes at config lines 19-21 ((int)(x/h) + 3), frames
  // from line 22 (default 300, at least 60, at most Nt), every Nt / frames steps. The reference caps
  // the frames by 85 % of host RAM; here they are kept in device memory, capped at a quarter of it.
  if (rc == FZ_OK && conf.size() > 20) {
    const int si = (int)(conf[18] / h) + 3, sj = (int)(conf[19] / h) + 3, sk = (int)(conf[20] / h) + 3;
    if (si >= 0 && si < Nx && sj >= 0 && sj < Ny && sk >= 0 && sk < Nz) {
      int64_t wanted = (conf.size() > 21 && conf[21] > 0) ? (int64_t)conf[21] : 300;
      wanted = std::max<int64_t>(wanted, 60);
      const int64_t per_frame = 3 * 4 * ((int64_t)Ny * Nz + (int64_t)Nx * Nz + (int64_t)Nx * Ny);
      size_t fr = 0, tot = 0;
      cudaMemGetInfo(&fr, &tot);
      int64_t frames = std::min<int64_t>(wanted, std::max<int64_t>(1, (int64_t)(fr / 4) / per_frame));
      frames = std::min<int64_t>(frames, Nt);
      const int64_t anim_step = std::max<int64_t>(1, Nt / std::max<int64_t>(frames, 1));
      // the time loop writes a frame at every step index n < Nt that anim_step divides
      // (main3D.cu:1337, 1393): ceil(Nt / anim_step) of them, one more than Nt / anim_step when
      // anim_step does not divide Nt
      frames = (Nt + anim_step - 1) / anim_step;
      rc = fz_set_slices(H, si, sj, sk, anim_step, frames);
    }
  }
  if (rc != FZ_OK) {
    fzi::set_global_error(rc, H->err);
    fz_destroy(H);
    return rc;
  }
  *out = H;
  if (n_steps_out) *n_steps_out = Nt;
  return FZ_OK;
}

}  // extern "C"
