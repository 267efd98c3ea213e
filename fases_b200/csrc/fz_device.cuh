// fz_device.cuh -- device-side types shared by the stepping kernels.
#pragma once
#include <cuda.h>  // CUtensorMap (type only; the driver entry point is fetched at run time)
#include <cuda_runtime.h>
#include <stdint.h>

namespace fz {

// Device grid layout. Cell (i,j,k) of the padded reference grid (ghost band of 3 cells,
// 3D-solver/include/parsing3D.h:128) lives at XOFF + i + Sx*(j + Ny*k). XOFF = 29 puts the first
// updated cell (i = 3) on a 128-byte boundary, and Sx is a multiple of 32 elements, so every
// warp-wide row segment of a stage tile is one aligned 128-byte line (FP32).
constexpr int XOFF = 29;
constexpr int GHOST = 3;

// Stage-kernel tile: 32 x 16 cells per CTA, one thread per (i, j) column, streaming along z
// (build options FZ_TX = 16 / FZ_TY = 8 select the other measured tile shapes).
#ifndef FZ_TX
#define FZ_TX 32
#endif
#ifndef FZ_TY
#define FZ_TY 16
#endif
constexpr int TX = FZ_TX;
constexpr int TY = FZ_TY;
static_assert(TX == 32 || (TX == 16 && TY % 4 == 0), "stage tile: 32 x TY, or 16 x TY with TY a multiple of 4");
constexpr int HX = 4;  // x halo held in shared memory (3 needed; 4 keeps rows 16-byte aligned)
constexpr int HY = 3;  // y halo
constexpr int PW = TX + 2 * HX;  // 40 tile columns
constexpr int PH = TY + 2 * HY;  // 22 tile rows
constexpr int NTHREADS = TX * TY;
// The adjoint stage kernel's tile (its shared-memory layout and work split are written for it).
constexpr int ATX = 32, ATY = 16, ANTHREADS = ATX * ATY;
constexpr int NBUF = 3;  // plane tiles in flight (TMA ring)

// Cell-class bits (one byte per cell, replaces the reference's 4-byte S read per stage).
constexpr uint8_t CLS_UPDATE = 1;  // interior cell with S >= h: written by the stage kernels
constexpr uint8_t CLS_SOURCE = 2;  // a point source sits here
constexpr uint8_t CLS_BAND = 4;    // an immersed band cell (written by the band kernel)

// Per-axis cPML coefficients at one index along the axis (functions3D.cuh:681-756), precomputed
// on the host once instead of powf/expf per cell and stage.
template <class R>
struct PmlCoef {
  int32_t tile;  // index in the 2d-thick psi tile along this axis, -1 outside the band
  R kinv1;       // 1/kappa - 1
  R b;           // exp(-(alpha + sigma/kappa) dt)
  R ca;          // sigma/(kappa (sigma + kappa alpha)) (b - 1), 0 where sigma = 0
};

template <class R>
struct Pair;
template <>
struct Pair<float> {
  typedef float2 T;
};
template <>
struct Pair<double> {
  typedef double2 T;
};

// Arguments of one stage launch.
constexpr int FZ_MAX_ZCHUNKS = 256;  // z chunks per member a stage launch can have

template <class R>
struct StageArgs {
  typedef typename Pair<R>::T P;
  const R* pi;  // stage input U_in
  const R* ui;
  const R* vi;
  const R* wi;
  const R* pb;  // U0 (stages 1 and 2)
  const R* ub;
  const R* vb;
  const R* wb;
  R* po;  // stage output
  R* uo;
  R* vo;
  R* wo;
  const uint8_t* cls;
  int32_t Nx, Ny, Nz;
  int64_t Sx;     // row pitch (elements)
  int64_t plane;  // Sx * Ny
  int32_t kz_chunk;  // largest z chunk (planes per CTA)
  int32_t zchunks;   // z chunks per batch member: blockIdx.z = member * zchunks + chunk
  // chunk c of a member covers its interior planes [zoff[c], zoff[c+1]) (counted from the first
  // interior plane); chunks may differ in length (long ones first, short ones for the last waves)
  int32_t zoff[FZ_MAX_ZCHUNKS + 1];
  R dt_h;   // dt / h
  R frc2;   // 0.5 * rho * c^2
  R firho;  // 0.5 / rho
  R fc;     // 0.5 * c
  R inv_h;  // 1 / h
  R wdt;    // stage weight * dt (cPML correction weight)
  // cPML (pml_on = 0: no face enabled)
  int32_t pml_on;
  int32_t pml_d2;  // 2 * pml_cells
  const PmlCoef<R>* pcx;
  const PmlCoef<R>* pcy;
  const PmlCoef<R>* pcz;
  P* psix;  // (psi_px, psi_ux) pairs [2d x Ny x Nz]
  P* psiy;  // (psi_py, psi_vy) pairs [Nx x 2d x Nz]
  P* psiz;  // (psi_pz, psi_wz) pairs [Nx x Ny x 2d]
  // sources
  int32_t nsrc;
  const int64_t* src_cell;  // device index
  const R* src_coef;        // dt c^2 sval rho A_s / h^3
  const R* src_freq;
  const R* u_s;
  int64_t n_us;
  int32_t src_opt;
  R src_w;      // stage weight of the injection (1, 1/4, 2/3)
  int32_t nn_mul, nn_add;  // nn = nn_mul * n + nn_add
  R half_dt;
  const int64_t* step;  // device step counter n
  int32_t* err;         // set to a nonzero FZ_KERR_* code when a bounded wait gives up
  // array sizes for the bounds-checked build: elements of one field array (all members), of the
  // psi tiles per axis, of the cPML tables per axis
  int64_t nfield;
  int64_t npsi[3];
  int64_t npc[3];
  // wait-test build only (-DFZ_WAIT_TEST): plane index of each chunk whose tile is never issued,
  // so that the bounded wait for it runs out (-1: none)
  int32_t test_skip_plane;
};

// Kernel error codes written to the handle's device error word.
constexpr int32_t KERR_TMA_TIMEOUT = 1;
constexpr int32_t KERR_NONFINITE = 2;  // a receiver sampled NaN or Inf (the solution blew up)
constexpr int32_t KERR_BOUNDS = 4;     // the bounds-checked build caught an index outside its array

// Index check of the bounds-checked build (compiled with -DFZ_BOUNDS_CHECK): an index outside
// [0, n) sets KERR_BOUNDS in the error word and the access is skipped. In the normal build the
// check is the constant true and costs nothing.
#if defined(__CUDACC__)
__device__ __forceinline__ bool fz_inb(int32_t* err, int64_t i, int64_t n) {
#ifdef FZ_BOUNDS_CHECK
  if (i < 0 || i >= n) {
    atomicOr(err, KERR_BOUNDS);
    return false;
  }
#else
  (void)err;
  (void)i;
  (void)n;
#endif
  return true;
}
#endif

// TMA descriptors of one stage launch: the stage-input fields p, u, v as halo tiles
// (PW x PH x 1), the base state U0 as own tiles (TX x TY x 1; stages 1 and 2) and the class bytes
// as an own tile.
struct StageMaps {
  CUtensorMap p, u, v;
  CUtensorMap bp, bu, bv, bw;
  CUtensorMap cls;
};

// Immersed band cells (compact list in the reference's build_boundary_map order).
template <class R>
struct BandArgs {
  int64_t nB;
  const int4* rec;  // per band cell: device index (lo, hi 32 bits), corner - cell, material (oid - 1)
  const R* geo;     // [4*nB]: sx, sy, sz, chi
  const R* nrm;     // [4*nB]: nx, ny, nz, unused
  const R* pi;            // stage input (probe source)
  const R* ui;
  const R* vi;
  const R* wi;
  R* po;  // stage output (blended in place)
  R* uo;
  R* vo;
  R* wo;
  int64_t Sx, plane;
  double Z0, dt;
  int32_t K, L;
  const double* Rinf;
  const double* A;
  const double* zeta;
  const double* B;
  const double* C;
  const double* alpha;
  const double* beta;
  // ADE states, state q of band cell b at [q*nB + b]
  double* phL;
  const double* phM;
  const double* phR;
  double* s1L;
  const double* s1M;
  const double* s1R;
  double* s2L;
  const double* s2M;
  const double* s2R;
  int32_t* err;    // device error word (bounds-checked build)
  int64_t nfield;  // elements of one field array (bounds-checked build)
};

// Receiver gather of one room (the arguments of its receiver kernel).
template <class R>
struct RecArgs {
  const R* p;
  const R* u;
  const R* v;
  const R* w;
  const int64_t* rcell;
  int32_t nrec;
  double* ir;
  double* vel;
  int64_t cap;
  int64_t* step;
  int32_t* err;
  int64_t nfield;
};

// Groups of rooms stepped by one launch per kernel kind (see k_stage_group).
constexpr int FZ_MAX_GROUP = 64;

// Members one stage launch of a group covers: their TMA descriptors travel as kernel parameters
// (1 KB each; kernel parameters may take up to 32 KB), the rest of their arguments in device memory.
constexpr int FZ_GROUP_LAUNCH = 28;

template <class R>
struct GroupStageArgs {
  StageMaps maps[FZ_GROUP_LAUNCH];  // member m's TMA descriptors (parameter space, as a one-room launch)
  const StageArgs<R>* args;  // [n] in device memory: each member's stage arguments
  int32_t n;
  int32_t cta_start[FZ_GROUP_LAUNCH + 1];  // first CTA of member m in this launch's grid; [n] = total
  int32_t gx[FZ_GROUP_LAUNCH], gy[FZ_GROUP_LAUNCH];  // member m's tiles along x and y
};

template <class R>
struct GroupBandArgs {
  const BandArgs<R>* args;  // [n] in device memory
  int32_t n;
  int32_t blk_start[FZ_MAX_GROUP + 1];  // first 256-thread block of member m; [n] = total
};

}  // namespace fz
