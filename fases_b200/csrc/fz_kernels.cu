// fz_kernels.cu -- sm_100a stepping kernels of the FASES time-domain solver hot path.
//
// One SSP-RK3 step of the reference (3D-solver/core/main3D.cu:1280-1319) is nine launches there:
// three stage kernels (functions3D.cuh:1086-1327), three source injections (1039-1047) and three
// full-grid immersed-boundary passes (462-565). Here it is seven: three fused stage kernels
// (WENO-Z reconstruction once per face, Godunov flux, RK combination, cPML and source injection
// in one pass), three sparse band kernels that touch only the immersed band cells, and one
// receiver gather.
#include <cuda_runtime.h>
#include <math.h>

#include "fz_device.cuh"
#include "fz_kernels.h"
#include "fz_pair.cuh"

namespace fz {


// ------------------------------------------------------------------------------------------
// TMA and mbarrier primitives (PTX). Plain per-CTA tensor loads, never multicast.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, P;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: gives up after ~2^31 clock cycles (about a second) and reports failure. The
// wait-test build (-DFZ_WAIT_TEST) gives up after 2^21 cycles (about a millisecond), so that a
// test can make a wait run out without a long stall.
#ifdef FZ_WAIT_TEST
constexpr long long kWaitCycles = 1ll << 21;
#else
constexpr long long kWaitCycles = 1ll << 31;
#endif
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > kWaitCycles) return false;
  }
  return true;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y,
                                            int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Error path of the stage kernel (out of line: it must not cost the stepping loop registers).
// Waits, bounded, for the tile copies a block still has in flight when the wait for plane it_fail
// ran out: plane it_fail itself (unless it was never issued: `skipped`) and plane it_fail + 1.
__device__ __noinline__ void drain_ring(uint64_t* mbar, int it_fail, int nplanes, int skipped) {
  const int hi = min(it_fail + 1, nplanes - 1);
  for (int q = it_fail; q <= hi; ++q)
    if (q != skipped) (void)mbar_wait_bounded(&mbar[q % NBUF], (uint32_t)((q / NBUF) & 1));
}

// Shared-memory layout of the stage kernel.
template <class R>
struct StageSmem {
  typedef typename Pair<R>::T P;
  // one field of one plane tile, padded to a multiple of 128 bytes (TMA destinations)
  static constexpr int FIELD = ((PH * PW * (int)sizeof(R) + 127) / 128) * 128;  // halo tile
  static constexpr int OWN = ((TX * TY * (int)sizeof(R) + 127) / 128) * 128;     // own tile
  static constexpr int CLSB = ((TX * TY + 127) / 128) * 128;                     // class bytes
  static constexpr int BUF = 3 * FIELD + 4 * OWN + CLSB;         // p,u,v halo | U0 own | cls
  static constexpr int TILES = NBUF * BUF;
  static constexpr int XC = TY * (TX + 2) * (int)sizeof(P);        // one V array of x-centres
  static constexpr int YC = (TY + 2) * TX * (int)sizeof(P);        // one V array of y-centres
  static constexpr int CENTRES = 2 * (2 * XC + 2 * YC);            // double buffered (m, p) x and y
  static constexpr int BYTES = TILES + CENTRES + 64 + 128;         // + mbarriers + base alignment
};

// ------------------------------------------------------------------------------------------
// Fused stage kernel. CTA = 32 x 16 columns marching in z over one z chunk of planes.
//  - x, y: plane k of p, u, v arrives by TMA into a ring of three shared-memory tiles (with a
//    3-cell halo), issued two planes ahead, so global latency overlaps the arithmetic of the
//    planes in between. Every x- and y-centre is evaluated once (the reference evaluates every
//    face from both sides) and exchanged through a double-buffered shared array: one barrier
//    per plane.
//  - z: a register queue of (p, w) over five planes, refilled one plane ahead; the z-centre of
//    plane k+1 is evaluated once and serves the flux above plane k and (next iteration) below
//    plane k+1.
// STAGE 0: U1 = U0 + dt L(U0); 1: U2 = 3/4 U0 + 1/4 (U1 + dt L(U1)); 2: U1 = (U0 + 2 (U2 + dt L(U2)))/3
// (functions3D.cuh:1149-1152, 1230-1233, 1311-1314), cPML with weights 1, 1/4, 2/3 and the psi
// advance in stage 2 (functions3D.cuh:1157-1162, 1237-1242, 1320-1325), then the point sources of
// the stage (main3D.cu:1288, 1296, 1304).
// ------------------------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ R source_sum(const StageArgs<R>& A, int64_t g) {
  const int64_t n = *A.step;
  const int64_t nn = A.nn_mul * n + A.nn_add;
  R add = R(0);
  for (int s = 0; s < A.nsrc; ++s) {
    if (A.src_cell[s] != g) continue;
    R amp;
    if (A.src_opt == 2) {
      const double ph = 2.0 * 3.14159265358979323846 * (double)A.src_freq[s] * (double)nn * (double)A.half_dt;
      amp = (R)sin(ph);
    } else {
      amp = (nn < A.n_us) ? A.u_s[nn] : R(0);
    }
    add += A.src_w * A.src_coef[s] * amp;
  }
  return add;
}

#ifndef FZ_STAGE_MINBLOCKS_F32
#define FZ_STAGE_MINBLOCKS_F32 (1024 / NTHREADS)  // 32 warps per SM in FP32 (64 registers, no spills)
#endif
// DIM2: planar solve (one updated z-plane, no z fluxes): the 3D scheme restricted to 2D.
// CTA coordinates of a stage-kernel launch of one room: the launch grid itself.
struct GridCta {
  static __device__ __forceinline__ int x() { return blockIdx.x; }
  static __device__ __forceinline__ int y() { return blockIdx.y; }
  static __device__ __forceinline__ int z() { return blockIdx.z; }
};

// The body of one stage-kernel CTA: tile (CTA::x(), CTA::y()) of z chunk slot CTA::z() (batch
// member x chunks) of the room A describes. A and M may live in parameter, shared or global memory.
template <class R, int STAGE, bool DIM2, class CTA>
__device__ __forceinline__ void stage_body(const StageArgs<R>& A, const StageMaps& M) {
  typedef typename Pair<R>::T P;
  typedef StageSmem<R> L;
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  // TMA destinations must be 128-byte aligned: align the base explicitly
  unsigned char* smem_raw = smem_dyn + ((128u - (smem_u32(smem_dyn) & 127u)) & 127u);
  R* tiles = reinterpret_cast<R*>(smem_raw);
  unsigned char* cbase = smem_raw + L::TILES;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem_raw + L::TILES + L::CENTRES);

  const int lt = threadIdx.y * TX + threadIdx.x;  // linear thread index (warps: 32 consecutive)
  // this thread's column (tx, ty) of the tile. 32-wide tiles: a warp is one row. 16-wide tiles: a
  // warp takes rows r and r + 2, whose halo-tile rows (24 floats apart x 2) fall in disjoint
  // halves of the shared-memory banks
  int tx, ty;
  if constexpr (TX == 32) {
    tx = threadIdx.x;
    ty = threadIdx.y;
  } else {
    const int w = lt >> 5, l = lt & 31;
    tx = l & (TX - 1);
    ty = 4 * (w >> 1) + (w & 1) + 2 * (l >> 4);
  }
  const int lo = ty * TX + tx;  // this cell in the own tiles and the class-byte tile
  const int i0 = GHOST + CTA::x() * TX, j0 = GHOST + CTA::y() * TY;
  const int i = i0 + tx, j = j0 + ty;
  // batch members are stacked along z (member m owns planes [m Nz, (m+1) Nz)); the cPML z table,
  // the psi tiles and the class bytes are laid out per member the same way
  const int member = CTA::z() / A.zchunks;
  const int chunk = CTA::z() - member * A.zchunks;
  const int kb = GHOST + member * A.Nz + A.zoff[chunk];
  const int ke = min(GHOST + member * A.Nz + A.zoff[chunk + 1], (member + 1) * A.Nz - GHOST);
  if (kb >= ke) return;
  const int nplanes = ke - kb;
  const int64_t Sx = A.Sx, plane = A.plane;
  const bool col_ok = (j < A.Ny) && (XOFF + i < Sx);
  const int64_t col = XOFF + i + Sx * (int64_t)j;
  const bool valid = (i < A.Nx - GHOST) && (j < A.Ny - GHOST);
  const int tma_x = XOFF + i0 - HX, tma_y = j0 - HY;
  constexpr uint32_t TILE_BYTES = 3u * PH * PW * sizeof(R) + (STAGE > 0 ? 4u * TX * TY * sizeof(R) : 0u) +
                                  (uint32_t)(TX * TY);

  unsigned char* const ring = reinterpret_cast<unsigned char*>(tiles);
  auto field = [&](int buf, int f) -> R* { return reinterpret_cast<R*>(ring + buf * L::BUF + f * L::FIELD); };
  auto own = [&](int buf, int f) -> R* {
    return reinterpret_cast<R*>(ring + buf * L::BUF + 3 * L::FIELD + f * L::OWN);
  };
  auto clsb = [&](int buf) -> uint8_t* { return ring + buf * L::BUF + 3 * L::FIELD + 4 * L::OWN; };
  // plane `it` of the chunk into ring slot it % NBUF (wait-test build: the plane A.test_skip_plane
  // is never issued, so the wait for it runs out)
  auto issue = [&](int it) {
#ifdef FZ_WAIT_TEST
    if (it == A.test_skip_plane) return;
#endif
    const int b = it % NBUF;
    const int z = kb + it;
    mbar_expect_tx(&mbar[b], TILE_BYTES);
    tma_load_3d(field(b, 0), &M.p, &mbar[b], tma_x, tma_y, z);
    tma_load_3d(field(b, 1), &M.u, &mbar[b], tma_x, tma_y, z);
    tma_load_3d(field(b, 2), &M.v, &mbar[b], tma_x, tma_y, z);
    if (STAGE > 0) {
      tma_load_3d(own(b, 0), &M.bp, &mbar[b], tma_x + HX, j0, z);
      tma_load_3d(own(b, 1), &M.bu, &mbar[b], tma_x + HX, j0, z);
      tma_load_3d(own(b, 2), &M.bv, &mbar[b], tma_x + HX, j0, z);
      tma_load_3d(own(b, 3), &M.bw, &mbar[b], tma_x + HX, j0, z);
    }
    tma_load_3d(clsb(b), &M.cls, &mbar[b], tma_x + HX, j0, z);
  };
  // Error path of a wait that ran out: every thread leaves through the same exit after the
  // block-wide barrier (which ORs the threads' failures); thread 0 first waits (bounded, drain_ring) for the copies this block still
  // has in flight -- plane it_fail (if it was issued) and plane it_fail + 1 (issued one iteration
  // earlier; plane it_fail + 2 is issued only after the abort check) -- so that no copy lands in
  // shared memory after the block has gone. If that wait runs out as well, the block exits
  // anyway and the error word already says that the results are invalid.
#if defined(FZ_V_SPLITBAR)
  __shared__ __align__(8) uint64_t cbar[2];  // centre buffers: one arrival per warp
  __shared__ int s_abort;
#endif
  if (lt == 0) {
    for (int b = 0; b < NBUF; ++b) mbar_init(&mbar[b], 1);
#if defined(FZ_V_SPLITBAR)
    mbar_init(&cbar[0], NTHREADS / 32);
    mbar_init(&cbar[1], NTHREADS / 32);
#endif
    fence_mbar_init();
#if defined(FZ_V_SPLITBAR)
    s_abort = 0;
#endif
  }
  __syncthreads();
  if (lt == 0) {
    issue(0);
    if (nplanes > 1) issue(1);
  }

  const P kA = pmk(A.frc2, A.firho);
  const P kC = psplat<R>(-A.fc);

  // z-queue loads: a column outside the grid (a ragged tile edge) reads the grid's last column
  // instead, so the loads need no test; such a thread stores nothing
  const int64_t colz = col_ok ? col : (XOFF + (int64_t)min(i, A.Nx - 1) + Sx * (int64_t)min(j, A.Ny - 1));
  auto ld_pw = [&](int kk) -> P {
    const int64_t g = colz + plane * kk;
    if (!fz_inb(A.err, g, A.nfield)) return psplat<R>(R(0));
    return pmk(A.pi[g], A.wi[g]);
  };

  // z prologue: centres kb-1 and kb give the flux through face kb-1/2 and V-(kb+1/2).
  const P zero = psplat<R>(R(0));
  P qa = zero, qb = zero, qc = zero, qd = zero, qe_next = zero, zm = zero, Fz_lo = zero;
  if (!DIM2) {
    const P z0 = ld_pw(kb - 3), z1 = ld_pw(kb - 2), z2 = ld_pw(kb - 1), z3 = ld_pw(kb), z4 = ld_pw(kb + 1);
    const P z5 = ld_pw(kb + 2);
    qe_next = ld_pw(kb + 3);
    P m0, p0, m1, p1;
    weno_center<R>(z0, z1, z2, z3, z4, m0, p0);
    weno_center<R>(z1, z2, z3, z4, z5, m1, p1);
    Fz_lo = godunov<R>(m0, p1, kA, kC);
    zm = m1;
    // queue of plane values k-1 .. k+2 for the centre of plane k+1
    qa = z2; qb = z3; qc = z4; qd = z5;
  }


  // cPML membership of this column along x and y (fixed during the march)
  const bool pml_xy = A.pml_on && valid && (A.pcx[i].tile >= 0 || A.pcy[j].tile >= 0);
  // z layers sit at the two ends of a member's planes, so a chunk reaches one only through its
  // first or last plane: chunks that do not skip the per-plane table read
  const bool pml_zc = A.pml_on && fz_inb(A.err, ke - 1, A.npc[2]) && (A.pcz[kb].tile >= 0 || A.pcz[ke - 1].tile >= 0);
  int buf = 0;
  uint32_t parity = 0;
  int64_t gk = col + plane * kb;  // offset of (i, j, k)
  int64_t gz = colz + plane * (kb + 4);  // z-queue load of the next iteration (plane k + 4)
  for (int it = 0; it < nplanes; ++it, gk += plane, gz += plane) {
    const int k = kb + it;
    P* XCm = reinterpret_cast<P*>(cbase + (it & 1) * (2 * L::XC + 2 * L::YC));
    P* XCp = XCm + TY * (TX + 2);
    P* YCm = XCp + TY * (TX + 2);
    P* YCp = YCm + (TY + 2) * TX;

    // ---- register loads for this plane (prefetched) and the next one
    const P qe = qe_next;
    P vmC = zero, Fz_hi = zero;
    if (!DIM2) {
      if (it + 1 < nplanes && fz_inb(A.err, gz, A.nfield)) qe_next = pmk(A.pi[gz], A.wi[gz]);
#if !defined(FZ_V_ZAFTER) && !defined(FZ_V_SPLITBAR)
      // ---- z: centre k+1 -> flux through face k+1/2
      P vpC;
      weno_center<R>(qa, qb, qc, qd, qe, vmC, vpC);
      Fz_hi = godunov<R>(zm, vpC, kA, kC);
#endif
    }

    // ---- plane k tile
    bool wait_failed = false;  // the block leaves after the barrier below; the tile is not stored
    if (!mbar_wait_bounded(&mbar[buf], parity)) {
      atomicOr(A.err, KERR_TMA_TIMEOUT);
      wait_failed = true;
#if defined(FZ_V_SPLITBAR)
      s_abort = 1;
#endif
    }
    const R* Tp = field(buf, 0);
    const R* Tu = field(buf, 1);
    const R* Tv = field(buf, 2);
    const uint8_t cls = clsb(buf)[lo];
    const bool pml_plane = pml_zc && fz_inb(A.err, k, A.npc[2]) && A.pcz[k].tile >= 0;
    // a warp whose 32 cells are all plain updates (in the room, no cPML, no source) updates them
    // after the barrier in one warp-uniform branch, without per-cell tests
    const bool warp_plain = __all_sync(0xffffffffu, valid && ((cls & (CLS_UPDATE | CLS_SOURCE)) == CLS_UPDATE) &&
                                                        !pml_xy && !pml_plane && fz_inb(A.err, gk, A.nfield));
#if defined(FZ_V_ZAFTER)
    if (!DIM2) {
      P vpC;
      weno_center<R>(qa, qb, qc, qd, qe, vmC, vpC);
      Fz_hi = godunov<R>(zm, vpC, kA, kC);
    }
#endif

    // ---- x and y centres of this thread's cell
    P xm, xp, ym, yp;
    {
      const int c0 = (ty + HY) * PW + (tx + HX);
      weno_center<R>(pmk(Tp[c0 - 2], Tu[c0 - 2]), pmk(Tp[c0 - 1], Tu[c0 - 1]), pmk(Tp[c0], Tu[c0]),
                     pmk(Tp[c0 + 1], Tu[c0 + 1]), pmk(Tp[c0 + 2], Tu[c0 + 2]), xm, xp);
      XCm[ty * (TX + 2) + tx + 1] = xm;
      XCp[ty * (TX + 2) + tx + 1] = xp;
      weno_center<R>(pmk(Tp[c0 - 2 * PW], Tv[c0 - 2 * PW]), pmk(Tp[c0 - PW], Tv[c0 - PW]), pmk(Tp[c0], Tv[c0]),
                     pmk(Tp[c0 + PW], Tv[c0 + PW]), pmk(Tp[c0 + 2 * PW], Tv[c0 + 2 * PW]), ym, yp);
      YCm[(ty + 1) * TX + tx] = ym;
      YCp[(ty + 1) * TX + tx] = yp;
    }
    // ---- halo centres: warp 0 the x edges (i0-1, i0+TX) of all 16 rows, warps 1-2 the y edge
    //      rows (j0-1, j0+TY)
    if (lt < 2 * TY) {
      const int r = lt >> 1, side = lt & 1;
      const int c0 = (r + HY) * PW + (side ? (HX + TX) : (HX - 1));
      P em, ep;
      weno_center<R>(pmk(Tp[c0 - 2], Tu[c0 - 2]), pmk(Tp[c0 - 1], Tu[c0 - 1]), pmk(Tp[c0], Tu[c0]),
                     pmk(Tp[c0 + 1], Tu[c0 + 1]), pmk(Tp[c0 + 2], Tu[c0 + 2]), em, ep);
      const int slot = r * (TX + 2) + (side ? TX + 1 : 0);
      XCm[slot] = em;
      XCp[slot] = ep;
    } else if (lt >= 32 && lt < 32 + 2 * TX) {
      const int e = lt - 32;
      const int c = e & (TX - 1);
      P em, ep;
      if constexpr (STAGE == 0 && sizeof(R) == 4 && TX == 32) {  // (16-wide tiles: both rows in one warp)
        // the fluxes use only V- of row j0-1 and only V+ of row j0+TY (elsewhere the two-branch
        // form costs the kernel a register spill, so the other instances compute both faces)
        if (e < TX) {
          const int c0 = (HY - 1) * PW + (c + HX);
          weno_center<R, WENO_LO>(pmk(Tp[c0 - 2 * PW], Tv[c0 - 2 * PW]), pmk(Tp[c0 - PW], Tv[c0 - PW]),
                                  pmk(Tp[c0], Tv[c0]), pmk(Tp[c0 + PW], Tv[c0 + PW]),
                                  pmk(Tp[c0 + 2 * PW], Tv[c0 + 2 * PW]), em, ep);
          YCm[c] = em;
        } else {
          const int c0 = (TY + HY) * PW + (c + HX);
          weno_center<R, WENO_HI>(pmk(Tp[c0 - 2 * PW], Tv[c0 - 2 * PW]), pmk(Tp[c0 - PW], Tv[c0 - PW]),
                                  pmk(Tp[c0], Tv[c0]), pmk(Tp[c0 + PW], Tv[c0 + PW]),
                                  pmk(Tp[c0 + 2 * PW], Tv[c0 + 2 * PW]), em, ep);
          YCp[(TY + 1) * TX + c] = ep;
        }
      } else {
        const int r = (e < TX) ? -1 : TY;
        const int c0 = (r + HY) * PW + (c + HX);
        weno_center<R>(pmk(Tp[c0 - 2 * PW], Tv[c0 - 2 * PW]), pmk(Tp[c0 - PW], Tv[c0 - PW]), pmk(Tp[c0], Tv[c0]),
                       pmk(Tp[c0 + PW], Tv[c0 + PW]), pmk(Tp[c0 + 2 * PW], Tv[c0 + 2 * PW]), em, ep);
        YCm[(r + 1) * TX + c] = em;
        YCp[(r + 1) * TX + c] = ep;
      }
    }
#if defined(FZ_V_SPLITBAR)
    // split barrier: each warp arrives once its centres are in shared memory, computes the z centre
    // (registers only) and only then waits for the other warps' centres
    __syncwarp();
    if ((lt & 31) == 0) mbar_arrive(&cbar[it & 1]);
    if (!DIM2) {
      P vpC;
      weno_center<R>(qa, qb, qc, qd, qe, vmC, vpC);
      Fz_hi = godunov<R>(zm, vpC, kA, kC);
    }
    if (!mbar_wait_bounded(&cbar[it & 1], (uint32_t)((it >> 1) & 1))) {
      atomicOr(A.err, KERR_TMA_TIMEOUT);
      return;
    }
    const bool abort_block = s_abort != 0;
#else
    // the per-plane barrier, with the OR of the threads' wait failures folded into it
    const bool abort_block = __syncthreads_or(wait_failed) != 0;
#endif
    if (abort_block) {
#ifdef FZ_WAIT_TEST
      if (lt == 0) drain_ring(mbar, it, nplanes, A.test_skip_plane);
#else
      if (lt == 0) drain_ring(mbar, it, nplanes, -1);
#endif
      return;
    }
    // the tile ring slot of plane it-1 is free now: fetch plane it+2 into it
    if (lt == 0 && it + 2 < nplanes) {
      fence_proxy_async();
      issue(it + 2);
    }

    // ---- the RK update of this cell before its cPML and source terms: face fluxes and flux
    //      differences (times h; .x pressure, .y velocity), stage combination
    auto rk_update = [&](int64_t g, P& Lx, P& Ly, P& Lz, R& pn, R& un, R& vn, R& wn) {
      Lx = godunov_diff<R>(XCm[ty * (TX + 2) + tx], xp, xm, XCp[ty * (TX + 2) + tx + 2], kA, kC);
      Ly = godunov_diff<R>(YCm[ty * TX + tx], yp, ym, YCp[(ty + 2) * TX + tx], kA, kC);
      Lz = psub(Fz_lo, Fz_hi);
      const R Lp = Lx.x + Ly.x + Lz.x;
      const int c0 = (ty + HY) * PW + (tx + HX);
      const R p_in = DIM2 ? Tp[c0] : qb.x, w_in = DIM2 ? A.wi[g] : qb.y;
      const R u_in = Tu[c0], v_in = Tv[c0];
      if (STAGE == 0) {
        pn = p_in + A.dt_h * Lp;
        un = u_in + A.dt_h * Lx.y;
        vn = v_in + A.dt_h * Ly.y;
        wn = w_in + A.dt_h * Lz.y;
      } else {
        // the stage combination a U0 + b (U_in + dt L) with a + b = 1, written as
        // U0 + b ((U_in + dt L) - U0): the weights sum to one exactly. In FP32 the rounded
        // 1/3 and 2/3 sum to 1 + 3e-8, a gain the whole field would pick up every step (the
        // reference divides by 3 instead, functions3D.cuh:1311-1314, which is unbiased too).
        const R bp = own(buf, 0)[lo], bu = own(buf, 1)[lo], bv = own(buf, 2)[lo], bw = own(buf, 3)[lo];
        const R wb = (STAGE == 1) ? R(0.25) : R(2.0 / 3.0);
        pn = bp + wb * ((p_in + A.dt_h * Lp) - bp);
        un = bu + wb * ((u_in + A.dt_h * Lx.y) - bu);
        vn = bv + wb * ((v_in + A.dt_h * Ly.y) - bv);
        wn = bw + wb * ((w_in + A.dt_h * Lz.y) - bw);
      }
    };
    if (warp_plain) {
      P Lx, Ly, Lz;
      R pn, un, vn, wn;
      rk_update(gk, Lx, Ly, Lz, pn, un, vn, wn);
      A.po[gk] = pn;
      A.uo[gk] = un;
      A.vo[gk] = vn;
      A.wo[gk] = wn;
    } else if (valid && (cls & (CLS_UPDATE | CLS_SOURCE)) && fz_inb(A.err, gk, A.nfield)) {
      const int64_t g = gk;
      if (cls & CLS_UPDATE) {
        P Lx, Ly, Lz;
        R pn, un, vn, wn;
        rk_update(g, Lx, Ly, Lz, pn, un, vn, wn);
        if (pml_xy || pml_plane) {
          // cPML (functions3D.cuh:725-755): field += w dt ((1/kappa - 1) D + psi), psi frozen
          // within the step and advanced once, in stage 2, by recursive convolution.
          const PmlCoef<R> cx = A.pcx[i], cy = A.pcy[j], cz = A.pcz[k];
          const int64_t d2 = A.pml_d2;
          if (cx.tile >= 0) {
            const int64_t X = cx.tile + d2 * ((int64_t)j + (int64_t)A.Ny * k);
            if (fz_inb(A.err, X, A.npsi[0])) {
            const P ps = A.psix[X];
            const R Dp = Lx.x * A.inv_h, Du = Lx.y * A.inv_h;
            pn += A.wdt * (cx.kinv1 * Dp + ps.x);
            un += A.wdt * (cx.kinv1 * Du + ps.y);
            if (STAGE == 2) A.psix[X] = pmk(cx.b * ps.x + cx.ca * Dp, cx.b * ps.y + cx.ca * Du);
            }
          }
          if (cy.tile >= 0) {
            const int64_t Y = (int64_t)i + (int64_t)A.Nx * ((int64_t)cy.tile + d2 * k);
            if (fz_inb(A.err, Y, A.npsi[1])) {
            const P ps = A.psiy[Y];
            const R Dp = Ly.x * A.inv_h, Dv = Ly.y * A.inv_h;
            pn += A.wdt * (cy.kinv1 * Dp + ps.x);
            vn += A.wdt * (cy.kinv1 * Dv + ps.y);
            if (STAGE == 2) A.psiy[Y] = pmk(cy.b * ps.x + cy.ca * Dp, cy.b * ps.y + cy.ca * Dv);
            }
          }
          if (cz.tile >= 0) {
            const int64_t Z = (int64_t)i + (int64_t)A.Nx * ((int64_t)j + (int64_t)A.Ny * cz.tile);
            if (fz_inb(A.err, Z, A.npsi[2])) {
            const P ps = A.psiz[Z];
            const R Dp = Lz.x * A.inv_h, Dw = Lz.y * A.inv_h;
            pn += A.wdt * (cz.kinv1 * Dp + ps.x);
            wn += A.wdt * (cz.kinv1 * Dw + ps.y);
            if (STAGE == 2) A.psiz[Z] = pmk(cz.b * ps.x + cz.ca * Dp, cz.b * ps.y + cz.ca * Dw);
            }
          }
        }
        if (cls & CLS_SOURCE) pn += source_sum(A, g);
        A.po[g] = pn;
        A.uo[g] = un;
        A.vo[g] = vn;
        A.wo[g] = wn;
      } else {
        // A source in a cell the stage kernels skip still adds to the stale output value, as
        // kernel_inject_src_SSP does (functions3D.cuh:1046).
        A.po[g] = A.po[g] + source_sum(A, g);
      }
    }

    if (++buf == NBUF) {
      buf = 0;
      parity ^= 1u;
    }
    Fz_lo = Fz_hi;
    zm = vmC;
    qa = qb;
    qb = qc;
    qc = qd;
    qd = qe;
  }
}

template <class R, int STAGE, bool DIM2>
__global__ void __launch_bounds__(NTHREADS, sizeof(R) == 4 ? FZ_STAGE_MINBLOCKS_F32 : 1)
    k_stage(const __grid_constant__ StageArgs<R> A, const __grid_constant__ StageMaps M) {
  stage_body<R, STAGE, DIM2, GridCta>(A, M);
}

// ------------------------------------------------------------------------------------------
// Immersed ADE band (functions3D.cuh:462-565 + ADE_solver 426-459), one thread per band cell of
// the compact list. Probe geometry (normal, trilinear corner and weights at C - 2h n, chi) is
// precomputed once on the host. The probe reads the stage-input fields, which no kernel of this
// stage writes; the blend reads and writes only the band cell itself.
// ------------------------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ R trilin(const R* __restrict__ f, int64_t q, int64_t Sx, int64_t plane, R sx,
                                    R sy, R sz) {
  const R c00 = __ldg(f + q) * (R(1) - sx) + __ldg(f + q + 1) * sx;
  const R c10 = __ldg(f + q + Sx) * (R(1) - sx) + __ldg(f + q + Sx + 1) * sx;
  const R c01 = __ldg(f + q + plane) * (R(1) - sx) + __ldg(f + q + plane + 1) * sx;
  const R c11 = __ldg(f + q + plane + Sx) * (R(1) - sx) + __ldg(f + q + plane + Sx + 1) * sx;
  const R c0 = c00 * (R(1) - sy) + c10 * sy, c1 = c01 * (R(1) - sy) + c11 * sy;
  return c0 * (R(1) - sz) + c1 * sz;
}

template <class R>
struct Vec4;
template <>
struct Vec4<float> {
  typedef float4 T;
};
template <>
struct Vec4<double> {
  typedef double4 T;
};

// STAGE selects the ADE stage coefficients (a, b, c) = (0,1,1), (3,1,4), (1,2,3)
// (main3D.cu:1290, 1298, 1306): left = (a middle + b (right + dt L(right))) / c.
// KM, LM > 0: at most KM real poles and LM complex pairs. Every load that does not depend on the
// probe (the cell's own fields, the ADE states of the stage) is then issued at the top, beside the
// probe gathers, so one thread keeps ~50 loads in flight; KM = LM = 0 is the general form with
// the state loads inside the pole loops.
template <class R, int STAGE, int KM, int LM>
__device__ __forceinline__ void band_body(const BandArgs<R>& B, const int64_t b) {
  typedef typename Vec4<R>::T V4;
  if (b >= B.nB) return;
  const int4 rc = __ldg(B.rec + b);
  const int64_t cell = (int64_t)(((uint64_t)(uint32_t)rc.y << 32) | (uint32_t)rc.x);
  const int64_t q = cell + rc.z;
  const int m = rc.w;
  const int64_t nB = B.nB;
  if (!fz_inb(B.err, cell, B.nfield) || !fz_inb(B.err, q, B.nfield) ||
      !fz_inb(B.err, q + B.plane + B.Sx + 1, B.nfield))
    return;
  const V4 g4 = reinterpret_cast<const V4*>(B.geo)[b];
  const V4 n4 = reinterpret_cast<const V4*>(B.nrm)[b];
  // the cell's own stage output (written by the stage kernel, blended here by this thread only)
  R po0 = R(0), uo0 = R(0), vo0 = R(0), wo0 = R(0);
  if (KM > 0) {
    po0 = B.po[cell];
    uo0 = B.uo[cell];
    vo0 = B.vo[cell];
    wo0 = B.wo[cell];
  }
  double rK[KM > 0 ? KM : 1], mK[KM > 0 ? KM : 1], r1L[LM > 0 ? LM : 1], r2L[LM > 0 ? LM : 1];
  double m1L[LM > 0 ? LM : 1], m2L[LM > 0 ? LM : 1];
#pragma unroll
  for (int k = 0; k < KM; ++k)
    if (k < B.K) {
      rK[k] = __ldg(B.phR + (int64_t)k * nB + b);
      if (STAGE > 0) mK[k] = __ldg(B.phM + (int64_t)k * nB + b);
    }
#pragma unroll
  for (int l = 0; l < LM; ++l)
    if (l < B.L) {
      r1L[l] = __ldg(B.s1R + (int64_t)l * nB + b);
      r2L[l] = __ldg(B.s2R + (int64_t)l * nB + b);
      if (STAGE > 0) {
        m1L[l] = __ldg(B.s1M + (int64_t)l * nB + b);
        m2L[l] = __ldg(B.s2M + (int64_t)l * nB + b);
      }
    }
  const R sx = g4.x, sy = g4.y, sz = g4.z, chi = g4.w;
  const R nx = n4.x, ny = n4.y, nz = n4.z;
  const R pD = trilin<R>(B.pi, q, B.Sx, B.plane, sx, sy, sz);
  const R uD = trilin<R>(B.ui, q, B.Sx, B.plane, sx, sy, sz);
  const R vD = trilin<R>(B.vi, q, B.Sx, B.plane, sx, sy, sz);
  const R wD = trilin<R>(B.wi, q, B.Sx, B.plane, sx, sy, sz);
  const R un = uD * nx + vD * ny + wD * nz;
  const R utx = uD - un * nx, uty = vD - un * ny, utz = wD - un * nz;
  const double wout = (double)pD + B.Z0 * (double)un;  // outgoing characteristic
  constexpr double a_ssp = (STAGE == 0) ? 0.0 : (STAGE == 1) ? 3.0 : 1.0;
  constexpr double b_ssp = (STAGE == 2) ? 2.0 : 1.0;
  constexpr double inv_c = (STAGE == 0) ? 1.0 : (STAGE == 1) ? 0.25 : 1.0 / 3.0;
  double sumA = 0.0, sumBC = 0.0;
  // one real pole / complex pair of the ADE stage recursion
  auto real_pole = [&](int k, double r, double mid) {
    const int mi = m * B.K + k;
    const double Lphi = wout - __ldg(B.zeta + mi) * r;
    double v = b_ssp * (r + B.dt * Lphi);
    if (STAGE > 0) v += a_ssp * mid;
    v *= inv_c;
    B.phL[(int64_t)k * nB + b] = v;
    sumA += __ldg(B.A + mi) * v;
  };
  auto pole_pair = [&](int l, double r1, double r2, double m1, double m2) {
    const int mi = m * B.L + l;
    const double al = __ldg(B.alpha + mi), be = __ldg(B.beta + mi);
    const double L1 = wout - (al * r1 + be * r2);
    const double L2 = be * r1 - al * r2;
    double n1 = b_ssp * (r1 + B.dt * L1);
    double n2 = b_ssp * (r2 + B.dt * L2);
    if (STAGE > 0) {
      n1 += a_ssp * m1;
      n2 += a_ssp * m2;
    }
    n1 *= inv_c;
    n2 *= inv_c;
    const int64_t si = (int64_t)l * nB + b;
    B.s1L[si] = n1;
    B.s2L[si] = n2;
    sumBC += __ldg(B.B + mi) * n1 + __ldg(B.C + mi) * n2;
  };
  if constexpr (KM > 0) {
#pragma unroll
    for (int k = 0; k < KM; ++k)
      if (k < B.K) real_pole(k, rK[k], STAGE > 0 ? mK[k] : 0.0);
#pragma unroll
    for (int l = 0; l < LM; ++l)
      if (l < B.L) pole_pair(l, r1L[l], r2L[l], STAGE > 0 ? m1L[l] : 0.0, STAGE > 0 ? m2L[l] : 0.0);
  } else {
    for (int k = 0; k < B.K; ++k) {
      const int64_t si = (int64_t)k * nB + b;
      real_pole(k, B.phR[si], STAGE > 0 ? B.phM[si] : 0.0);
    }
    for (int l = 0; l < B.L; ++l) {
      const int64_t si = (int64_t)l * nB + b;
      pole_pair(l, B.s1R[si], B.s2R[si], STAGE > 0 ? B.s1M[si] : 0.0, STAGE > 0 ? B.s2M[si] : 0.0);
    }
  }
  const double win = __ldg(B.Rinf + m) * wout + sumA + sumBC;  // incoming characteristic
  const R pb = (R)(0.5 * (win + wout));
  const R unb = (R)((wout - win) / (2.0 * B.Z0));
  const R ub = unb * nx + utx, vb = unb * ny + uty, wb = unb * nz + utz;
  const R omc = R(1) - chi;
  if (KM == 0) {
    po0 = B.po[cell];
    uo0 = B.uo[cell];
    vo0 = B.vo[cell];
    wo0 = B.wo[cell];
  }
  B.uo[cell] = omc * uo0 + chi * ub;
  B.vo[cell] = omc * vo0 + chi * vb;
  B.wo[cell] = omc * wo0 + chi * wb;
  B.po[cell] = omc * po0 + chi * pb;
}

#define FZ_BAND_BOUNDS(R, KM) __launch_bounds__(256, (sizeof(R) == 4 && KM > 0 && KM <= 2) ? 4 : 3)

template <class R, int STAGE, int KM, int LM>
__global__ void FZ_BAND_BOUNDS(R, KM) k_band(const __grid_constant__ BandArgs<R> B) {
  band_body<R, STAGE, KM, LM>(B, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}

// Receiver gather after the last stage of a step (main3D.cu:1399-1414), into a device buffer;
// then advances the device step counter. One block.
template <class R>
__device__ __forceinline__ void receivers_body(const R* __restrict__ p, const R* __restrict__ u,
                                               const R* __restrict__ v, const R* __restrict__ w,
                                               const int64_t* __restrict__ rcell, int nrec, double* ir, double* vel,
                                               int64_t cap, int64_t* step, int32_t* err, int64_t nfield) {
  const int64_t n = *step;
  for (int r = threadIdx.x; r < nrec; r += blockDim.x) {
    const int64_t c = rcell[r];
    if (!fz_inb(err, c, nfield)) continue;
    const double pp = (double)p[c], uu = (double)u[c], vv = (double)v[c], ww = (double)w[c];
    // health word: a blown-up solution reaches the receivers (their samples are read anyway)
    if (!isfinite(pp) || !isfinite(uu) || !isfinite(vv) || !isfinite(ww)) atomicOr(err, KERR_NONFINITE);
    if (n < cap) {
      const int64_t o = (int64_t)r * cap + n;
      ir[o] = pp;
      vel[3 * o + 0] = uu;
      vel[3 * o + 1] = vv;
      vel[3 * o + 2] = ww;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) *step = n + 1;
}

template <class R>
__global__ void k_receivers(const R* __restrict__ p, const R* __restrict__ u, const R* __restrict__ v,
                            const R* __restrict__ w, const int64_t* __restrict__ rcell, int nrec,
                            double* ir, double* vel, int64_t cap, int64_t* step, int32_t* err, int64_t nfield) {
  receivers_body<R>(p, u, v, w, rcell, nrec, ir, vel, cap, step, err, nfield);
}

// ------------------------------------------------------------------------------------------
// Groups of rooms in one launch per kernel kind. The CTAs (band blocks) of every member room are
// laid end to end in one 1-D grid: a CTA finds its room from the prefix table of CTA counts,
// copies that room's launch arguments from device memory into shared memory (its TMA descriptors
// come as kernel parameters, as in a one-room launch) and runs the same body as the one-room
// kernel, so each room's cells are updated exactly as a launch of its own would update them.
// ------------------------------------------------------------------------------------------
__shared__ int g_group_cta[3];  // tile coordinates of this CTA inside its room

struct GroupCta {
  static __device__ __forceinline__ int x() { return g_group_cta[0]; }
  static __device__ __forceinline__ int y() { return g_group_cta[1]; }
  static __device__ __forceinline__ int z() { return g_group_cta[2]; }
};

// the member whose range [start[m], start[m+1]) holds `blk` (uniform across the block)
__device__ __forceinline__ int group_member(const int32_t* start, int n, int blk) {
  int m = 0;
  while (m + 1 < n && blk >= start[m + 1]) ++m;
  return m;
}

// word-wise copy of one member's argument block into shared memory by the whole block
template <class T>
__device__ __forceinline__ void copy_args(T& dst, const T* src, int t, int nt) {
  static_assert(sizeof(T) % 4 == 0, "argument blocks are whole words");
  const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
  uint32_t* d = reinterpret_cast<uint32_t*>(&dst);
  for (int w = t; w < (int)(sizeof(T) / 4); w += nt) d[w] = __ldg(s + w);
}

template <class R, int STAGE>
__global__ void __launch_bounds__(NTHREADS, sizeof(R) == 4 ? FZ_STAGE_MINBLOCKS_F32 : 1)
    k_stage_group(const __grid_constant__ GroupStageArgs<R> G) {
  __shared__ __align__(16) StageArgs<R> sA;
  const int t = threadIdx.y * blockDim.x + threadIdx.x;
  const int m = group_member(G.cta_start, G.n, blockIdx.x);
  copy_args(sA, G.args + m, t, NTHREADS);
  if (t == 0) {
    const int local = (int)blockIdx.x - G.cta_start[m];
    const int gx = G.gx[m], gy = G.gy[m];
    g_group_cta[0] = local % gx;
    g_group_cta[1] = (local / gx) % gy;
    g_group_cta[2] = local / (gx * gy);
  }
  __syncthreads();
  stage_body<R, STAGE, false, GroupCta>(sA, G.maps[m]);
}

template <class R, int STAGE, int KM, int LM>
__global__ void FZ_BAND_BOUNDS(R, KM) k_band_group(const __grid_constant__ GroupBandArgs<R> G) {
  __shared__ __align__(16) BandArgs<R> sB;
  const int m = group_member(G.blk_start, G.n, blockIdx.x);
  copy_args(sB, G.args + m, threadIdx.x, blockDim.x);
  __syncthreads();
  band_body<R, STAGE, KM, LM>(sB, (int64_t)((int)blockIdx.x - G.blk_start[m]) * blockDim.x + threadIdx.x);
}

// one block per member
template <class R>
__global__ void k_receivers_group(const RecArgs<R>* __restrict__ args) {
  const RecArgs<R>& a = args[blockIdx.x];
  receivers_body<R>(a.p, a.u, a.v, a.w, a.rcell, a.nrec, a.ir, a.vel, a.cap, a.step, a.err, a.nfield);
}

// Non-finite values in a state (p, u, v, w over n cells), counted into *count.
template <class R>
__global__ void k_count_nonfinite(const R* __restrict__ p, const R* __restrict__ u, const R* __restrict__ v,
                                  const R* __restrict__ w, int64_t n, unsigned long long* count) {
  unsigned long long k = 0;
  // four cells per thread and pass, their sixteen loads issued together
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t c0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c0 < n; c0 += 4 * stride) {
    R x[4][4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int64_t c = c0 + q * stride;
      const bool in = c < n;
      x[q][0] = in ? p[c] : R(0);
      x[q][1] = in ? u[c] : R(0);
      x[q][2] = in ? v[c] : R(0);
      x[q][3] = in ? w[c] : R(0);
    }
#pragma unroll
    for (int q = 0; q < 4; q++)
      k += (!isfinite(x[q][0])) + (!isfinite(x[q][1])) + (!isfinite(x[q][2])) + (!isfinite(x[q][3]));
  }
  for (int o = 16; o > 0; o >>= 1) k += __shfl_down_sync(0xffffffffu, k, o);
  if ((threadIdx.x & 31) == 0 && k) atomicAdd(count, k);
}

// Animation frame after a step (main3D.cu:1326-1394): pressure on the planes x = i0, y = j0, z = k0
// and the in-plane components of the unit energy-flow direction sign(p) u / |u|, written when the
// step just completed (the device step counter, already advanced) is a multiple of anim_step
// counted from the first. Frame layout: pX[Ny Nz] pY[Nx Nz] pZ[Nx Ny], then (Iy, Iz) on X,
// (Ix, Iz) on Y, (Ix, Iy) on Z -- each plane in the reference's order (j + Ny k, i + Nx k, i + Nx j).
template <class R>
__global__ void k_slices(const R* __restrict__ p, const R* __restrict__ u, const R* __restrict__ v,
                         const R* __restrict__ w, int Nx, int Ny, int Nz, int64_t Sx, int i0, int j0, int k0,
                         const int64_t* __restrict__ step, int64_t anim_step, int64_t cap, float* __restrict__ out) {
  const int64_t n = *step - 1;
  if (n < 0 || n % anim_step != 0) return;
  const int64_t f = n / anim_step;
  if (f >= cap) return;
  const int64_t nX = (int64_t)Ny * Nz, nY = (int64_t)Nx * Nz, nZ = (int64_t)Nx * Ny, tot = nX + nY + nZ;
  float* fr = out + f * 3 * tot;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    int i, j, k;
    if (e < nX) {
      j = (int)(e % Ny); k = (int)(e / Ny); i = i0;
    } else if (e < nX + nY) {
      const int64_t q = e - nX;
      i = (int)(q % Nx); k = (int)(q / Nx); j = j0;
    } else {
      const int64_t q = e - nX - nY;
      i = (int)(q % Nx); j = (int)(q / Nx); k = k0;
    }
    const int64_t c = XOFF + i + Sx * ((int64_t)j + (int64_t)Ny * k);
    const float pp = (float)p[c], uu = (float)u[c], vv = (float)v[c], ww = (float)w[c];
    const float sp = (pp >= 0.f) ? 1.f : -1.f;
    const float inv = sp / (sqrtf(uu * uu + vv * vv + ww * ww) + 1e-20f);
    fr[e] = pp;
    float c1, c2;
    if (e < nX) { c1 = vv * inv; c2 = ww * inv; }
    else if (e < nX + nY) { c1 = uu * inv; c2 = ww * inv; }
    else { c1 = uu * inv; c2 = vv * inv; }
    // component planes follow the pressure planes: [c1X c2X | c1Y c2Y | c1Z c2Z]
    const int64_t base = (e < nX) ? tot : (e < nX + nY) ? tot + 2 * nX : tot + 2 * nX + 2 * nY;
    const int64_t off = (e < nX) ? e : (e < nX + nY) ? e - nX : e - nX - nY;
    const int64_t m = (e < nX) ? nX : (e < nX + nY) ? nY : nZ;
    fr[base + off] = c1;
    fr[base + m + off] = c2;
  }
}

// FP64 energy 0.5 sum(p^2/(rho c^2) + rho |u|^2) (functions3D.cuh:111-129). Padding cells are
// zero, so summing the whole allocation sums the grid.
template <class R>
__global__ void k_energy(const R* __restrict__ p, const R* __restrict__ u, const R* __restrict__ v,
                         const R* __restrict__ w, int64_t n, double inv_rc2, double rho, double* out) {
  double s = 0.0;
  // four cells per thread and pass, their sixteen loads issued together
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t c0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c0 < n; c0 += 4 * stride) {
    R x[4][4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int64_t c = c0 + q * stride;
      const bool in = c < n;
      x[q][0] = in ? p[c] : R(0);
      x[q][1] = in ? u[c] : R(0);
      x[q][2] = in ? v[c] : R(0);
      x[q][3] = in ? w[c] : R(0);
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const double pp = x[q][0], uu = x[q][1], vv = x[q][2], ww = x[q][3];
      s += pp * pp * inv_rc2 + rho * (uu * uu + vv * vv + ww * ww);
    }
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) atomicAdd(out, 0.5 * s);
  }
}

// ------------------------------------------------------------------------------------------
// Launchers
// ------------------------------------------------------------------------------------------
template <class R>
size_t stage_smem_bytes() {
  return (size_t)StageSmem<R>::BYTES;
}

template <class R>
cudaError_t stage_setup() {
  const int bytes = (int)stage_smem_bytes<R>();
  const void* fns[6] = {(const void*)k_stage<R, 0, false>, (const void*)k_stage<R, 1, false>,
                        (const void*)k_stage<R, 2, false>, (const void*)k_stage<R, 0, true>,
                        (const void*)k_stage<R, 1, true>,  (const void*)k_stage<R, 2, true>};
  for (const void* f : fns) {
    const cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
  }
  const void* gfns[3] = {(const void*)k_stage_group<R, 0>, (const void*)k_stage_group<R, 1>,
                         (const void*)k_stage_group<R, 2>};
  for (const void* f : gfns) {
    const cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <class R>
cudaError_t stage_occupancy(int* blocks_per_sm) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_stage<R, 0, false>, NTHREADS,
                                                        stage_smem_bytes<R>());
}

template <class R>
cudaError_t launch_stage(int stage, bool two_d, const StageArgs<R>& a, const StageMaps& m, dim3 grid,
                         cudaStream_t s) {
  const dim3 block(TX, TY, 1);
  const size_t smem = stage_smem_bytes<R>();
  if (!two_d) {
    if (stage == 0)
      k_stage<R, 0, false><<<grid, block, smem, s>>>(a, m);
    else if (stage == 1)
      k_stage<R, 1, false><<<grid, block, smem, s>>>(a, m);
    else
      k_stage<R, 2, false><<<grid, block, smem, s>>>(a, m);
  } else {
    if (stage == 0)
      k_stage<R, 0, true><<<grid, block, smem, s>>>(a, m);
    else if (stage == 1)
      k_stage<R, 1, true><<<grid, block, smem, s>>>(a, m);
    else
      k_stage<R, 2, true><<<grid, block, smem, s>>>(a, m);
  }
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_band(int stage, const BandArgs<R>& a, cudaStream_t s) {
  if (a.nB <= 0) return cudaSuccess;
  const int bs = 256;
  const int64_t nb = (a.nB + bs - 1) / bs;
  // pole counts of up to 2 (4) real poles and complex pairs take the fixed-size form
  const int fit = (a.K <= 2 && a.L <= 2) ? 2 : (a.K <= 4 && a.L <= 4) ? 4 : 0;
#define FZ_BAND_LAUNCH(ST)                                                    \
  if (fit == 2)                                                               \
    k_band<R, ST, 2, 2><<<(unsigned)nb, bs, 0, s>>>(a);                       \
  else if (fit == 4)                                                          \
    k_band<R, ST, 4, 4><<<(unsigned)nb, bs, 0, s>>>(a);                       \
  else                                                                        \
    k_band<R, ST, 0, 0><<<(unsigned)nb, bs, 0, s>>>(a);
  if (stage == 0) {
    FZ_BAND_LAUNCH(0)
  } else if (stage == 1) {
    FZ_BAND_LAUNCH(1)
  } else {
    FZ_BAND_LAUNCH(2)
  }
#undef FZ_BAND_LAUNCH
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_receivers(const R* p, const R* u, const R* v, const R* w, const int64_t* rcell, int nrec,
                             double* ir, double* vel, int64_t cap, int64_t* step, int32_t* err, int64_t nfield,
                             cudaStream_t s) {
  k_receivers<R><<<1, 256, 0, s>>>(p, u, v, w, rcell, nrec, ir, vel, cap, step, err, nfield);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_count_nonfinite(const R* p, const R* u, const R* v, const R* w, int64_t n,
                                   unsigned long long* count, int nsm, cudaStream_t s) {
  k_count_nonfinite<R><<<nsm * 8, 256, 0, s>>>(p, u, v, w, n, count);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_slices(const R* p, const R* u, const R* v, const R* w, int Nx, int Ny, int Nz, int64_t Sx, int i0,
                          int j0, int k0, const int64_t* step, int64_t anim_step, int64_t cap, float* out,
                          int nsm, cudaStream_t s) {
  k_slices<R><<<nsm, 256, 0, s>>>(p, u, v, w, Nx, Ny, Nz, Sx, i0, j0, k0, step, anim_step, cap, out);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_energy(const R* p, const R* u, const R* v, const R* w, int64_t n, double inv_rc2,
                          double rho, double* out, int nsm, cudaStream_t s) {
  k_energy<R><<<nsm * 8, 256, 0, s>>>(p, u, v, w, n, inv_rc2, rho, out);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_stage_group(int stage, const GroupStageArgs<R>& g, int ctas, cudaStream_t s) {
  if (ctas <= 0) return cudaSuccess;
  const dim3 block(TX, TY, 1);
  const size_t smem = stage_smem_bytes<R>();
  if (stage == 0)
    k_stage_group<R, 0><<<ctas, block, smem, s>>>(g);
  else if (stage == 1)
    k_stage_group<R, 1><<<ctas, block, smem, s>>>(g);
  else
    k_stage_group<R, 2><<<ctas, block, smem, s>>>(g);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_band_group(int stage, const GroupBandArgs<R>& g, int blocks, int fit, cudaStream_t s) {
  if (blocks <= 0) return cudaSuccess;
#define FZ_BANDG_LAUNCH(ST)                                      \
  if (fit == 2)                                                  \
    k_band_group<R, ST, 2, 2><<<blocks, 256, 0, s>>>(g);         \
  else if (fit == 4)                                             \
    k_band_group<R, ST, 4, 4><<<blocks, 256, 0, s>>>(g);         \
  else                                                           \
    k_band_group<R, ST, 0, 0><<<blocks, 256, 0, s>>>(g);
  if (stage == 0) {
    FZ_BANDG_LAUNCH(0)
  } else if (stage == 1) {
    FZ_BANDG_LAUNCH(1)
  } else {
    FZ_BANDG_LAUNCH(2)
  }
#undef FZ_BANDG_LAUNCH
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_receivers_group(const RecArgs<R>* args, int n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_receivers_group<R><<<n, 256, 0, s>>>(args);
  return cudaGetLastError();
}

#define FZ_INSTANTIATE(R)                                                                          \
  template size_t stage_smem_bytes<R>();                                                           \
  template cudaError_t stage_setup<R>();                                                           \
  template cudaError_t stage_occupancy<R>(int*);                                                   \
  template cudaError_t launch_stage<R>(int, bool, const StageArgs<R>&, const StageMaps&, dim3, cudaStream_t); \
  template cudaError_t launch_band<R>(int, const BandArgs<R>&, cudaStream_t);                      \
  template cudaError_t launch_receivers<R>(const R*, const R*, const R*, const R*, const int64_t*, \
                                           int, double*, double*, int64_t, int64_t*, int32_t*,     \
                                           int64_t, cudaStream_t);                                 \
  template cudaError_t launch_count_nonfinite<R>(const R*, const R*, const R*, const R*, int64_t,  \
                                                 unsigned long long*, int, cudaStream_t);         \
  template cudaError_t launch_slices<R>(const R*, const R*, const R*, const R*, int, int, int, int64_t, int, int, \
                                        int, const int64_t*, int64_t, int64_t, float*, int, cudaStream_t);       \
  template cudaError_t launch_energy<R>(const R*, const R*, const R*, const R*, int64_t, double,   \
                                        double, double*, int, cudaStream_t);                       \
  template cudaError_t launch_stage_group<R>(int, const GroupStageArgs<R>&, int, cudaStream_t);    \
  template cudaError_t launch_band_group<R>(int, const GroupBandArgs<R>&, int, int, cudaStream_t); \
  template cudaError_t launch_receivers_group<R>(const RecArgs<R>*, int, cudaStream_t);

FZ_INSTANTIATE(float)
FZ_INSTANTIATE(double)

}  // namespace fz
