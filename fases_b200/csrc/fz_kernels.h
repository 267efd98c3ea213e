// fz_kernels.h -- host-callable launchers of the sm_100a stepping kernels (fz_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fz_device.cuh"

namespace fz {

template <class R>
size_t stage_smem_bytes();
template <class R>
cudaError_t stage_setup();
template <class R>
cudaError_t stage_occupancy(int* blocks_per_sm);
template <class R>
cudaError_t launch_stage(int stage, bool two_d, const StageArgs<R>& a, const StageMaps& m, dim3 grid,
                         cudaStream_t s);
template <class R>
cudaError_t launch_band(int stage, const BandArgs<R>& a, cudaStream_t s);
template <class R>
cudaError_t launch_receivers(const R* p, const R* u, const R* v, const R* w, const int64_t* rcell,
                             int nrec, double* ir, double* vel, int64_t cap, int64_t* step, int32_t* err,
                             int64_t nfield, cudaStream_t s);
template <class R>
cudaError_t launch_count_nonfinite(const R* p, const R* u, const R* v, const R* w, int64_t n,
                                   unsigned long long* count, int nsm, cudaStream_t s);
template <class R>
cudaError_t launch_slices(const R* p, const R* u, const R* v, const R* w, int Nx, int Ny, int Nz, int64_t Sx, int i0,
                          int j0, int k0, const int64_t* step, int64_t anim_step, int64_t cap, float* out,
                          int nsm, cudaStream_t s);
// groups of rooms: one launch per kernel kind over the member rooms' CTAs laid end to end
template <class R>
cudaError_t launch_stage_group(int stage, const GroupStageArgs<R>& g, int ctas, cudaStream_t s);
template <class R>
cudaError_t launch_band_group(int stage, const GroupBandArgs<R>& g, int blocks, int fit, cudaStream_t s);
template <class R>
cudaError_t launch_receivers_group(const RecArgs<R>* args, int n, cudaStream_t s);
template <class R>
cudaError_t launch_energy(const R* p, const R* u, const R* v, const R* w, int64_t n, double inv_rc2,
                          double rho, double* out, int nsm, cudaStream_t s);

}  // namespace fz
