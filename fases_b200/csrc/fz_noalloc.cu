// fz_noalloc.cu -- acoustic energy of caller-owned device fields, with no device allocation.
//
// fz_energy needs a solver handle, and the handle allocates device memory (cudaMalloc) for its
// fields and for the scratch of its reduction. Some callers cannot allocate: a host program
// that already owns its field arrays inside a memory pool it manages itself, a real-time audio
// or plugin thread where a cudaMalloc (which can synchronise the device) is not allowed, or code
// that runs while another component holds the allocator. fz_energy_noalloc serves them: the
// caller passes its own device arrays and a device output slot, and the reduction's scratch
// (one partial sum per block) lives in a fixed file-scope device array instead of an
// allocation.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/fz.h"
#include "fz_internal.h"

// The scratch: one FP64 partial sum per block of the first pass, at most FZ_NOALLOC_MAX_BLOCKS
// blocks (32 KB). Every GPU that loads the library holds this array until the process exits.
// All calls share it and it keeps the last call's partial sums: the first pass writes every
// entry the second pass reads, so nothing has to be cleared, but two calls that overlap on the
// GPU (different streams, no ordering between them) race on it.
static __device__ __align__(256) double g_energy_partials[FZ_NOALLOC_MAX_BLOCKS];

namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 64;                                   // elements per thread
constexpr int64_t kPerBlock = (int64_t)kThreads * kPerThread;   // 16384 elements per block
static_assert(kPerBlock * FZ_NOALLOC_MAX_BLOCKS == FZ_NOALLOC_MAX_CELLS, "scratch size and element limit disagree");

__global__ void __launch_bounds__(kThreads) k_energy_partials(const float* __restrict__ p, const float* __restrict__ u,
                                                              const float* __restrict__ v, const float* __restrict__ w,
                                                              int64_t n, double inv_rc2, double rho, double* partials) {
  const int64_t base = (int64_t)blockIdx.x * kPerBlock;
  double s = 0.0;
  for (int q = 0; q < kPerThread; ++q) {
    const int64_t c = base + (int64_t)q * kThreads + threadIdx.x;
    if (c < n) {
      const double pp = p[c], uu = u[c], vv = v[c], ww = w[c];
      s += pp * pp * inv_rc2 + rho * (uu * uu + vv * vv + ww * ww);
    }
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ double red[kThreads / 32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = (threadIdx.x < kThreads / 32) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
  }
}

__global__ void __launch_bounds__(kThreads) k_energy_finish(const double* partials, int nb, double* out) {
  double s = 0.0;
  for (int b = threadIdx.x; b < nb; b += kThreads) s += partials[b];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ double red[kThreads / 32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = (threadIdx.x < kThreads / 32) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) *out = 0.5 * s;
  }
}

// Device address of the scratch array, looked up once per device and context. In host code the
// symbol g_energy_partials is only a host-side stand-in: a kernel given it would read the wrong
// memory, so kernels get the address from cudaGetSymbolAddress, taken with that device current.
// The address belongs to the module loaded into the device's current context; after
// cudaDeviceReset (or any other re-creation of the primary context) the module is loaded again,
// possibly elsewhere, so the cached address is keyed on the context it was taken in.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch[kMaxDevices] = {nullptr};
void* g_scratch_ctx[kMaxDevices] = {nullptr};

// cuCtxGetCurrent, fetched from the driver at run time (no link-time libcuda dependency).
typedef int (*CtxGetCurrentFn)(void**);
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (CtxGetCurrentFn)p;
  }
  return fn;
}

}  // namespace

extern "C" int fz_energy_noalloc(const float* p, const float* u, const float* v, const float* w, int64_t n,
                                 double rho, double c, double* out, void* stream) {
  if (!p || !u || !v || !w || !out) return fzi::set_global_error(FZ_EINVAL, "fz_energy_noalloc: NULL pointer");
  if (n < 0) return fzi::set_global_error(FZ_EINVAL, "fz_energy_noalloc: negative element count");
  if (!(rho > 0) || !(c > 0)) return fzi::set_global_error(FZ_EINVAL, "fz_energy_noalloc: rho and c must be > 0");
  if (n > FZ_NOALLOC_MAX_CELLS)
    return fzi::set_global_error(FZ_EINVAL, "fz_energy_noalloc: " + std::to_string(n) + " elements exceed the limit of " +
                                                std::to_string((long long)FZ_NOALLOC_MAX_CELLS) +
                                                " (the fixed scratch holds " +
                                                std::to_string(FZ_NOALLOC_MAX_BLOCKS) + " block partial sums)");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fzi::set_global_error(FZ_ECUDA, std::string("fz_energy_noalloc: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fzi::set_global_error(FZ_EINVAL, "fz_energy_noalloc: device ordinal too large");
  double* scratch = nullptr;
  {
    // set-up once per device (and context), with that device current (the calling thread's
    // current device). Before the runtime's first call on this thread the current context can
    // still be unset: the lookup then runs, and makes the device's primary context current.
    CtxGetCurrentFn getctx = ctx_get_current();
    if (!getctx) return fzi::set_global_error(FZ_ECUDA, "fz_energy_noalloc: cuCtxGetCurrent not available");
    void* ctx = nullptr;
    if (getctx(&ctx) != 0) ctx = nullptr;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!ctx || !g_scratch[dev] || g_scratch_ctx[dev] != ctx) {
      g_scratch[dev] = nullptr;
      g_scratch_ctx[dev] = nullptr;
      double* a = nullptr;
      e = cudaGetSymbolAddress((void**)&a, g_energy_partials);
      if (e != cudaSuccess)
        return fzi::set_global_error(FZ_ECUDA, std::string("fz_energy_noalloc: cudaGetSymbolAddress: ") +
                                                   cudaGetErrorString(e));
      if (getctx(&ctx) != 0 || !ctx) return fzi::set_global_error(FZ_ECUDA, "fz_energy_noalloc: no current CUDA context");
      g_scratch[dev] = a;
      g_scratch_ctx[dev] = ctx;
    }
    scratch = g_scratch[dev];
  }
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int nb = (int)((n + kPerBlock - 1) / kPerBlock);
  if (nb == 0) {
    e = cudaMemsetAsync(out, 0, sizeof(double), s);
  } else {
    const double inv_rc2 = 1.0 / (rho * c * c);
    k_energy_partials<<<nb, kThreads, 0, s>>>(p, u, v, w, n, inv_rc2, rho, scratch);
    e = cudaGetLastError();
    if (e == cudaSuccess) {
      k_energy_finish<<<1, kThreads, 0, s>>>(scratch, nb, out);
      e = cudaGetLastError();
    }
  }
  if (e != cudaSuccess) return fzi::set_global_error(FZ_ECUDA, std::string("fz_energy_noalloc: ") + cudaGetErrorString(e));
  return FZ_OK;
}
