// clb_noalloc.cu - volume averages of caller-owned device lattices with no device allocation.
//
// Some callers cannot call cudaMalloc: a host runtime that owns the whole device memory pool and
// hands out no more, or an embedding that forbids device allocation after start-up (a long-running
// service with a fixed memory budget).  clb_scalar_averages_noalloc serves them: the caller passes
// device pointers for the inputs and the output, and the per-block partial sums of the reduction
// live in the file-scope array below instead of a cudaMalloc'd buffer.
//
// The array is sized for kNoAllocMaxRows block rows (192 KiB); every GPU that loads the library
// holds it until the process exits.  All calls share it and it keeps the last call's contents;
// each call's blocks overwrite exactly the rows the same call then sums, so nothing has to start
// at zero.  Calls that overlap on the GPU (other streams, other host threads) race on the array.
//
// Set-up: the first call on a device (more exactly, in a device context) looks up the array's
// device address with cudaGetSymbolAddress, with that device current, and caches it beside the
// context it belongs to; a new context on the device (after cudaDeviceReset) is looked up again.

#include "../../include/clb200.h"
#include "clb_internal.cuh"
#include "clb_scalar.cuh"

#include <cuda.h>

#include <algorithm>
#include <mutex>
#include <string>

namespace clb {
void set_global_error(const std::string &m);
}

using namespace clb;

namespace {

constexpr int kNoAllocMaxRows = 8192;           // block partial rows of the reduction
constexpr int kNoAllocMaxN = 1024;              // lattices up to 1024^3 fit the rows below
constexpr int kNoAllocBZ = 32, kNoAllocBY = 8;  // the sweep's column tile
constexpr int kNoAllocMaxDevices = 64;

// In host code this name is a host-side stand-in, not a device address: host code only ever uses
// the address cudaGetSymbolAddress returns for the current device.
static __device__ __align__(256) double g_noalloc_partials[kNoAllocMaxRows * kRedSlots];

std::mutex g_mu;
double *g_dev_ptr[kNoAllocMaxDevices] = {};
CUcontext g_dev_ctx[kNoAllocMaxDevices] = {};

// The driver's cuCtxGetCurrent, through the runtime's entry-point query (no -lcuda link).
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
CtxGetCurrentFn ctx_get_current()
{
  static CtxGetCurrentFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<CtxGetCurrentFn>(p);
  }
  return fn;
}

// Fixed-order sum of the block rows, divided by N^3, into the caller's three outputs.
__global__ void __launch_bounds__(256)
    k_noalloc_finalize(const double *__restrict__ partials, int nblocks, double inv_n3, double *__restrict__ out)
{
  __shared__ double smem[(256 / 32) * kRedSlots];
  double v[kRedSlots] = {0, 0, 0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < kRedSlots; ++k) v[k] += partials[(size_t)b * kRedSlots + k];
  block_reduce<kRedSlots, 256>(v, smem);
  if (threadIdx.x == 0)
    for (int k = 0; k < kRedSlots; ++k) out[k] = v[k] * inv_n3;
}

// Device address of the scratch array on the current device, looked up once per device context.
cudaError_t scratch_on_current_device(double **ptr)
{
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_mu);
  // cudaGetSymbolAddress makes the device's primary context current if none is; the context is
  // read after it, so the cache entry names the context the address belongs to.
  if (g_dev_ptr[dev]) {
    CUcontext ctx = nullptr;
    CtxGetCurrentFn get = ctx_get_current();
    if (!get || get(&ctx) != CUDA_SUCCESS || ctx != g_dev_ctx[dev]) g_dev_ptr[dev] = nullptr;
  }
  if (!g_dev_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess) return e;
    CUcontext ctx = nullptr;
    CtxGetCurrentFn get = ctx_get_current();
    if (get) (void)get(&ctx);
    g_dev_ptr[dev] = static_cast<double *>(p);
    g_dev_ctx[dev] = ctx;
  }
  *ptr = g_dev_ptr[dev];
  return cudaSuccess;
}

template <int NS>
void launch(const double *f, const double *p, ScalarArgs a, dim3 grid, double *partials, cudaStream_t s)
{
  k_scalar_sweep<double, NS, kNoAllocBZ, kNoAllocBY, false, false, 3><<<grid, dim3(kNoAllocBZ, kNoAllocBY), 0, s>>>(
      f, p, const_cast<double *>(f), const_cast<double *>(p), a, nullptr, partials);
}

} // namespace

extern "C" int clb_scalar_averages_noalloc(const double *d_fields, const double *d_momenta, int32_t N,
                                           int32_t n_scalars, double dx, double c0, double q, double *d_out,
                                           void *stream)
{
  if (!d_fields || !d_momenta || !d_out) {
    set_global_error("clb_scalar_averages_noalloc: null device pointer");
    return CLB_EINVAL;
  }
  if (N < 2 || N > kNoAllocMaxN) {
    set_global_error("clb_scalar_averages_noalloc: N = " + std::to_string(N) +
                     " is outside [2, 1024]: the fixed scratch array holds 8192 block rows (192 KiB)");
    return CLB_EINVAL;
  }
  if (n_scalars < 1 || n_scalars > 2) {
    set_global_error("clb_scalar_averages_noalloc: n_scalars must be 1 or 2");
    return CLB_EINVAL;
  }
  if (!(dx > 0)) {
    set_global_error("clb_scalar_averages_noalloc: dx must be positive");
    return CLB_EINVAL;
  }
  // A launch error left by earlier work in the process stays with its owner: report it without
  // clearing it, so the error that the launches below return is this call's own.
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) {
    set_global_error(std::string("clb_scalar_averages_noalloc: an earlier CUDA error is pending: ") +
                     cudaGetErrorString(e));
    return CLB_ECUDA;
  }
  double *partials = nullptr;
  e = scratch_on_current_device(&partials);
  if (e != cudaSuccess) {
    set_global_error(std::string("clb_scalar_averages_noalloc: scratch address: ") + cudaGetErrorString(e));
    return CLB_ECUDA;
  }
  const int gx = (N + kNoAllocBZ - 1) / kNoAllocBZ, gy = (N + kNoAllocBY - 1) / kNoAllocBY;
  int xs = std::max(1, std::min(N / 4, (148 * 8 * 2 + gx * gy - 1) / (gx * gy)));
  xs = std::min(xs, kNoAllocMaxRows / (gx * gy));
  const int LX = (N + xs - 1) / xs;
  xs = (N + LX - 1) / LX;
  ScalarArgs a{};
  a.N = N;
  a.LX = LX;
  a.inv_dx2 = 1.0 / (dx * dx);
  const double coup[CLB_MAX_COUPLINGS] = {c0, q};
  a.cs.mc = ScalarModel::couplings(coup);
  const dim3 grid(gx, gy, xs);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (n_scalars == 1)
    launch<1>(d_fields, d_momenta, a, grid, partials, s);
  else
    launch<2>(d_fields, d_momenta, a, grid, partials, s);
  k_noalloc_finalize<<<1, 256, 0, s>>>(partials, gx * gy * xs, 1.0 / ((double)N * N * N), d_out);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_global_error(std::string("clb_scalar_averages_noalloc: launch: ") + cudaGetErrorString(e));
    return CLB_ECUDA;
  }
  return CLB_OK;
}
