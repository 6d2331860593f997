// plc_mean_noalloc: the bulk mean of mod_utils::Mean without any device
// allocation.
//
// Some callers cannot call cudaMalloc: a host application that reserves all
// GPU memory in its own pool at start-up and forbids further allocation, or a
// time loop that must not take the implicit device synchronisation that
// cudaMalloc/cudaFree imply.  They hold their fields in their own buffers and
// have no plc context.  This entry point serves them: the caller passes the
// field, the dzflzi coefficients and the output location (all device
// memory), and the reduction keeps its partial sums in a file-scope
// __device__ array of this library instead of allocated scratch.
//
// Limits and sharing:
//  * the array holds one double-double partial sum per z plane, so nz is at
//    most kNoAllocMaxPlanes (8192); larger nz is rejected with PLC_ERR_SIZE;
//  * the array (2*8192+2 doubles, 128 KiB) is held by every GPU that loads
//    this library until the process exits;
//  * every call shares the one array and it keeps the last call's contents:
//    the arrival counter is cleared at the start of each call, and calls
//    whose kernels overlap on the GPU (different streams) race on it;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (once per device, with that device current), so
//    make that first call before any stream capture.

#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "plc_internal.h"

namespace plc {
namespace {

constexpr int kNoAllocMaxPlanes = 8192;
constexpr int kNoAllocMaxDevices = 64;

// [0, 2*kNoAllocMaxPlanes): (hi, lo) partial sum of each z plane;
// [2*kNoAllocMaxPlanes]: arrival counter (an unsigned int in the first word).
static __device__ __align__(256) double g_noalloc_scratch[2 * kNoAllocMaxPlanes + 2];

std::mutex g_setup_mu;
double *g_scratch_addr[kNoAllocMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on the current device (host code may
// not use the symbol itself as an address).
int scratch_address(double **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(nullptr, e, "cudaGetDevice");
  if (dev < 0 || dev >= kNoAllocMaxDevices)
    return set_error(nullptr, PLC_ERR_ARG, "plc_mean_noalloc: device index out of range");
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(nullptr, e, "cudaGetSymbolAddress");
    g_scratch_addr[dev] = static_cast<double *>(p);
  }
  *out = g_scratch_addr[dev];
  return PLC_OK;
}

// Double-double accumulation (Knuth's TwoSum); the rounded total does not
// depend on the summation order, so this value equals plc_mean's.
struct DD2 {
  double hi, lo;
};
__device__ __forceinline__ void dd2_merge(DD2 &a, double bhi, double blo) {
  const double s = a.hi + bhi;
  const double bb = s - a.hi;
  const double e = (a.hi - (s - bb)) + (bhi - bb);
  a.hi = s;
  a.lo = (a.lo + blo) + e;
}

__device__ void dd2_block_sum(DD2 &v, double *smem /*64*/) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    const double h = __shfl_down_sync(0xffffffffu, v.hi, o);
    const double l = __shfl_down_sync(0xffffffffu, v.lo, o);
    dd2_merge(v, h, l);
  }
  if (lane == 0) {
    smem[wid] = v.hi;
    smem[32 + wid] = v.lo;
  }
  __syncthreads();
  if (wid == 0) {
    DD2 x{0.0, 0.0};
    if (lane < nw) x = DD2{smem[lane], smem[32 + lane]};
    for (int o = 16; o > 0; o >>= 1) {
      const double h = __shfl_down_sync(0xffffffffu, x.hi, o);
      const double l = __shfl_down_sync(0xffffffffu, x.lo, o);
      dd2_merge(x, h, l);
    }
    v = x;
  }
  __syncthreads();
}

// One block per z plane: sum(var*dzflzi(k)) over the plane's interior; the
// last block to finish merges the plane sums and writes the mean.
__global__ void __launch_bounds__(256) k_mean_noalloc(const double *__restrict__ var,
                                                      const double *__restrict__ dzflzi, int nx,
                                                      int ny, int nz, int nxg, int nyg,
                                                      double *scratch, double *out) {
  __shared__ double smem[64];
  __shared__ bool am_last;
  const int k = blockIdx.x + 1;
  const long long X = nx + 2, XY = X * (ny + 2);
  const double dzl = dzflzi[k];
  DD2 s{0.0, 0.0};
  const int nxy = nx * ny;
  for (int t = threadIdx.x; t < nxy; t += blockDim.x) {
    const int j = t / nx, i = t - j * nx;
    dd2_merge(s, var[(i + 1) + X * (j + 1) + XY * k] * dzl, 0.0);
  }
  dd2_block_sum(s, smem);
  unsigned int *counter = reinterpret_cast<unsigned int *>(scratch + 2 * kNoAllocMaxPlanes);
  if (threadIdx.x == 0) {
    scratch[2 * blockIdx.x] = s.hi;
    scratch[2 * blockIdx.x + 1] = s.lo;
    __threadfence();
    am_last = (atomicAdd(counter, 1u) == (unsigned)nz - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  DD2 tot{0.0, 0.0};
  for (int b = threadIdx.x; b < nz; b += blockDim.x)
    dd2_merge(tot, __ldcg(scratch + 2 * b), __ldcg(scratch + 2 * b + 1));
  dd2_block_sum(tot, smem);
  if (threadIdx.x == 0) {
    const double total = tot.hi + tot.lo;
    out[0] = total / nxg / nyg;  // mod_utils.cc:50
    *counter = 0u;
  }
}

}  // namespace
}  // namespace plc

extern "C" int plc_mean_noalloc(const double *d_var, const double *d_dzflzi, int nx, int ny,
                                int nz, int nx_global, int ny_global, double *d_mean,
                                void *stream) {
  using namespace plc;
  if (!d_var || !d_dzflzi || !d_mean)
    return set_error(nullptr, PLC_ERR_ARG, "plc_mean_noalloc: null device pointer");
  if (nx < 1 || ny < 1 || nz < 1 || nx_global == 0 || ny_global == 0)
    return set_error(nullptr, PLC_ERR_ARG, "plc_mean_noalloc: sizes must be positive");
  if (nz > kNoAllocMaxPlanes)
    return set_error(nullptr, PLC_ERR_SIZE,
                     "plc_mean_noalloc: nz = " + std::to_string(nz) +
                         " exceeds the static scratch capacity of 8192 z planes");
  if ((long long)nx * ny > 0x7fffffffll)
    return set_error(nullptr, PLC_ERR_SIZE, "plc_mean_noalloc: nx*ny exceeds 2^31-1");
  double *scratch = nullptr;
  if (int rc = scratch_address(&scratch)) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the arrival counter must start at zero (the array keeps the last call's
  // contents); the plane partials are all rewritten before they are read
  cudaError_t e = cudaMemsetAsync(scratch + 2 * kNoAllocMaxPlanes, 0, sizeof(double), s);
  if (e != cudaSuccess) return cuda_status(nullptr, e, "plc_mean_noalloc: clear counter");
  k_mean_noalloc<<<nz, 256, 0, s>>>(d_var, d_dzflzi, nx, ny, nz, nx_global, ny_global, scratch,
                                    d_mean);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(nullptr, e, "plc_mean_noalloc launch");
  return PLC_OK;
}
