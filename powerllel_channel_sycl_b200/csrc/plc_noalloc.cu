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
//  * the array holds kNoAllocMaxPartials (8192) double-double partial sums,
//    at least one per z plane, so nz is at most 8192; larger nz is rejected
//    with PLC_ERR_SIZE.  Thin channels split each plane over several blocks
//    (up to 8192 / nz of them) so that the reduction still spreads over the
//    GPU's SMs;
//  * the array (2*8192+2 doubles, 128 KiB) is held by every GPU that loads
//    this library until the process exits;
//  * every call shares the one array and it keeps the last call's contents:
//    the arrival counter is cleared at the start of each call, and calls
//    whose kernels overlap on the GPU (different streams) race on it;
//  * the array's device address belongs to the CUDA context that loaded the
//    library's module.  A call on a stream that is not being captured looks
//    the address up again (cudaGetSymbolAddress, with the caller's device and
//    context current) and remembers it for that context; a call made during
//    stream capture uses the remembered address, so make one call outside
//    capture first in every context (after a cudaDeviceReset, too).

#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "plc_internal.h"

namespace plc {
namespace {

constexpr int kNoAllocMaxPartials = 8192;
constexpr int kNoAllocMaxContexts = 64;
// blocks a launch aims at: four per SM of a B200
constexpr int kNoAllocTargetBlocks = 4 * 148;

// [0, 2*kNoAllocMaxPartials): (hi, lo) partial sum of each block;
// [2*kNoAllocMaxPartials]: arrival counter (an unsigned int in the first word).
static __device__ __align__(256) double g_noalloc_scratch[2 * kNoAllocMaxPartials + 2];

struct ContextAddress {
  CUcontext ctx;
  double *addr;
};
std::mutex g_setup_mu;
ContextAddress g_addr[kNoAllocMaxContexts];
int g_naddr = 0;

// The calling thread's current CUDA context, through the driver entry point
// that the runtime resolves (no link-time dependency on libcuda).
int current_context(CUcontext *out) {
  using GetCurrentFn = CUresult (*)(CUcontext *);
  static GetCurrentFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q);
    if (e != cudaSuccess) return cuda_status(nullptr, e, "cudaGetDriverEntryPoint");
    if (q != cudaDriverEntryPointSuccess || !p)
      return set_error(nullptr, PLC_ERR_CUDA, "plc_mean_noalloc: cuCtxGetCurrent unavailable");
    fn = reinterpret_cast<GetCurrentFn>(p);
  }
  if (fn(out) != CUDA_SUCCESS)
    return set_error(nullptr, PLC_ERR_CUDA, "plc_mean_noalloc: cuCtxGetCurrent failed");
  return PLC_OK;
}

// Device address of g_noalloc_scratch in the current context (host code may
// not use the symbol itself as an address).  Outside stream capture it is
// looked up afresh, which also covers a context rebuilt by cudaDeviceReset;
// during capture the address remembered for this context is used.
int scratch_address(cudaStream_t s, double **out) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(s, &cs);
  if (e != cudaSuccess) return cuda_status(nullptr, e, "cudaStreamIsCapturing");
  if (cs == cudaStreamCaptureStatusNone) {
    // the first runtime call makes the device's primary context current
    // when the caller has none
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(nullptr, e, "cudaGetSymbolAddress");
    CUcontext ctx = nullptr;
    if (int rc = current_context(&ctx)) return rc;
    std::lock_guard<std::mutex> lk(g_setup_mu);
    int slot = 0;
    while (slot < g_naddr && g_addr[slot].ctx != ctx) ++slot;
    if (slot == g_naddr) {
      if (g_naddr == kNoAllocMaxContexts) slot = g_naddr - 1;  // overwrite the newest
      else ++g_naddr;
    }
    g_addr[slot] = ContextAddress{ctx, static_cast<double *>(p)};
    *out = static_cast<double *>(p);
    return PLC_OK;
  }
  CUcontext ctx = nullptr;
  if (int rc = current_context(&ctx)) return rc;
  std::lock_guard<std::mutex> lk(g_setup_mu);
  for (int slot = 0; slot < g_naddr; ++slot)
    if (g_addr[slot].ctx == ctx) {
      *out = g_addr[slot].addr;
      return PLC_OK;
    }
  return set_error(nullptr, PLC_ERR_ARG,
                   "plc_mean_noalloc: first call in this CUDA context made during stream "
                   "capture; call it once outside capture first");
}

// Double-double accumulation (Knuth's TwoSum): each addition's rounding error
// is carried in the low word, so the rounded total is nearly independent of
// the summation order and agrees with plc_mean's to within an ulp.
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

// `chunks` blocks per z plane: sum(var*dzflzi(k)) over a slice of the
// plane's interior; the last block to finish merges the block sums and
// writes the mean.
__global__ void __launch_bounds__(256) k_mean_noalloc(const double *__restrict__ var,
                                                      const double *__restrict__ dzflzi, int nx,
                                                      int ny, int nz, int chunks, int nxg,
                                                      int nyg, double *scratch, double *out) {
  __shared__ double smem[64];
  __shared__ bool am_last;
  const int k = blockIdx.x / chunks + 1;
  const int c = blockIdx.x - (k - 1) * chunks;
  const long long X = nx + 2, XY = X * (ny + 2);
  const double dzl = dzflzi[k];
  DD2 s{0.0, 0.0};
  const long long nxy = (long long)nx * ny;
  const long long per = (nxy + chunks - 1) / chunks;
  const long long t0 = c * per, t1 = t0 + per < nxy ? t0 + per : nxy;
  for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
    const long long j = t / nx, i = t - j * nx;
    dd2_merge(s, var[(i + 1) + X * (j + 1) + XY * k] * dzl, 0.0);
  }
  dd2_block_sum(s, smem);
  unsigned int *counter = reinterpret_cast<unsigned int *>(scratch + 2 * kNoAllocMaxPartials);
  if (threadIdx.x == 0) {
    scratch[2 * blockIdx.x] = s.hi;
    scratch[2 * blockIdx.x + 1] = s.lo;
    __threadfence();
    am_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  DD2 tot{0.0, 0.0};
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
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
  if (nz > kNoAllocMaxPartials)
    return set_error(nullptr, PLC_ERR_SIZE,
                     "plc_mean_noalloc: nz = " + std::to_string(nz) +
                         " exceeds the static scratch capacity of 8192 z planes");
  const long long nxy = (long long)nx * ny;
  // blocks per plane: enough to spread a thin channel over the SMs, at most
  // one per 256 points of a plane and 8192 in all
  long long chunks = (kNoAllocTargetBlocks + nz - 1) / nz;
  if (chunks > (nxy + 255) / 256) chunks = (nxy + 255) / 256;
  if (chunks > kNoAllocMaxPartials / nz) chunks = kNoAllocMaxPartials / nz;
  if (chunks < 1) chunks = 1;
  double *scratch = nullptr;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (int rc = scratch_address(s, &scratch)) return rc;
  // the arrival counter must start at zero (the array keeps the last call's
  // contents); the block partials are all rewritten before they are read
  cudaError_t e = cudaMemsetAsync(scratch + 2 * kNoAllocMaxPartials, 0, sizeof(double), s);
  if (e != cudaSuccess) return cuda_status(nullptr, e, "plc_mean_noalloc: clear counter");
  k_mean_noalloc<<<(int)(nz * chunks), 256, 0, s>>>(d_var, d_dzflzi, nx, ny, nz, (int)chunks,
                                                    nx_global, ny_global, scratch, d_mean);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(nullptr, e, "plc_mean_noalloc launch");
  return PLC_OK;
}
