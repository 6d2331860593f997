// Tensor-core kernels of the learned initialiser's generator (plc_gen.cu):
// BF16 channels-last 3-D convolutions as implicit GEMMs on tcgen05 with FP32
// accumulators in tensor memory, periodic in x and y and zero-padded in z
// (the walls) -- the forward pass, the input gradient (the same kernel) and
// the weight gradient.
//
// Tensors are [b][z][y][x][c] with c fastest.  A 3x3x3 convolution is
//   Y[m][co] = sum_{tap, ci} W[tap][co][ci] * X[m + off(tap)][ci],
// tap = (dz+1)*9 + (dy+1)*3 + (dx+1), off(tap) = (dz, dy, dx); the adjoint
// (gradient with respect to X) is the same convolution of dY with the
// weights W'[tap][ci][co] = W[26 - tap][co][ci].
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace plc {
namespace gen {

using bf16 = __nv_bfloat16;

struct Shape {
  int B, Z, Y, X;  // batch and spatial extents
  __host__ __device__ long long voxels() const { return (long long)B * Z * Y * X; }
};

// voxel m -> (b, z, y, x); 32-bit arithmetic (plc_gen_create keeps every
// tensor below 2^31 voxels), a 64-bit division being a long software routine
__device__ __forceinline__ void unflatten(const Shape &s, long long m, int &b, int &z, int &y,
                                          int &x) {
  const unsigned um = (unsigned)m, X = (unsigned)s.X, Y = (unsigned)s.Y, Z = (unsigned)s.Z;
  unsigned r = um / X;
  x = (int)(um - r * X);
  const unsigned r2 = r / Y;
  y = (int)(r - r2 * Y);
  const unsigned r3 = r2 / Z;
  z = (int)(r2 - r3 * Z);
  b = (int)r3;
}
// the voxel at offset (dz, dy, dx) from (b, z, y, x): periodic in x, y; -1
// outside the walls in z
__device__ __forceinline__ long long shifted(const Shape &s, int b, int z, int y, int x, int dz,
                                             int dy, int dx) {
  const int zz = z + dz;
  if (zz < 0 || zz >= s.Z) return -1;
  int yy = y + dy, xx = x + dx;
  yy = yy < 0 ? yy + s.Y : (yy >= s.Y ? yy - s.Y : yy);
  xx = xx < 0 ? xx + s.X : (xx >= s.X ? xx - s.X : xx);
  return (((long long)b * s.Z + zz) * s.Y + yy) * s.X + xx;
}

// ===========================================================================
// The convolution on the 5th-generation tensor cores (tcgen05): a
// block of 128 threads owns 128 voxels x N output channels (N = Co <= 128),
// with the FP32 accumulator tile in tensor memory (TMEM).  K = 27 taps x Ci
// in steps of 16 channels; kTcG steps form a stage: the im2col rows of A and
// the weight rows of B in the K-major core-matrix layout of the UMMA
// descriptors without swizzle (8 rows x 16 bytes per core matrix, the two
// 8-channel halves of a step 128 bytes apart, 8-row groups 256 bytes apart).
// Stages rotate through kTcNB buffers filled by cp.async (zero fill for the
// walls) two stages ahead: thread 0 issues a stage's tcgen05.mma and commits
// them to that buffer's mbarrier, which the threads wait on before refilling
// the buffer.  The epilogue reads the accumulators with tcgen05.ld (warp w
// owns TMEM lanes 32w..32w+31, i.e. voxels) and stores FP32 rows.  Every wait
// is bounded; on a timeout the block flags *err, skips its stores and still
// releases its TMEM.
// ===========================================================================
constexpr int kTcM = 128;
constexpr int kTcG = 2;                        // 16-channel K steps per buffer
constexpr int kTcNB = 3;                       // buffers: copies run two stages ahead of the MMAs
constexpr int kTcABytes = kTcM * 16 * 2;       // 4 KB per step
constexpr long long kTcWaitLimit = 1ll << 24;  // mbarrier polls before giving up

__device__ __forceinline__ unsigned tc_smem_u32(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
// UMMA shared-memory descriptor, K-major, no swizzle: start address, leading
// byte offset (between the two K halves), stride byte offset (between 8-row
// groups), version 1
__device__ __forceinline__ unsigned long long tc_desc(unsigned saddr) {
  return (unsigned long long)((saddr >> 4) & 0x3FFF) | ((unsigned long long)(128 >> 4) << 16) |
         ((unsigned long long)(256 >> 4) << 32) | (1ull << 46);
}
// instruction descriptor: F32 accumulator, BF16 A and B, both K-major, M = 128
__host__ __device__ constexpr unsigned tc_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(n >> 3) << 17) | ((unsigned)(kTcM >> 4) << 24);
}
__device__ __forceinline__ bool tc_wait(unsigned long long *bar, unsigned parity) {
  const unsigned a = tc_smem_u32(bar);
  for (long long it = 0; it < kTcWaitLimit; ++it) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// 16-byte asynchronous copy global -> shared; src_bytes 0 fills zeros
__device__ __forceinline__ void tc_cp16(void *dst, const void *src, unsigned src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(tc_smem_u32(dst)), "l"(src),
               "r"(src_bytes)
               : "memory");
}

// A/B core-matrix layout offset (bytes) of row r, channel half h of one step
__device__ __forceinline__ int tc_off(int r, int h) { return (r >> 3) * 256 + h * 128 + (r & 7) * 16; }

template <int N>
__global__ void __launch_bounds__(128) k_conv3d_tc(Shape s, const bf16 *__restrict__ X,
                                                   const bf16 *__restrict__ W, float *__restrict__ Y,
                                                   int Ci, int *err) {
  constexpr int kNCols = N <= 32 ? 32 : (N <= 64 ? 64 : 128);  // TMEM columns (power of 2)
  constexpr int kBBytes = N * 16 * 2;
  constexpr int kBuf = kTcG * (kTcABytes + kBBytes);
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  __shared__ __align__(8) unsigned long long bar[kTcNB];
  __shared__ unsigned tmem_base_s;
  __shared__ int fail_s;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const long long M = s.voxels();
  const long long m0 = (long long)blockIdx.x * kTcM;
  unsigned char *buf0 = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<unsigned long long>(tc_smem) + 1023ull) & ~1023ull);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tc_smem_u32(&tmem_base_s)),
                 "r"(kNCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (t == 0) {
    for (int q = 0; q < kTcNB; ++q)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem_u32(&bar[q])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fail_s = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = tmem_base_s;

  // this thread's A row: voxel m0 + t
  const long long am = m0 + t;
  int ab = 0, az = 0, ay = 0, ax = 0;
  if (am < M) unflatten(s, am, ab, az, ay, ax);
  const int CC = Ci / 16;  // K steps per tap
  const int KT = 27 * CC;
  const int nstage = (KT + kTcG - 1) / kTcG;
  // copies of stage st into buffer st % kTcNB (one commit group per stage)
  auto load_stage = [&](int st) {
    unsigned char *A = buf0 + (st % kTcNB) * kBuf;
    unsigned char *Bm = A + kTcG * kTcABytes;
#pragma unroll
    for (int g = 0; g < kTcG; ++g) {
      const int kk = st * kTcG + g;
      if (kk >= KT) break;
      unsigned char *Ag = A + g * kTcABytes;
      unsigned char *Bg = Bm + g * kBBytes;
      const int tap = kk / CC, c0 = (kk - tap * CC) * 16;
      const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
      const long long src = am < M ? shifted(s, ab, az, ay, ax, dz, dy, dx) : -1;
      const bf16 *xs = src >= 0 ? X + src * Ci + c0 : X;
      tc_cp16(Ag + tc_off(t, 0), xs, src >= 0 ? 16u : 0u);
      tc_cp16(Ag + tc_off(t, 1), src >= 0 ? xs + 8 : X, src >= 0 ? 16u : 0u);
      for (int e = t; e < 2 * N; e += 128) {
        const int n = e >> 1, h = e & 1;
        tc_cp16(Bg + tc_off(n, h), W + ((long long)tap * N + n) * Ci + c0 + h * 8, 16u);
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  load_stage(0);
  if (nstage > 1) load_stage(1);
  bool ok = true;
  for (int st = 0; st < nstage; ++st) {
    const int b = st % kTcNB;
    unsigned char *A = buf0 + b * kBuf;
    unsigned char *Bm = A + kTcG * kTcABytes;
    if (st + 1 < nstage)
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    else
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    // the copies become visible to the tensor core's async proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (t == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int g = 0; g < kTcG; ++g) {
        const int kk = st * kTcG + g;
        if (kk >= KT) break;
        const unsigned long long da = tc_desc(tc_smem_u32(A + g * kTcABytes));
        const unsigned long long db = tc_desc(tc_smem_u32(Bm + g * kBBytes));
        const unsigned acc = kk > 0 ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
            :
            : "r"(tmem), "l"(da), "l"(db), "r"(tc_idesc(N)), "r"(acc), "r"(0u), "r"(0u), "r"(0u),
              "r"(0u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       tc_smem_u32(&bar[b]))
                   : "memory");
    }
    if (st + 2 < nstage) {
      // buffer (st + 2) % kTcNB was read by the MMAs of stage st - 1
      if (st >= 1) {
        if (t == 0 && !tc_wait(&bar[(st - 1) % kTcNB], (unsigned)(((st - 1) / kTcNB) & 1)))
          fail_s = 1;
        __syncthreads();
        if (fail_s) {
          ok = false;
          break;
        }
      }
      load_stage(st + 2);
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  // all MMAs complete: the last commit covers every earlier tcgen05 operation
  if (ok) {
    const int last = nstage - 1;
    if (t == 0 && !tc_wait(&bar[last % kTcNB], (unsigned)((last / kTcNB) & 1))) fail_s = 1;
    __syncthreads();
    ok = !fail_s;
  }
  if (ok) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const long long row = m0 + warp * 32 + lane;
#pragma unroll
    for (int c0 = 0; c0 < N; c0 += 16) {
      unsigned r[16];
      const unsigned addr = tmem + ((unsigned)(warp * 32) << 16) + (unsigned)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
          "%14,%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
            "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
            "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(addr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < M) {
        float4 *dst = reinterpret_cast<float4 *>(Y + row * N + c0);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          dst[q] = make_float4(__uint_as_float(r[4 * q]), __uint_as_float(r[4 * q + 1]),
                               __uint_as_float(r[4 * q + 2]), __uint_as_float(r[4 * q + 3]));
      }
    }
  } else if (t == 0) {
    atomicExch(err, 1);
    // let the MMAs still in flight finish (bounded) before the TMEM goes back
    for (int q = 0; q < kTcNB; ++q) tc_wait(&bar[q], 0);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kNCols));
  }
}

template <int N, int G = kTcG, int NB = kTcNB>
constexpr size_t tc_smem_bytes() {
  return NB * (size_t)G * (kTcABytes + N * 16 * 2) + 1024;
}


// ---------------------------------------------------------------------------
// Weight gradient on tcgen05: D[co][ci] (+)= sum_m dY[m][co] X[m + off(tap)][ci]
// for one tap over a range of voxels (split K), M = 128 (co, zero-padded
// above Co), N = Ci <= 128, K = 16 voxels per MMA.  Both operands are staged
// MN-major (channels contiguous, as they lie in memory): element (mn, k) of
// a step at (mn/8)*256 + (k/8)*128 + (k%8)*16 + (mn%8)*2 bytes, i.e. stride
// byte offset 256 between 8-channel groups and leading byte offset 128
// between the two 8-voxel halves.  The block's tile is added to dW with
// FP32 atomics.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr unsigned tc_idesc_mn(int n) {
  return tc_idesc(n) | (1u << 15) | (1u << 16);  // A and B MN-major
}
// byte offset of channel mn, voxel k of one MN-major step
__device__ __forceinline__ int tc_off_mn(int mn, int k) {
  return (mn >> 3) * 256 + (k >> 3) * 128 + (k & 7) * 16;
}

constexpr int kWgG = 2;   // K steps (16 voxels each) per buffer of the weight gradient
constexpr int kWgNB = 3;  // buffers: the copies run two stages ahead of the MMAs

template <int N>
__global__ void __launch_bounds__(128) k_conv3d_wgrad_tc(Shape s, const bf16 *__restrict__ dY,
                                                         const bf16 *__restrict__ X,
                                                         float *__restrict__ dW, int Co,
                                                         long long chunk, int *err) {
  constexpr int kNCols = N <= 32 ? 32 : (N <= 64 ? 64 : 128);
  constexpr int kBBytes = N * 16 * 2;
  constexpr int kBuf = kWgG * (kTcABytes + kBBytes);
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  __shared__ __align__(8) unsigned long long bar[kWgNB];
  __shared__ unsigned tmem_base_s;
  __shared__ int fail_s;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int tap = blockIdx.z;
  const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
  const long long M = s.voxels();
  const long long k0 = (long long)blockIdx.x * chunk;
  const long long k1 = k0 + chunk < M ? k0 + chunk : M;
  unsigned char *buf0 = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<unsigned long long>(tc_smem) + 1023ull) & ~1023ull);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tc_smem_u32(&tmem_base_s)),
                 "r"(kNCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (t == 0) {
    for (int q = 0; q < kWgNB; ++q)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem_u32(&bar[q])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fail_s = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = tmem_base_s;

  const long long nsteps = (k1 - k0 + 15) / 16;
  const int nstage = (int)((nsteps + kWgG - 1) / kWgG);
  const int ca = Co / 8, cb = N / 8;  // 16-byte channel chunks of a voxel row
  // the copies of stage st into buffer st % kWgNB (one commit group per stage)
  auto load_stage = [&](int st) {
    unsigned char *A = buf0 + (st % kWgNB) * kBuf;
    unsigned char *Bm = A + kWgG * kTcABytes;
#pragma unroll
    for (int g = 0; g < kWgG; ++g) {
      const long long step = (long long)st * kWgG + g;
      unsigned char *Ag = A + g * kTcABytes;
      unsigned char *Bg = Bm + g * kBBytes;
      const long long mb = k0 + step * 16;
      for (int e = t; e < 16 * 16; e += 128) {  // A: 16 voxels x 128 co
        const int k = e >> 4, q = e & 15;
        const long long m = mb + k;
        const bool v = step < nsteps && q < ca && m < k1;
        tc_cp16(Ag + tc_off_mn(q * 8, k), v ? (const void *)(dY + m * Co + q * 8) : (const void *)dY,
                v ? 16u : 0u);
      }
      for (int e = t; e < 16 * cb; e += 128) {  // B: 16 voxels x N ci of the shifted input
        const int k = e / cb, q = e - k * cb;
        const long long m = mb + k;
        long long src = -1;
        if (step < nsteps && m < k1) {
          int bb, z, y, x;
          unflatten(s, m, bb, z, y, x);
          src = shifted(s, bb, z, y, x, dz, dy, dx);
        }
        tc_cp16(Bg + tc_off_mn(q * 8, k), src >= 0 ? (const void *)(X + src * N + q * 8) : (const void *)X,
                src >= 0 ? 16u : 0u);
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  load_stage(0);
  if (nstage > 1) load_stage(1);
  bool ok = true;
  for (int st = 0; st < nstage; ++st) {
    const int b = st % kWgNB;
    unsigned char *A = buf0 + b * kBuf;
    unsigned char *Bm = A + kWgG * kTcABytes;
    // stage st's copies landed (stage st + 1 may still be in flight)
    if (st + 1 < nstage)
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    else
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (t == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int g = 0; g < kWgG; ++g) {
        const long long step = (long long)st * kWgG + g;
        if (step >= nsteps) break;
        const unsigned long long da = tc_desc(tc_smem_u32(A + g * kTcABytes));
        const unsigned long long db = tc_desc(tc_smem_u32(Bm + g * kBBytes));
        const unsigned acc = step > 0 ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
            :
            : "r"(tmem), "l"(da), "l"(db), "r"(tc_idesc_mn(N)), "r"(acc), "r"(0u), "r"(0u),
              "r"(0u), "r"(0u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       tc_smem_u32(&bar[b]))
                   : "memory");
    }
    if (st + 2 < nstage) {
      // buffer (st + 2) % kWgNB was read by the MMAs of stage st - 1
      if (st >= 1) {
        if (t == 0 && !tc_wait(&bar[(st - 1) % kWgNB], (unsigned)(((st - 1) / kWgNB) & 1)))
          fail_s = 1;
        __syncthreads();
        if (fail_s) {
          ok = false;
          break;
        }
      }
      load_stage(st + 2);
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  if (ok && nstage > 0) {
    const int last = nstage - 1;
    if (t == 0 && !tc_wait(&bar[last % kWgNB], (unsigned)((last / kWgNB) & 1))) fail_s = 1;
    __syncthreads();
    ok = !fail_s;
  }
  if (ok && nstage > 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int co = warp * 32 + lane;
#pragma unroll
    for (int c0 = 0; c0 < N; c0 += 16) {
      unsigned r[16];
      const unsigned addr = tmem + ((unsigned)(warp * 32) << 16) + (unsigned)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
          "%14,%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
            "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
            "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(addr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (co < Co) {
        float *dst = dW + ((long long)tap * Co + co) * N + c0;
#pragma unroll
        for (int q = 0; q < 16; ++q) atomicAdd(dst + q, __uint_as_float(r[q]));
      }
    }
  } else if (!ok && t == 0) {
    atomicExch(err, 1);
    for (int q = 0; q < kWgNB; ++q) tc_wait(&bar[q], 0);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kNCols));
  }
}

}  // namespace gen
}  // namespace plc
