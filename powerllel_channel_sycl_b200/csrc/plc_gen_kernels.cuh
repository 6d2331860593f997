// Kernels of the learned initialiser's generator (plc_gen.cu): BF16
// channels-last 3-D convolutions as implicit GEMMs on the tensor cores
// (mma.sync m16n8k16, FP32 accumulation), periodic in x and y and
// zero-padded in z (the walls), with the FiLM / activation, upsampling,
// statistics-loss and optimiser kernels around them.
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

__device__ __forceinline__ void ldsm_x4(unsigned (&r)[4], const void *smem) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}
__device__ __forceinline__ void ldsm_x4_t(unsigned (&r)[4], const void *smem) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}
// D = A * B + D, A 16x16 row-major BF16, B 16x8 column-major BF16, D FP32
__device__ __forceinline__ void mma_bf16(float (&d)[4], const unsigned (&a)[4], unsigned b0,
                                         unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// voxel m -> (b, z, y, x)
__device__ __forceinline__ void unflatten(const Shape &s, long long m, int &b, int &z, int &y,
                                          int &x) {
  x = (int)(m % s.X);
  long long r = m / s.X;
  y = (int)(r % s.Y);
  r /= s.Y;
  z = (int)(r % s.Z);
  b = (int)(r / s.Z);
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

// ---------------------------------------------------------------------------
// Forward convolution (and, with the transposed-flipped weights, the
// gradient with respect to the input).  Block: 64 voxels x BN output
// channels, 4 warps of 16 voxels each; K runs over 27 taps x Ci in chunks
// of 16 channels, staged in shared memory (rows padded to 48 bytes: the
// ldmatrix row addresses of a phase fall in distinct banks).
// ---------------------------------------------------------------------------
constexpr int kConvBM = 64;
constexpr int kSmemRow = 24;  // bf16 per staged row (16 + 8 padding)

template <int BN>
__global__ void __launch_bounds__(128) k_conv3d(Shape s, const bf16 *__restrict__ X,
                                                const bf16 *__restrict__ W, float *__restrict__ Y,
                                                int Ci, int Co) {
  __shared__ __align__(16) bf16 As[kConvBM][kSmemRow];
  __shared__ __align__(16) bf16 Bs[BN][kSmemRow];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const long long M = s.voxels();
  const long long m0 = (long long)blockIdx.x * kConvBM;
  const int n0 = blockIdx.y * BN;
  // the A row this thread stages (two threads per row, 8 channels each)
  const int arow = t >> 1, ahalf = (t & 1) * 8;
  const long long am = m0 + arow;
  int ab = 0, az = 0, ay = 0, ax = 0;
  if (am < M) unflatten(s, am, ab, az, ay, ax);
  float acc[BN / 8][4];
#pragma unroll
  for (int j = 0; j < BN / 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
  for (int tap = 0; tap < 27; ++tap) {
    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
    const long long src = am < M ? shifted(s, ab, az, ay, ax, dz, dy, dx) : -1;
    for (int c0 = 0; c0 < Ci; c0 += 16) {
      uint4 va = make_uint4(0u, 0u, 0u, 0u);
      if (src >= 0) va = *reinterpret_cast<const uint4 *>(X + src * Ci + c0 + ahalf);
      *reinterpret_cast<uint4 *>(&As[arow][ahalf]) = va;
      if (t < 2 * BN) {
        const int brow = t >> 1, bhalf = (t & 1) * 8;
        *reinterpret_cast<uint4 *>(&Bs[brow][bhalf]) = *reinterpret_cast<const uint4 *>(
            W + ((long long)tap * Co + n0 + brow) * Ci + c0 + bhalf);
      }
      __syncthreads();
      unsigned a[4];
      ldsm_x4(a, &As[warp * 16 + (lane & 15)][(lane >> 4) * 8]);
#pragma unroll
      for (int j = 0; j < BN / 16; ++j) {
        unsigned b[4];
        ldsm_x4(b, &Bs[j * 16 + (lane & 7) + ((lane >> 4) << 3)][((lane >> 3) & 1) * 8]);
        mma_bf16(acc[2 * j], a, b[0], b[1]);
        mma_bf16(acc[2 * j + 1], a, b[2], b[3]);
      }
      __syncthreads();
    }
  }
  const int g = lane >> 2, tig = lane & 3;
  const long long r0 = m0 + warp * 16 + g, r1 = r0 + 8;
#pragma unroll
  for (int j = 0; j < BN / 8; ++j) {
    const int col = n0 + j * 8 + tig * 2;
    if (r0 < M) *reinterpret_cast<float2 *>(Y + r0 * Co + col) = make_float2(acc[j][0], acc[j][1]);
    if (r1 < M) *reinterpret_cast<float2 *>(Y + r1 * Co + col) = make_float2(acc[j][2], acc[j][3]);
  }
}

// ---------------------------------------------------------------------------
// Weight gradient: dW[tap][co][ci] += sum_m dY[m][co] * X[m + off(tap)][ci].
// Block: 64 co x 64 ci of one tap over a range of voxels (split K, FP32
// atomics at the end); chunks of 16 voxels staged as [m][co] and [m][ci]
// and read transposed by ldmatrix.trans.
// ---------------------------------------------------------------------------
constexpr int kWgRow = 72;  // bf16 per staged row (64 + 8 padding)

__global__ void __launch_bounds__(128) k_conv3d_wgrad(Shape s, const bf16 *__restrict__ dY,
                                                      const bf16 *__restrict__ X,
                                                      float *__restrict__ dW, int Ci, int Co,
                                                      long long chunk) {
  __shared__ __align__(16) bf16 As[16][kWgRow];
  __shared__ __align__(16) bf16 Bs[16][kWgRow];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int tap = blockIdx.z;
  const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
  const int tiles_ci = (Ci + 63) / 64;
  const int co0 = (blockIdx.y / tiles_ci) * 64, ci0 = (blockIdx.y % tiles_ci) * 64;
  const int nco = Co - co0 < 64 ? Co - co0 : 64;  // 16, 32, 48 or 64
  const int nci = Ci - ci0 < 64 ? Ci - ci0 : 64;
  const long long M = s.voxels();
  const long long k0 = (long long)blockIdx.x * chunk;
  const long long k1 = k0 + chunk < M ? k0 + chunk : M;
  float acc[8][4];
#pragma unroll
  for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
  // staging: 16 rows x 64 channels = 128 chunks of 8 bf16, one per thread
  const int srow = t >> 3, scol = (t & 7) * 8;
  for (long long mb = k0; mb < k1; mb += 16) {
    const long long m = mb + srow;
    uint4 va = make_uint4(0u, 0u, 0u, 0u), vb = make_uint4(0u, 0u, 0u, 0u);
    if (m < k1) {
      if (scol < nco) va = *reinterpret_cast<const uint4 *>(dY + m * Co + co0 + scol);
      if (scol < nci) {
        int b, z, y, x;
        unflatten(s, m, b, z, y, x);
        const long long src = shifted(s, b, z, y, x, dz, dy, dx);
        if (src >= 0) vb = *reinterpret_cast<const uint4 *>(X + src * Ci + ci0 + scol);
      }
    }
    *reinterpret_cast<uint4 *>(&As[srow][scol]) = va;
    *reinterpret_cast<uint4 *>(&Bs[srow][scol]) = vb;
    __syncthreads();
    if (warp * 16 < nco) {
      unsigned a[4];
      {
        const int q = lane >> 3, r = lane & 7;
        ldsm_x4_t(a, &As[r + (q >> 1) * 8][warp * 16 + (q & 1) * 8]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (j * 16 < nci) {
          unsigned b[4];
          const int q = lane >> 3, r = lane & 7;
          ldsm_x4_t(b, &Bs[r + (q & 1) * 8][j * 16 + (q >> 1) * 8]);
          mma_bf16(acc[2 * j], a, b[0], b[1]);
          mma_bf16(acc[2 * j + 1], a, b[2], b[3]);
        }
      }
    }
    __syncthreads();
  }
  if (warp * 16 >= nco) return;
  const int g = lane >> 2, tig = lane & 3;
  const int co_a = co0 + warp * 16 + g, co_b = co_a + 8;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int ci = ci0 + j * 8 + tig * 2;
    if (j * 8 >= nci) continue;
    float *wa = dW + ((long long)tap * Co + co_a) * Ci + ci;
    float *wb = dW + ((long long)tap * Co + co_b) * Ci + ci;
    atomicAdd(wa, acc[j][0]);
    atomicAdd(wa + 1, acc[j][1]);
    atomicAdd(wb, acc[j][2]);
    atomicAdd(wb + 1, acc[j][3]);
  }
}

}  // namespace gen
}  // namespace plc
