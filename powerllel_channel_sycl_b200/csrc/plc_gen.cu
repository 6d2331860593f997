// Learned initialiser: a conditional 3-D convolutional generator that
// proposes a developed-turbulence velocity field for a given Re_tau.  No
// counterpart in the reference (its initial fields are the laminar profiles
// plus cell noise of mod_initFlow.cc).
//
// Network (levels l = 0..3, coarse to fine, each doubling the grid):
//   level 0: latent (Gaussian, C_lat channels on nx/8 x ny/8 x nz/8)
//            -> conv -> FiLM -> LReLU -> conv -> FiLM -> LReLU
//   level l: nearest x2 upsampling -> conv -> FiLM -> LReLU -> conv -> FiLM -> LReLU
//   output:  conv (C_3 -> 3 used of 16) -> FiLM   (u, v, w at the cell centres)
// Convolutions are 3x3x3, periodic in x and y, zero-padded in z (the walls).
// FiLM is the conditioning: per z-plane and channel, gamma = 1 + A0 + A1 r and
// beta = B0 + B1 r with r = (Re_tau - 260) / 140, which also gives the
// network its wall-normal position.  Weights and activations are BF16 with
// FP32 accumulation; master weights, gradients and Adam moments FP32.
//
// Training matches statistics: per z-plane of the output, the means, second
// moments, u-w covariance and the lagged covariances of u, v, w at 1, 2, 4, 8
// cells along x and y, against the same statistics of DNS snapshots
// coarse-grained to the generator's grid (plc_gen_stats_of).  The loss is the
// mean squared, scale-normalised difference; its gradient is analytic.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <random>
#include <string>
#include <vector>

#include "plc_gen_kernels.cuh"
#include "plc_internal.h"

using plc::gen::bf16;
using plc::gen::Shape;

namespace plc {
namespace gen {
namespace {

constexpr int kLevels = 4;
constexpr int kOutC = 16;  // output channels (u, v, w and zero padding)

// statistics per z-plane: 0-2 means u v w; 3-5 variances; 6 u-w covariance;
// 7 + f*8 + dir*4 + q: lagged covariance of field f along x (dir 0) or y
// (dir 1) at a lag of 2^q cells
constexpr int kLagBase = 7;

__device__ __forceinline__ float lrelu(float h) { return h > 0.f ? h : 0.2f * h; }

// ---- FiLM tables: gamma, beta per (sample, plane, channel) -----------------
__global__ void k_film_tables(const float *__restrict__ film, int Z, int C, const float *r, int B,
                              float *gam, float *bet) {
  const long long n = (long long)B * Z * C;
  const long long zc = (long long)Z * C;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(e / zc);
    const long long q = e - b * zc;  // z*C + c
    const float rb = r[b];
    gam[e] = 1.f + film[q] + film[zc + q] * rb;
    bet[e] = film[2 * zc + q] + film[3 * zc + q] * rb;
  }
}

// act = lrelu(gamma * pre + beta) in BF16, or (output layer) out = gamma * pre + beta
template <bool ACT>
__global__ void k_film_fwd(Shape s, int C, const float *__restrict__ pre,
                           const float *__restrict__ gam, const float *__restrict__ bet,
                           bf16 *act, float *out) {
  const long long n = s.voxels() * C;
  const long long plane = (long long)s.Y * s.X;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const long long m = e / C;
    const int c = (int)(e - m * C);
    const long long bz = m / plane;  // b*Z + z
    const long long q = bz * C + c;
    const float h = gam[q] * pre[e] + bet[q];
    if (ACT)
      act[e] = __float2bfloat16(lrelu(h));
    else
      out[e] = h;
  }
}

// Backward of FiLM (+ LReLU): dpre = dact * slope * gamma (BF16, the operand
// of the weight and input gradients), dgamma / dbeta summed over each plane.
// One block per (sample, plane).
template <bool ACT>
__global__ void __launch_bounds__(256) k_film_bwd(Shape s, int C, const float *__restrict__ dact,
                                                  const float *__restrict__ pre,
                                                  const float *__restrict__ gam,
                                                  const float *__restrict__ bet, bf16 *dpre,
                                                  float *dgam, float *dbet) {
  __shared__ float sg[128], sb[128];
  for (int c = threadIdx.x; c < C; c += blockDim.x) sg[c] = sb[c] = 0.f;
  __syncthreads();
  const long long bz = blockIdx.x;
  const long long plane = (long long)s.Y * s.X;
  const long long base = bz * plane * C;
  const float *g = gam + bz * C, *be = bet + bz * C;
  for (long long e = threadIdx.x; e < plane * C; e += blockDim.x) {
    const int c = (int)(e % C);
    const float p = pre[base + e];
    float dh = dact[base + e];
    if (ACT) dh *= (g[c] * p + be[c]) > 0.f ? 1.f : 0.2f;
    dpre[base + e] = __float2bfloat16(dh * g[c]);
    atomicAdd(&sg[c], dh * p);
    atomicAdd(&sb[c], dh);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < C; c += blockDim.x) {
    dgam[bz * C + c] = sg[c];
    dbet[bz * C + c] = sb[c];
  }
}

// gradients of the FiLM parameters from the per-sample tables
__global__ void k_film_param_grad(int Z, int C, int B, const float *r, const float *dgam,
                                  const float *dbet, float *grad) {
  const long long zc = (long long)Z * C;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < zc;
       q += (long long)gridDim.x * blockDim.x) {
    float a0 = 0.f, a1 = 0.f, b0 = 0.f, b1 = 0.f;
    for (int b = 0; b < B; ++b) {
      const float dg = dgam[b * zc + q], db = dbet[b * zc + q];
      a0 += dg;
      a1 += dg * r[b];
      b0 += db;
      b1 += db * r[b];
    }
    grad[q] += a0;
    grad[zc + q] += a1;
    grad[2 * zc + q] += b0;
    grad[3 * zc + q] += b1;
  }
}

// nearest-neighbour x2 upsampling of BF16 (8 channels per thread)
__global__ void k_upsample(Shape fine, int C, const bf16 *__restrict__ in, bf16 *out) {
  const int c8 = C / 8;
  const long long n = fine.voxels() * c8;
  const Shape coarse{fine.B, fine.Z / 2, fine.Y / 2, fine.X / 2};
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const long long m = e / c8;
    const int q = (int)(e - m * c8);
    int b, z, y, x;
    unflatten(fine, m, b, z, y, x);
    const long long mc = (((long long)b * coarse.Z + z / 2) * coarse.Y + y / 2) * coarse.X + x / 2;
    reinterpret_cast<uint4 *>(out)[m * c8 + q] = reinterpret_cast<const uint4 *>(in)[mc * c8 + q];
  }
}

// its adjoint: the sum over the 8 children (FP32)
__global__ void k_upsample_bwd(Shape coarse, int C, const float *__restrict__ dfine, float *dcoarse) {
  const long long n = coarse.voxels() * C;
  const Shape fine{coarse.B, coarse.Z * 2, coarse.Y * 2, coarse.X * 2};
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const long long m = e / C;
    const int c = (int)(e - m * C);
    int b, z, y, x;
    unflatten(coarse, m, b, z, y, x);
    float acc = 0.f;
    for (int d = 0; d < 8; ++d) {
      const long long mf = (((long long)b * fine.Z + 2 * z + (d >> 2)) * fine.Y + 2 * y +
                            ((d >> 1) & 1)) * fine.X + 2 * x + (d & 1);
      acc += dfine[mf * C + c];
    }
    dcoarse[e] = acc;
  }
}

// SplitMix64 (Steele, Lea and Flood, 2014): a counter-based stream
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
__device__ __forceinline__ float uniform01(unsigned long long h) {
  return ((h >> 40) + 0.5f) * (1.0f / 16777216.0f);  // 24 bits, in (0, 1)
}

// Gaussian latent (Box-Muller on two uniforms of the stream)
__global__ void k_latent(long long n, unsigned long long seed, bf16 *z) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const unsigned long long h1 = splitmix64(seed * 0x100000001B3ull + 2 * (unsigned long long)e);
    const unsigned long long h2 = splitmix64(h1 ^ 0xD1B54A32D192ED03ull);
    const float u1 = uniform01(h1), u2 = uniform01(h2);
    z[e] = __float2bfloat16(sqrtf(-2.f * logf(u1)) * cospif(2.f * u2));
  }
}

// batch targets drawn from the stream (training), and their r values
__global__ void k_pick_targets(unsigned long long seed, int B, int ntargets, const float *re_tau,
                               int *tidx, float *r) {
  for (int b = threadIdx.x; b < B; b += blockDim.x) {
    const unsigned long long h = splitmix64(seed * 0x9E3779B97F4A7C15ull + b);
    const int t = (int)(h % (unsigned long long)ntargets);
    tidx[b] = t;
    r[b] = (re_tau[t] - 260.f) / 140.f;
  }
}

// ---- statistics of u, v, w (channels 0-2 of OC) per (sample, plane) --------
__device__ __forceinline__ int wrapi(int a, int n) { return a >= n ? a - n : (a < 0 ? a + n : a); }

// One block per (sample, plane): raw sums in FP64, then the statistics; in
// loss mode the plane's loss term and the coefficients dL/dstat.
__global__ void __launch_bounds__(256) k_stats(Shape s, int OC, const float *__restrict__ out,
                                               const int *__restrict__ tidx,
                                               const float *__restrict__ targets, float sc_mean,
                                               float sc_var, float *coef, float *means,
                                               double *loss, double *stats) {
  constexpr int NS = PLC_GEN_NSTAT;
  __shared__ double red[8][NS];
  const int bz = blockIdx.x, b = bz / s.Z, z = bz - b * s.Z;
  const long long base = (long long)bz * s.Y * s.X;
  double a[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) a[q] = 0.0;
  for (int p = threadIdx.x; p < s.Y * s.X; p += blockDim.x) {
    const int y = p / s.X, x = p - y * s.X;
    const float *o = out + (base + p) * OC;
    const double f[3] = {o[0], o[1], o[2]};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      a[c] += f[c];
      a[3 + c] += f[c] * f[c];
    }
    a[6] += f[0] * f[2];
#pragma unroll
    for (int qd = 0; qd < 4; ++qd) {
      const int lag = 1 << qd;
      const float *ox = out + (base + (long long)y * s.X + wrapi(x + lag, s.X)) * OC;
      const float *oy = out + (base + (long long)wrapi(y + lag, s.Y) * s.X + x) * OC;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        a[kLagBase + c * 8 + qd] += f[c] * (double)ox[c];
        a[kLagBase + c * 8 + 4 + qd] += f[c] * (double)oy[c];
      }
    }
  }
  // warp sums, then across the 8 warps
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    double v = a[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][q] = v;
  }
  __syncthreads();
  if (warp != 0) return;
  // warp 0: lane q < NS finishes statistic q
  __shared__ double raw[NS];
  const int q = lane;
  const bool valid = q < NS;
  if (valid) {
    double sum = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) sum += red[w][q];
    raw[q] = sum / ((double)s.Y * s.X);
  }
  __syncwarp();
  double l = 0.0;
  if (valid) {
    const double mu[3] = {raw[0], raw[1], raw[2]};
    double st;
    if (q < 3) st = raw[q];
    else if (q < 6) st = raw[q] - mu[q - 3] * mu[q - 3];
    else if (q == 6) st = raw[6] - mu[0] * mu[2];
    else {
      const int c = (q - kLagBase) / 8;
      st = raw[q] - mu[c] * mu[c];
    }
    if (stats) stats[(long long)bz * NS + q] = st;
    if (q < 3 && means) means[bz * 3 + q] = (float)mu[q];
    if (coef) {
      const double T = targets[((long long)tidx[b] * s.Z + z) * NS + q];
      const double sc = q < 3 ? sc_mean : sc_var;
      const double d = (st - T) / sc;
      const double norm = 1.0 / ((double)s.B * s.Z);
      coef[bz * NS + q] = (float)(2.0 * d / sc * norm);
      l = d * d * norm;
    }
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
  if (lane == 0 && coef) atomicAdd(loss, l);
}

// dL/d(u, v, w) from the coefficients of k_stats (statistics of raw means
// and products: see the derivation at the top of the file)
__global__ void k_stats_grad(Shape s, int OC, const float *__restrict__ out,
                             const float *__restrict__ coef, const float *__restrict__ means,
                             float *dout) {
  constexpr int NS = PLC_GEN_NSTAT;
  const long long n = s.voxels();
  const float inv_a = 1.f / (float)(s.Y * s.X);
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n;
       m += (long long)gridDim.x * blockDim.x) {
    int b, z, y, x;
    unflatten(s, m, b, z, y, x);
    const long long bz = (long long)b * s.Z + z;
    const long long base = bz * s.Y * s.X;
    const float *g = coef + bz * NS;
    const float *mu = means + bz * 3;
    const float *o = out + m * OC;
    float d[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) d[c] = g[c] + 2.f * g[3 + c] * (o[c] - mu[c]);
    d[0] += g[6] * (o[2] - mu[2]);
    d[2] += g[6] * (o[0] - mu[0]);
#pragma unroll
    for (int qd = 0; qd < 4; ++qd) {
      const int lag = 1 << qd;
      const float *xp = out + (base + (long long)y * s.X + wrapi(x + lag, s.X)) * OC;
      const float *xm = out + (base + (long long)y * s.X + wrapi(x - lag, s.X)) * OC;
      const float *yp = out + (base + (long long)wrapi(y + lag, s.Y) * s.X + x) * OC;
      const float *ym = out + (base + (long long)wrapi(y - lag, s.Y) * s.X + x) * OC;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        d[c] += g[kLagBase + c * 8 + qd] * (xp[c] + xm[c] - 2.f * mu[c]);
        d[c] += g[kLagBase + c * 8 + 4 + qd] * (yp[c] + ym[c] - 2.f * mu[c]);
      }
    }
    float *dd = dout + m * OC;
    dd[0] = d[0] * inv_a;
    dd[1] = d[1] * inv_a;
    dd[2] = d[2] * inv_a;
    for (int c = 3; c < OC; ++c) dd[c] = 0.f;
  }
}

// ---- optimiser and weight copies ------------------------------------------
__global__ void k_adam(long long n, float *p, const float *g, float *m, float *v, float lr,
                       float b1, float b2, float eps, float bc1, float bc2) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const float ge = g[e];
    const float me = b1 * m[e] + (1.f - b1) * ge;
    const float ve = b2 * v[e] + (1.f - b2) * ge * ge;
    m[e] = me;
    v[e] = ve;
    p[e] -= lr * (me / bc1) / (sqrtf(ve / bc2) + eps);
  }
}

// BF16 copies of a layer's weights: W[tap][co][ci] and the adjoint's
// W'[tap][ci][co] = W[26 - tap][co][ci]
__global__ void k_weights_bf16(const float *__restrict__ w, int ci, int co, bf16 *wb, bf16 *wt) {
  const long long n = 27ll * ci * co;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int tap = (int)(e / ((long long)ci * co));
    const long long r = e - (long long)tap * ci * co;
    const int o = (int)(r / ci), i = (int)(r - (long long)o * ci);
    const bf16 x = __float2bfloat16(w[e]);
    wb[e] = x;
    wt[((long long)(26 - tap) * ci + i) * co + o] = x;
  }
}

// ---- DNS fields <-> the generator's grid -----------------------------------
// Box average of the cell-centred velocities (u + u_crf, v, w) over the
// rx x ry x rz cells of each generator voxel, weighted by dzf.
template <class T>
__global__ void k_coarsen(Geo g, const T *__restrict__ u, const T *__restrict__ v,
                          const T *__restrict__ w, double u_crf, Shape s, int rx, int ry, int rz,
                          float *out) {
  const long long n = (long long)s.Z * s.Y * s.X;
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n;
       m += (long long)gridDim.x * blockDim.x) {
    const int X = (int)(m % s.X), Y = (int)((m / s.X) % s.Y), Z = (int)(m / ((long long)s.X * s.Y));
    double su = 0, sv = 0, sw = 0, sz = 0;
    for (int kk = 1; kk <= rz; ++kk) {
      const int k = Z * rz + kk;
      const double dz = 1.0 / g.dzf_inv[k];
      for (int jj = 1; jj <= ry; ++jj)
        for (int ii = 1; ii <= rx; ++ii) {
          const int i = X * rx + ii, j = Y * ry + jj;
          const long long c = g.at(i, j, k);
          su += dz * 0.5 * ((double)u[c - 1] + (double)u[c]);
          sv += dz * 0.5 * ((double)v[c - g.X] + (double)v[c]);
          sw += dz * 0.5 * ((double)w[c - g.XY] + (double)w[c]);
        }
      sz += dz * rx * ry;
    }
    float *o = out + m * kOutC;
    o[0] = (float)(su / sz + u_crf);
    o[1] = (float)(sv / sz);
    o[2] = (float)(sw / sz);
    for (int c = 3; c < kOutC; ++c) o[c] = 0.f;
  }
}

// Interpolation of the generator's output (sample 0) onto the DNS grid:
// periodic linear in x and y between generator cell centres, linear in the
// physical z between centres and to zero at the walls.  zl / zh / zw give,
// per DNS centre (rows 0..nz+1) and face (rows nz+2..2nz+2), the lower and
// upper generator plane (-1 = wall) and the upper weight.
struct ZMap {
  const int *lo, *hi;
  const double *wt;
};

__device__ __forceinline__ float sample_xy(const float *out, const Shape &s, int z, double xg,
                                           double yg, int c) {
  if (z < 0) return 0.f;
  const double fx = floor(xg), fy = floor(yg);
  const int x0 = wrapi((int)fx, s.X), y0 = wrapi((int)fy, s.Y);
  const int x1 = wrapi(x0 + 1, s.X), y1 = wrapi(y0 + 1, s.Y);
  const double ax = xg - fx, ay = yg - fy;
  auto at = [&](int y, int x) { return (double)out[(((long long)z * s.Y + y) * s.X + x) * kOutC + c]; };
  return (float)((1 - ay) * ((1 - ax) * at(y0, x0) + ax * at(y0, x1)) +
                 ay * ((1 - ax) * at(y1, x0) + ax * at(y1, x1)));
}

template <class T>
__global__ void k_to_grid(Geo g, Shape s, const float *__restrict__ out, ZMap zm, double u_crf,
                          T *u, T *v, T *w) {
  const int i = blockIdx.x * 32 + threadIdx.x + 1;
  const int j = blockIdx.y * 8 + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  if (i > g.nx || j > g.ny) return;
  const long long c = g.at(i, j, k);
  // generator cell-centre coordinates of the DNS centre / faces
  const double sx = (double)s.X / g.nx, sy = (double)s.Y / g.ny;
  const double xc = (i - 0.5) * sx - 0.5, xf = i * sx - 0.5;
  const double yc = (j - 0.5) * sy - 0.5, yf = j * sy - 0.5;
  auto interp = [&](int row, double xg, double yg, int comp) {
    const double wt = zm.wt[row];
    return (float)((1.0 - wt) * sample_xy(out, s, zm.lo[row], xg, yg, comp) +
                   wt * sample_xy(out, s, zm.hi[row], xg, yg, comp));
  };
  u[c] = T(interp(k, xf, yc, 0) - u_crf);
  v[c] = T(interp(k, xc, yf, 1));
  w[c] = T(interp(g.nz + 2 + k, xc, yc, 2));
}

unsigned grid1d(long long n, int threads = 256) {
  long long b = (n + threads - 1) / threads;
  return (unsigned)std::max(1ll, std::min(b, 148ll * 32));
}

}  // namespace
}  // namespace gen
}  // namespace plc

// ============================================================================
// host side
// ============================================================================
using namespace plc;
using namespace plc::gen;

struct GenLayer {
  int ci, co, level;
  bool has_act;  // FiLM followed by LReLU (hidden layers)
  long long w_off, film_off;  // offsets into the FP32 parameters
  bf16 *wb = nullptr, *wt = nullptr;
  bf16 *in = nullptr;         // conv input (owned unless aliasing)
  bool own_in = false;
  float *pre = nullptr;       // conv output
  bf16 *act = nullptr;        // activation (BF16), hidden layers
  float *gam = nullptr, *bet = nullptr, *dgam = nullptr, *dbet = nullptr;
};

struct plc_gen {
  plc_gen_config cfg{};
  int device = 0;
  cudaStream_t stream = nullptr;
  Shape lv[kLevels];
  std::vector<GenLayer> layers;
  long long nparams = 0;
  float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  float *out = nullptr;                 // [B][Z][Y][X][16]
  float *bufA = nullptr, *bufB = nullptr;
  bf16 *dbf = nullptr;                  // BF16 operand of the gradients
  long long buf_elems = 0;
  float *r = nullptr;                   // [B]
  int *tidx = nullptr;                  // [B]
  float *coef = nullptr, *means = nullptr;
  double *loss = nullptr;               // [iters] (training) or [1]
  long long loss_cap = 0;
  double *stats = nullptr;              // [B][Z][NS]
  float *targets = nullptr, *target_re = nullptr;
  int ntargets = 0;
  float sc_mean = 1.f, sc_var = 1.f;
  long long adam_t = 0;
  float *coarse = nullptr;              // [Z][Y][X][16], plc_gen_stats_of
  int *derr = nullptr;                  // device error word of the tcgen05 kernels
  std::string err;
};

namespace {
std::string g_gen_err;

int gen_error(plc_gen *gn, int code, const std::string &msg) {
  if (gn) gn->err = msg;
  g_gen_err = msg;
  return code;
}
#define GEN_CUDA(gn, call)                                                              \
  do {                                                                                  \
    cudaError_t _e = (call);                                                            \
    if (_e != cudaSuccess)                                                              \
      return gen_error(gn, PLC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
  } while (0)

template <class P>
cudaError_t dalloc(P **ptr, long long n) {
  return cudaMalloc(reinterpret_cast<void **>(ptr), (size_t)std::max(1ll, n) * sizeof(P));
}

void gen_free(plc_gen *gn) {
  for (GenLayer &L : gn->layers) {
    cudaFree(L.wb);
    cudaFree(L.wt);
    if (L.own_in) cudaFree(L.in);
    cudaFree(L.pre);
    cudaFree(L.act);
    cudaFree(L.gam);
    cudaFree(L.bet);
    cudaFree(L.dgam);
    cudaFree(L.dbet);
  }
  for (void *q : {(void *)gn->p, (void *)gn->g, (void *)gn->m, (void *)gn->v, (void *)gn->out,
                  (void *)gn->bufA, (void *)gn->bufB, (void *)gn->dbf, (void *)gn->r,
                  (void *)gn->tidx, (void *)gn->coef, (void *)gn->means, (void *)gn->loss,
                  (void *)gn->stats, (void *)gn->targets, (void *)gn->target_re,
                  (void *)gn->coarse, (void *)gn->derr})
    cudaFree(q);
  if (gn->stream) cudaStreamDestroy(gn->stream);
}

// forward convolution and input gradient: the tcgen05 kernel, 128 voxels x
// all output channels per block
template <int N>
cudaError_t conv_tc(plc_gen *gn, Shape s, const bf16 *x, const bf16 *w, float *y, int ci) {
  const unsigned gx = (unsigned)((s.voxels() + kTcM - 1) / kTcM);
  k_conv3d_tc<N><<<gx, 128, tc_smem_bytes<N>(), gn->stream>>>(s, x, w, y, ci, gn->derr);
  return cudaGetLastError();
}

int conv(plc_gen *gn, Shape s, const bf16 *x, const bf16 *w, float *y, int ci, int co) {
  cudaError_t e;
  switch (co) {
    case 16: e = conv_tc<16>(gn, s, x, w, y, ci); break;
    case 32: e = conv_tc<32>(gn, s, x, w, y, ci); break;
    case 48: e = conv_tc<48>(gn, s, x, w, y, ci); break;
    case 64: e = conv_tc<64>(gn, s, x, w, y, ci); break;
    case 80: e = conv_tc<80>(gn, s, x, w, y, ci); break;
    case 96: e = conv_tc<96>(gn, s, x, w, y, ci); break;
    case 112: e = conv_tc<112>(gn, s, x, w, y, ci); break;
    case 128: e = conv_tc<128>(gn, s, x, w, y, ci); break;
    default: return gen_error(gn, PLC_ERR_ARG, "convolution channels must be a multiple of 16 <= 128");
  }
  GEN_CUDA(gn, e);
  return PLC_OK;
}

cudaError_t conv_configure() {
  cudaError_t e = cudaSuccess;
  auto one = [&](auto kern, size_t bytes) {
    if (e == cudaSuccess) e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  };
  one(k_conv3d_tc<16>, tc_smem_bytes<16>());
  one(k_conv3d_tc<32>, tc_smem_bytes<32>());
  one(k_conv3d_tc<48>, tc_smem_bytes<48>());
  one(k_conv3d_tc<64>, tc_smem_bytes<64>());
  one(k_conv3d_tc<80>, tc_smem_bytes<80>());
  one(k_conv3d_tc<96>, tc_smem_bytes<96>());
  one(k_conv3d_tc<112>, tc_smem_bytes<112>());
  one(k_conv3d_tc<128>, tc_smem_bytes<128>());
  one(k_conv3d_wgrad_tc<16>, tc_smem_bytes<16, kWgG, kWgNB>());
  one(k_conv3d_wgrad_tc<32>, tc_smem_bytes<32, kWgG, kWgNB>());
  one(k_conv3d_wgrad_tc<48>, tc_smem_bytes<48, kWgG, kWgNB>());
  one(k_conv3d_wgrad_tc<64>, tc_smem_bytes<64, kWgG, kWgNB>());
  one(k_conv3d_wgrad_tc<80>, tc_smem_bytes<80, kWgG, kWgNB>());
  one(k_conv3d_wgrad_tc<96>, tc_smem_bytes<96, kWgG, kWgNB>());
  one(k_conv3d_wgrad_tc<112>, tc_smem_bytes<112, kWgG, kWgNB>());
  one(k_conv3d_wgrad_tc<128>, tc_smem_bytes<128, kWgG, kWgNB>());
  return e;
}

// the device error word of the tcgen05 kernels (a bounded wait that gave up)
int check_device_error(plc_gen *gn) {
  int flag = 0;
  GEN_CUDA(gn, cudaMemcpyAsync(&flag, gn->derr, sizeof(int), cudaMemcpyDeviceToHost, gn->stream));
  GEN_CUDA(gn, cudaStreamSynchronize(gn->stream));
  if (flag) return gen_error(gn, PLC_ERR_CUDA, "a tensor-core convolution's bounded wait timed out");
  return PLC_OK;
}

template <int N>
cudaError_t wgrad_tc(plc_gen *gn, Shape s, const bf16 *dy, const bf16 *x, float *dw, int co) {
  const long long M = s.voxels();
  // about 8 blocks per SM over the 27 taps, at least 16 voxels each
  long long splits = std::max(1ll, std::min((long long)(148 * 8) / 27 + 1, (M + 15) / 16));
  long long chunk = (M + splits - 1) / splits;
  chunk = (chunk + 15) / 16 * 16;
  splits = (M + chunk - 1) / chunk;
  k_conv3d_wgrad_tc<N><<<dim3((unsigned)splits, 1, 27), 128, tc_smem_bytes<N, kWgG, kWgNB>(), gn->stream>>>(
      s, dy, x, dw, co, chunk, gn->derr);
  return cudaGetLastError();
}

// weight gradient on the tensor cores: M = co (zero-padded to 128), N = ci
int wgrad(plc_gen *gn, Shape s, const bf16 *dy, const bf16 *x, float *dw, int ci, int co) {
  if (co > 128 || co % 16) return gen_error(gn, PLC_ERR_ARG, "weight gradient: co must be a multiple of 16 <= 128");
  cudaError_t e;
  switch (ci) {
    case 16: e = wgrad_tc<16>(gn, s, dy, x, dw, co); break;
    case 32: e = wgrad_tc<32>(gn, s, dy, x, dw, co); break;
    case 48: e = wgrad_tc<48>(gn, s, dy, x, dw, co); break;
    case 64: e = wgrad_tc<64>(gn, s, dy, x, dw, co); break;
    case 80: e = wgrad_tc<80>(gn, s, dy, x, dw, co); break;
    case 96: e = wgrad_tc<96>(gn, s, dy, x, dw, co); break;
    case 112: e = wgrad_tc<112>(gn, s, dy, x, dw, co); break;
    case 128: e = wgrad_tc<128>(gn, s, dy, x, dw, co); break;
    default: return gen_error(gn, PLC_ERR_ARG, "weight gradient: ci must be a multiple of 16 <= 128");
  }
  GEN_CUDA(gn, e);
  return PLC_OK;
}

int refresh_weights(plc_gen *gn) {
  for (GenLayer &L : gn->layers) {
    k_weights_bf16<<<grid1d(27ll * L.ci * L.co), 256, 0, gn->stream>>>(gn->p + L.w_off, L.ci, L.co,
                                                                       L.wb, L.wt);
    GEN_CUDA(gn, cudaGetLastError());
  }
  return PLC_OK;
}

// forward pass for the batch r values already in gn->r
int forward(plc_gen *gn, unsigned long long latent_seed) {
  const int B = gn->cfg.batch;
  GenLayer &L0 = gn->layers[0];
  k_latent<<<grid1d(gn->lv[0].voxels() * L0.ci), 256, 0, gn->stream>>>(
      gn->lv[0].voxels() * L0.ci, latent_seed, L0.in);
  GEN_CUDA(gn, cudaGetLastError());
  for (size_t i = 0; i < gn->layers.size(); ++i) {
    GenLayer &L = gn->layers[i];
    const Shape s = gn->lv[L.level];
    if (i > 0 && L.own_in) {  // first conv of a finer level: upsample the previous activation
      const GenLayer &P = gn->layers[i - 1];
      k_upsample<<<grid1d(s.voxels() * L.ci / 8), 256, 0, gn->stream>>>(s, L.ci, P.act, L.in);
      GEN_CUDA(gn, cudaGetLastError());
    }
    if (int rc = conv(gn, s, L.in, L.wb, L.pre, L.ci, L.co)) return rc;
    k_film_tables<<<grid1d((long long)B * s.Z * L.co), 256, 0, gn->stream>>>(
        gn->p + L.film_off, s.Z, L.co, gn->r, B, L.gam, L.bet);
    GEN_CUDA(gn, cudaGetLastError());
    if (L.has_act)
      k_film_fwd<true><<<grid1d(s.voxels() * L.co), 256, 0, gn->stream>>>(s, L.co, L.pre, L.gam,
                                                                          L.bet, L.act, nullptr);
    else
      k_film_fwd<false><<<grid1d(s.voxels() * L.co), 256, 0, gn->stream>>>(
          s, L.co, L.pre, L.gam, L.bet, nullptr, gn->out);
    GEN_CUDA(gn, cudaGetLastError());
  }
  return PLC_OK;
}

// loss (added to *loss_slot) and parameter gradients (added to gn->g) of the
// last forward pass against the targets gn->tidx
int backward(plc_gen *gn, double *loss_slot) {
  const Shape so = gn->lv[kLevels - 1];
  const int B = gn->cfg.batch;
  k_stats<<<(unsigned)(so.B * so.Z), 256, 0, gn->stream>>>(so, kOutC, gn->out, gn->tidx,
                                                           gn->targets, gn->sc_mean, gn->sc_var,
                                                           gn->coef, gn->means, loss_slot, nullptr);
  GEN_CUDA(gn, cudaGetLastError());
  k_stats_grad<<<grid1d(so.voxels()), 256, 0, gn->stream>>>(so, kOutC, gn->out, gn->coef,
                                                             gn->means, gn->bufA);
  GEN_CUDA(gn, cudaGetLastError());
  float *dact = gn->bufA, *dnext = gn->bufB;
  for (int i = (int)gn->layers.size() - 1; i >= 0; --i) {
    GenLayer &L = gn->layers[i];
    const Shape s = gn->lv[L.level];
    if (L.has_act)
      k_film_bwd<true><<<(unsigned)(s.B * s.Z), 256, 0, gn->stream>>>(
          s, L.co, dact, L.pre, L.gam, L.bet, gn->dbf, L.dgam, L.dbet);
    else
      k_film_bwd<false><<<(unsigned)(s.B * s.Z), 256, 0, gn->stream>>>(
          s, L.co, dact, L.pre, L.gam, L.bet, gn->dbf, L.dgam, L.dbet);
    GEN_CUDA(gn, cudaGetLastError());
    k_film_param_grad<<<grid1d((long long)s.Z * L.co), 256, 0, gn->stream>>>(
        s.Z, L.co, B, gn->r, L.dgam, L.dbet, gn->g + L.film_off);
    GEN_CUDA(gn, cudaGetLastError());
    if (int rc = wgrad(gn, s, gn->dbf, L.in, gn->g + L.w_off, L.ci, L.co)) return rc;
    if (i == 0) break;  // no gradient for the latent
    if (int rc = conv(gn, s, gn->dbf, L.wt, dnext, L.co, L.ci)) return rc;
    if (L.own_in) {  // input was the upsampled activation of the coarser level
      const Shape sc = gn->lv[L.level - 1];
      k_upsample_bwd<<<grid1d(sc.voxels() * L.ci), 256, 0, gn->stream>>>(sc, L.ci, dnext, dact);
      GEN_CUDA(gn, cudaGetLastError());
    } else {
      std::swap(dact, dnext);
    }
  }
  return PLC_OK;
}

int upload_r(plc_gen *gn, const double *re_tau) {
  std::vector<float> r(gn->cfg.batch);
  for (int b = 0; b < gn->cfg.batch; ++b) r[b] = (float)((re_tau[b] - 260.0) / 140.0);
  GEN_CUDA(gn, cudaMemcpyAsync(gn->r, r.data(), r.size() * sizeof(float), cudaMemcpyHostToDevice,
                               gn->stream));
  GEN_CUDA(gn, cudaStreamSynchronize(gn->stream));
  return PLC_OK;
}

int adam_step(plc_gen *gn, float lr) {
  const float b1 = 0.9f, b2 = 0.999f;
  ++gn->adam_t;
  const float bc1 = 1.f - std::pow(b1, (float)gn->adam_t), bc2 = 1.f - std::pow(b2, (float)gn->adam_t);
  k_adam<<<grid1d(gn->nparams), 256, 0, gn->stream>>>(gn->nparams, gn->p, gn->g, gn->m, gn->v, lr,
                                                      b1, b2, 1e-8f, bc1, bc2);
  GEN_CUDA(gn, cudaGetLastError());
  return refresh_weights(gn);
}

// z maps of plc_gen_propose: generator plane centres in the physical z of
// the DNS mesh (generator plane K = DNS cells K*rz+1 .. (K+1)*rz)
void z_map(const plc_ctx *c, int Zg, std::vector<int> &lo, std::vector<int> &hi,
           std::vector<double> &wt) {
  const int nz = c->nz, rz = nz / Zg;
  std::vector<double> zf(nz + 1, 0.0);
  for (int k = 1; k <= nz; ++k) zf[k] = zf[k - 1] + c->h_dzf_global[k];
  std::vector<double> zg(Zg);
  for (int K = 0; K < Zg; ++K) zg[K] = 0.5 * (zf[K * rz] + zf[(K + 1) * rz]);
  const double lz = zf[nz];
  auto one = [&](double z, int &l, int &h, double &w) {
    if (z <= zg[0]) {  // between the bottom wall (0) and the first centre
      l = -1;
      h = 0;
      w = z / zg[0];
    } else if (z >= zg[Zg - 1]) {
      l = Zg - 1;
      h = -1;
      w = (z - zg[Zg - 1]) / (lz - zg[Zg - 1]);
    } else {
      int K = 0;
      while (K + 1 < Zg && zg[K + 1] < z) ++K;
      l = K;
      h = K + 1;
      w = (z - zg[K]) / (zg[K + 1] - zg[K]);
    }
  };
  lo.assign(2 * nz + 3, -1);
  hi.assign(2 * nz + 3, -1);
  wt.assign(2 * nz + 3, 0.0);
  for (int k = 1; k <= nz; ++k) one(0.5 * (zf[k - 1] + zf[k]), lo[k], hi[k], wt[k]);
  for (int k = 0; k <= nz; ++k) one(zf[k], lo[nz + 2 + k], hi[nz + 2 + k], wt[nz + 2 + k]);
}

}  // namespace

extern "C" {

const char *plc_gen_last_error(const plc_gen *gn) { return gn ? gn->err.c_str() : g_gen_err.c_str(); }

int plc_gen_config_default(plc_gen_config *cfg) {
  if (!cfg) return gen_error(nullptr, PLC_ERR_ARG, "null config");
  cfg->nx = 64;
  cfg->ny = 48;
  cfg->nz = 64;
  cfg->channels[0] = 128;
  cfg->channels[1] = 96;
  cfg->channels[2] = 64;
  cfg->channels[3] = 32;
  cfg->latent_channels = 16;
  cfg->batch = 4;
  cfg->seed = 1;
  return PLC_OK;
}

int plc_gen_create(const plc_gen_config *cfg, int device, plc_gen **out) {
  if (!cfg || !out) return gen_error(nullptr, PLC_ERR_ARG, "null argument");
  *out = nullptr;
  const plc_gen_config &C = *cfg;
  if (C.nx % 8 || C.ny % 8 || C.nz % 8 || C.nx < 8 || C.ny < 8 || C.nz < 8)
    return gen_error(nullptr, PLC_ERR_SIZE, "generator grid must be divisible by 8");
  if (C.batch < 1 || C.latent_channels < 16 || C.latent_channels % 16)
    return gen_error(nullptr, PLC_ERR_ARG, "batch >= 1 and latent channels a multiple of 16");
  for (int l = 0; l < kLevels; ++l)
    if (C.channels[l] < 16 || C.channels[l] > 128 || C.channels[l] % 16)
      return gen_error(nullptr, PLC_ERR_ARG, "channels must be multiples of 16 in [16, 128]");
  plc_gen *gn = new plc_gen;
  gn->cfg = C;
  gn->device = device;
  auto fail = [&](int rc) {
    const std::string msg = gn->err;
    gen_free(gn);
    delete gn;
    return gen_error(nullptr, rc, msg);
  };
  cudaError_t e;
  if ((e = cudaSetDevice(device)) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&gn->stream, cudaStreamNonBlocking)) != cudaSuccess) {
    gn->err = std::string("CUDA: ") + cudaGetErrorString(e);
    return fail(PLC_ERR_CUDA);
  }
  for (int l = 0; l < kLevels; ++l) {
    const int sh = kLevels - 1 - l;
    gn->lv[l] = Shape{C.batch, C.nz >> sh, C.ny >> sh, C.nx >> sh};
  }
  if (gn->lv[kLevels - 1].voxels() * 128 >= (1ll << 31)) {  // 32-bit voxel and element indices
    gn->err = "generator grid x batch too large";
    return fail(PLC_ERR_SIZE);
  }
  // layers and parameter layout
  long long off = 0;
  auto add = [&](int ci, int co, int level, bool act) {
    GenLayer L;
    L.ci = ci;
    L.co = co;
    L.level = level;
    L.has_act = act;
    L.w_off = off;
    off += 27ll * ci * co;
    gn->layers.push_back(L);
  };
  add(C.latent_channels, C.channels[0], 0, true);
  add(C.channels[0], C.channels[0], 0, true);
  for (int l = 1; l < kLevels; ++l) {
    add(C.channels[l - 1], C.channels[l], l, true);
    add(C.channels[l], C.channels[l], l, true);
  }
  add(C.channels[kLevels - 1], kOutC, kLevels - 1, false);
  for (GenLayer &L : gn->layers) {
    L.film_off = off;
    off += 4ll * gn->lv[L.level].Z * L.co;
  }
  gn->nparams = off;
  // device memory
  const Shape top = gn->lv[kLevels - 1];
  long long maxe = 0;
  for (size_t i = 0; i < gn->layers.size(); ++i) {
    GenLayer &L = gn->layers[i];
    const Shape s = gn->lv[L.level];
    maxe = std::max(maxe, s.voxels() * std::max(L.ci, L.co));
    const long long tz = (long long)C.batch * s.Z * L.co;
    if ((e = dalloc(&L.wb, 27ll * L.ci * L.co)) || (e = dalloc(&L.wt, 27ll * L.ci * L.co)) ||
        (e = dalloc(&L.pre, s.voxels() * L.co)) || (e = dalloc(&L.gam, tz)) ||
        (e = dalloc(&L.bet, tz)) || (e = dalloc(&L.dgam, tz)) || (e = dalloc(&L.dbet, tz)))
      break;
    if (L.has_act && (e = dalloc(&L.act, s.voxels() * L.co))) break;
    const bool first_of_level = i == 0 || gn->layers[i - 1].level != L.level;
    if (first_of_level) {
      L.own_in = true;
      if ((e = dalloc(&L.in, s.voxels() * L.ci))) break;
    } else {
      L.in = gn->layers[i - 1].act;
    }
  }
  if (e != cudaSuccess) {
    gn->err = std::string("generator allocation: ") + cudaGetErrorString(e);
    return fail(PLC_ERR_NOMEM);
  }
  gn->buf_elems = std::max(maxe, top.voxels() * kOutC);
  const long long bzn = (long long)C.batch * top.Z;
  if ((e = dalloc(&gn->p, gn->nparams)) || (e = dalloc(&gn->g, gn->nparams)) ||
      (e = dalloc(&gn->m, gn->nparams)) || (e = dalloc(&gn->v, gn->nparams)) ||
      (e = dalloc(&gn->out, top.voxels() * kOutC)) || (e = dalloc(&gn->bufA, gn->buf_elems)) ||
      (e = dalloc(&gn->bufB, gn->buf_elems)) || (e = dalloc(&gn->dbf, gn->buf_elems)) ||
      (e = dalloc(&gn->r, C.batch)) || (e = dalloc(&gn->tidx, C.batch)) ||
      (e = dalloc(&gn->coef, bzn * PLC_GEN_NSTAT)) || (e = dalloc(&gn->means, bzn * 3)) ||
      (e = dalloc(&gn->stats, bzn * PLC_GEN_NSTAT)) ||
      (e = dalloc(&gn->coarse, (long long)top.Z * top.Y * top.X * kOutC)) ||
      (e = dalloc(&gn->derr, 1)) || (e = cudaMemset(gn->derr, 0, sizeof(int))) ||
      (e = conv_configure())) {
    gn->err = std::string("generator allocation: ") + cudaGetErrorString(e);
    return fail(PLC_ERR_NOMEM);
  }
  // initial weights: He-normal (gain 2 for LReLU layers, 1 for the output,
  // whose channels beyond u, v, w stay zero); FiLM parameters zero
  std::vector<float> h(gn->nparams, 0.f);
  std::mt19937_64 rng(C.seed);
  for (const GenLayer &L : gn->layers) {
    const double sd = std::sqrt((L.has_act ? 2.0 : 1.0) / (27.0 * L.ci));
    std::normal_distribution<double> nd(0.0, sd);
    for (int tap = 0; tap < 27; ++tap)
      for (int o = 0; o < L.co; ++o)
        for (int i = 0; i < L.ci; ++i) {
          const double x = nd(rng);
          if (L.has_act || o < 3) h[L.w_off + ((long long)tap * L.co + o) * L.ci + i] = (float)x;
        }
  }
  if ((e = cudaMemcpy(gn->p, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice)) ||
      (e = cudaMemset(gn->m, 0, gn->nparams * sizeof(float))) ||
      (e = cudaMemset(gn->v, 0, gn->nparams * sizeof(float)))) {
    gn->err = std::string("generator init: ") + cudaGetErrorString(e);
    return fail(PLC_ERR_CUDA);
  }
  if (int rc = refresh_weights(gn)) return fail(rc);
  if ((e = cudaStreamSynchronize(gn->stream)) != cudaSuccess) {
    gn->err = std::string("generator init: ") + cudaGetErrorString(e);
    return fail(PLC_ERR_CUDA);
  }
  *out = gn;
  return PLC_OK;
}

int plc_gen_destroy(plc_gen *gn) {
  if (!gn) return PLC_OK;
  if (gn->stream) cudaStreamSynchronize(gn->stream);
  gen_free(gn);
  delete gn;
  return PLC_OK;
}

int plc_gen_num_params(const plc_gen *gn, long long *n) {
  if (!gn || !n) return gen_error(nullptr, PLC_ERR_ARG, "null argument");
  *n = gn->nparams;
  return PLC_OK;
}

int plc_gen_get_params(plc_gen *gn, float *h) {
  if (!gn || !h) return gen_error(gn, PLC_ERR_ARG, "null argument");
  GEN_CUDA(gn, cudaMemcpyAsync(h, gn->p, gn->nparams * sizeof(float), cudaMemcpyDeviceToHost,
                               gn->stream));
  GEN_CUDA(gn, cudaStreamSynchronize(gn->stream));
  return PLC_OK;
}

int plc_gen_set_params(plc_gen *gn, const float *h) {
  if (!gn || !h) return gen_error(gn, PLC_ERR_ARG, "null argument");
  GEN_CUDA(gn, cudaMemcpyAsync(gn->p, h, gn->nparams * sizeof(float), cudaMemcpyHostToDevice,
                               gn->stream));
  if (int rc = refresh_weights(gn)) return rc;
  GEN_CUDA(gn, cudaStreamSynchronize(gn->stream));
  return PLC_OK;
}

int plc_gen_set_targets(plc_gen *gn, int n, const double *re_tau, const double *stats) {
  if (!gn || n < 1 || !re_tau || !stats) return gen_error(gn, PLC_ERR_ARG, "bad argument");
  const int Z = gn->lv[kLevels - 1].Z, NS = PLC_GEN_NSTAT;
  std::vector<float> t((size_t)n * Z * NS), re(n);
  double s_mean = 0, s_var = 0;
  for (int q = 0; q < n; ++q) {
    re[q] = (float)re_tau[q];
    for (int z = 0; z < Z; ++z)
      for (int s = 0; s < NS; ++s) {
        const double x = stats[((size_t)q * Z + z) * NS + s];
        t[((size_t)q * Z + z) * NS + s] = (float)x;
        if (s == 0) s_mean += x * x;
        if (s == 3) s_var += x * x;
      }
  }
  // scales: the RMS of the mean streamwise velocity and of its variance
  gn->sc_mean = (float)std::max(1e-6, std::sqrt(s_mean / (n * Z)));
  gn->sc_var = (float)std::max(1e-9, std::sqrt(s_var / (n * Z)));
  cudaFree(gn->targets);
  cudaFree(gn->target_re);
  gn->targets = nullptr;
  gn->target_re = nullptr;
  GEN_CUDA(gn, dalloc(&gn->targets, (long long)t.size()));
  GEN_CUDA(gn, dalloc(&gn->target_re, n));
  GEN_CUDA(gn, cudaMemcpy(gn->targets, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice));
  GEN_CUDA(gn, cudaMemcpy(gn->target_re, re.data(), re.size() * sizeof(float), cudaMemcpyHostToDevice));
  gn->ntargets = n;
  return PLC_OK;
}

int plc_gen_latent(plc_gen *gn, unsigned long long seed, float *h) {
  if (!gn || !h) return gen_error(gn, PLC_ERR_ARG, "null argument");
  const GenLayer &L0 = gn->layers[0];
  const long long n = gn->lv[0].voxels() * L0.ci;
  k_latent<<<grid1d(n), 256, 0, gn->stream>>>(n, seed, L0.in);
  GEN_CUDA(gn, cudaGetLastError());
  std::vector<bf16> tmp(n);
  GEN_CUDA(gn, cudaMemcpyAsync(tmp.data(), L0.in, n * sizeof(bf16), cudaMemcpyDeviceToHost, gn->stream));
  GEN_CUDA(gn, cudaStreamSynchronize(gn->stream));
  for (long long e = 0; e < n; ++e) h[e] = __bfloat162float(tmp[e]);
  return PLC_OK;
}

int plc_gen_forward(plc_gen *gn, const double *re_tau, unsigned long long latent_seed, float *h_out) {
  if (!gn || !re_tau) return gen_error(gn, PLC_ERR_ARG, "null argument");
  if (int rc = upload_r(gn, re_tau)) return rc;
  if (int rc = forward(gn, latent_seed)) return rc;
  if (int rc = check_device_error(gn)) return rc;
  if (h_out) {
    const Shape s = gn->lv[kLevels - 1];
    std::vector<float> o(s.voxels() * kOutC);
    GEN_CUDA(gn, cudaMemcpyAsync(o.data(), gn->out, o.size() * sizeof(float), cudaMemcpyDeviceToHost,
                                 gn->stream));
    GEN_CUDA(gn, cudaStreamSynchronize(gn->stream));
    for (long long m = 0; m < s.voxels(); ++m)
      for (int c = 0; c < 3; ++c) h_out[m * 3 + c] = o[m * kOutC + c];
  }
  GEN_CUDA(gn, cudaStreamSynchronize(gn->stream));
  return PLC_OK;
}

int plc_gen_output_stats(plc_gen *gn, double *h_stats) {
  if (!gn || !h_stats) return gen_error(gn, PLC_ERR_ARG, "null argument");
  const Shape s = gn->lv[kLevels - 1];
  k_stats<<<(unsigned)(s.B * s.Z), 256, 0, gn->stream>>>(s, kOutC, gn->out, nullptr, nullptr, 1.f,
                                                         1.f, nullptr, nullptr, nullptr, gn->stats);
  GEN_CUDA(gn, cudaGetLastError());
  GEN_CUDA(gn, cudaMemcpyAsync(h_stats, gn->stats, (size_t)s.B * s.Z * PLC_GEN_NSTAT * sizeof(double),
                               cudaMemcpyDeviceToHost, gn->stream));
  GEN_CUDA(gn, cudaStreamSynchronize(gn->stream));
  return PLC_OK;
}

int plc_gen_loss_grad(plc_gen *gn, const int *target_idx, const double *re_tau,
                      unsigned long long latent_seed, double *loss, float *h_grads) {
  if (!gn || !target_idx || !re_tau || !loss) return gen_error(gn, PLC_ERR_ARG, "null argument");
  if (!gn->targets) return gen_error(gn, PLC_ERR_STATE, "no training targets set");
  for (int b = 0; b < gn->cfg.batch; ++b)
    if (target_idx[b] < 0 || target_idx[b] >= gn->ntargets)
      return gen_error(gn, PLC_ERR_ARG, "target index out of range");
  GEN_CUDA(gn, cudaMemcpyAsync(gn->tidx, target_idx, gn->cfg.batch * sizeof(int),
                               cudaMemcpyHostToDevice, gn->stream));
  if (int rc = upload_r(gn, re_tau)) return rc;
  if (gn->loss_cap < 1) {
    cudaFree(gn->loss);
    GEN_CUDA(gn, dalloc(&gn->loss, 1));
    gn->loss_cap = 1;
  }
  GEN_CUDA(gn, cudaMemsetAsync(gn->loss, 0, sizeof(double), gn->stream));
  GEN_CUDA(gn, cudaMemsetAsync(gn->g, 0, gn->nparams * sizeof(float), gn->stream));
  if (int rc = forward(gn, latent_seed)) return rc;
  if (int rc = backward(gn, gn->loss)) return rc;
  if (int rc = check_device_error(gn)) return rc;
  GEN_CUDA(gn, cudaMemcpyAsync(loss, gn->loss, sizeof(double), cudaMemcpyDeviceToHost, gn->stream));
  if (h_grads)
    GEN_CUDA(gn, cudaMemcpyAsync(h_grads, gn->g, gn->nparams * sizeof(float), cudaMemcpyDeviceToHost,
                                 gn->stream));
  GEN_CUDA(gn, cudaStreamSynchronize(gn->stream));
  return PLC_OK;
}

int plc_gen_train(plc_gen *gn, int iters, double lr, unsigned long long seed, double *h_loss) {
  if (!gn || iters < 1) return gen_error(gn, PLC_ERR_ARG, "bad argument");
  if (!gn->targets) return gen_error(gn, PLC_ERR_STATE, "no training targets set");
  if (gn->loss_cap < iters) {
    cudaFree(gn->loss);
    gn->loss = nullptr;
    GEN_CUDA(gn, dalloc(&gn->loss, iters));
    gn->loss_cap = iters;
  }
  GEN_CUDA(gn, cudaMemsetAsync(gn->loss, 0, iters * sizeof(double), gn->stream));
  const int warm = std::min(100, iters / 10 + 1);
  for (int it = 0; it < iters; ++it) {
    // linear warm-up, then cosine decay to 5 % of lr
    const double f = it < warm ? (it + 1.0) / warm
                               : 0.05 + 0.95 * 0.5 * (1.0 + std::cos(M_PI * (it - warm) / (iters - warm)));
    k_pick_targets<<<1, 32, 0, gn->stream>>>(seed * 1000003ull + it, gn->cfg.batch, gn->ntargets,
                                             gn->target_re, gn->tidx, gn->r);
    GEN_CUDA(gn, cudaGetLastError());
    GEN_CUDA(gn, cudaMemsetAsync(gn->g, 0, gn->nparams * sizeof(float), gn->stream));
    if (int rc = forward(gn, seed * 7919ull + 0x5bd1e995ull * (unsigned long long)it)) return rc;
    if (int rc = backward(gn, gn->loss + it)) return rc;
    if (int rc = adam_step(gn, (float)(lr * f))) return rc;
  }
  if (int rc = check_device_error(gn)) return rc;
  if (h_loss)
    GEN_CUDA(gn, cudaMemcpyAsync(h_loss, gn->loss, iters * sizeof(double), cudaMemcpyDeviceToHost,
                                 gn->stream));
  GEN_CUDA(gn, cudaStreamSynchronize(gn->stream));
  return PLC_OK;
}

int plc_gen_adam_step(plc_gen *gn, double lr) {
  if (!gn) return gen_error(nullptr, PLC_ERR_ARG, "null generator");
  if (int rc = adam_step(gn, (float)lr)) return rc;
  GEN_CUDA(gn, cudaStreamSynchronize(gn->stream));
  return PLC_OK;
}

int plc_gen_stats_of(plc_gen *gn, plc_ctx *c, double *h_stats) {
  if (!gn || !c || !h_stats) return gen_error(gn, PLC_ERR_ARG, "null argument");
  const Shape top = gn->lv[kLevels - 1];
  if (c->nx % top.X || c->ny % top.Y || c->nz % top.Z)
    return gen_error(gn, PLC_ERR_SIZE, "the context's grid must be a multiple of the generator's");
  const Shape s1{1, top.Z, top.Y, top.X};
  const int rx = c->nx / top.X, ry = c->ny / top.Y, rz = c->nz / top.Z;
  GEN_CUDA(gn, cudaStreamSynchronize(c->stream));
  const long long n = (long long)top.Z * top.Y * top.X;
  if (c->mixed)
    k_coarsen<float><<<grid1d(n), 256, 0, gn->stream>>>(c->geo(), c->f_field[PLC_U], c->f_field[PLC_V],
                                                        c->f_field[PLC_W], c->prm.u_crf, s1, rx, ry,
                                                        rz, gn->coarse);
  else
    k_coarsen<double><<<grid1d(n), 256, 0, gn->stream>>>(c->geo(), c->d_field[PLC_U],
                                                         c->d_field[PLC_V], c->d_field[PLC_W],
                                                         c->prm.u_crf, s1, rx, ry, rz, gn->coarse);
  GEN_CUDA(gn, cudaGetLastError());
  k_stats<<<(unsigned)top.Z, 256, 0, gn->stream>>>(s1, kOutC, gn->coarse, nullptr, nullptr, 1.f, 1.f,
                                                   nullptr, nullptr, nullptr, gn->stats);
  GEN_CUDA(gn, cudaGetLastError());
  GEN_CUDA(gn, cudaMemcpyAsync(h_stats, gn->stats, (size_t)top.Z * PLC_GEN_NSTAT * sizeof(double),
                               cudaMemcpyDeviceToHost, gn->stream));
  GEN_CUDA(gn, cudaStreamSynchronize(gn->stream));
  return PLC_OK;
}

int plc_gen_propose(plc_gen *gn, plc_ctx *c, double re_tau, unsigned long long latent_seed) {
  if (!gn || !c) return gen_error(gn, PLC_ERR_ARG, "null argument");
  const Shape top = gn->lv[kLevels - 1];
  if (c->nz % top.Z) return gen_error(gn, PLC_ERR_SIZE, "the context's nz must be a multiple of the generator's");
  std::vector<double> re(gn->cfg.batch, re_tau);
  if (int rc = upload_r(gn, re.data())) return rc;
  if (int rc = forward(gn, latent_seed)) return rc;
  if (int rc = check_device_error(gn)) return rc;
  std::vector<int> lo, hi;
  std::vector<double> wt;
  z_map(c, top.Z, lo, hi, wt);
  int *dlo = nullptr, *dhi = nullptr;
  double *dwt = nullptr;
  GEN_CUDA(gn, dalloc(&dlo, (long long)lo.size()));
  cudaError_t e = dalloc(&dhi, (long long)hi.size());
  if (e == cudaSuccess) e = dalloc(&dwt, (long long)wt.size());
  if (e == cudaSuccess) e = cudaMemcpy(dlo, lo.data(), lo.size() * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dhi, hi.data(), hi.size() * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dwt, wt.data(), wt.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaStreamSynchronize(gn->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  const ZMap zm{dlo, dhi, dwt};
  const Shape s1{1, top.Z, top.Y, top.X};  // sample 0 of the batch
  const dim3 grid((c->nx + 31) / 32, (c->ny + 7) / 8, c->nz);
  if (e == cudaSuccess) {
    if (c->mixed)
      k_to_grid<float><<<grid, dim3(32, 8), 0, c->stream>>>(c->geo(), s1, gn->out, zm, c->prm.u_crf,
                                                            c->f_field[PLC_U], c->f_field[PLC_V],
                                                            c->f_field[PLC_W]);
    else
      k_to_grid<double><<<grid, dim3(32, 8), 0, c->stream>>>(c->geo(), s1, gn->out, zm, c->prm.u_crf,
                                                             c->d_field[PLC_U], c->d_field[PLC_V],
                                                             c->d_field[PLC_W]);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(dlo);
  cudaFree(dhi);
  cudaFree(dwt);
  if (e != cudaSuccess) return gen_error(gn, PLC_ERR_CUDA, std::string("plc_gen_propose: ") + cudaGetErrorString(e));
  // the solver's own projection makes the field divergence-free
  if (int rc = plc_project(c)) return gen_error(gn, rc, std::string("plc_project: ") + plc_last_error(c));
  return PLC_OK;
}

}  // extern "C"
