// Diagnostics of the channel on the device: the running statistics of
// mod_statistics (src/mod_statistics.cc:30-106) and the monitor quantities of
// mod_monitor (src/mod_monitor.cc:57-205) -- bulk velocities, probe point,
// wall skin friction, region extracts -- plus plane-averaged profiles of the
// statistics.  The reference keeps its statistics in host-side loops over
// USM memory; here the sums live in device FP64 arrays and one kernel adds a
// sample.  Compiled without FMA contraction: each sum adds the value or the
// product exactly as the reference writes it, so the sums are bit-identical to
// the CPU restatement.  Kernels are templates on the field type (FP64, or FP32
// in the mixed form, whose sums are still FP64).

#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
#include <string>

#include "plc_device.cuh"
#include "plc_internal.h"

namespace plc {
namespace {

constexpr int BX = 32, BY = 8;

struct StatSums {
  double *s[kStatVars];  // nullptr: not sampled
};

// calcStat's accumulation of one sample, mod_statistics.cc:40-104.  The sums
// are nx*ny*nz, x fastest, without halos (Array3DH0).
template <class T>
__global__ void __launch_bounds__(BX *BY) k_calc_stat(Geo g, double u_crf, const T *__restrict__ u,
                                                      const T *__restrict__ v,
                                                      const T *__restrict__ w,
                                                      const T *__restrict__ p, StatSums sums) {
  const int i = blockIdx.x * BX + threadIdx.x + 1;
  const int j = blockIdx.y * BY + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  if (i > g.nx || j > g.ny) return;
  const long long c = g.at(i, j, k);
  const long long o = (i - 1) + (long long)g.nx * ((j - 1) + (long long)g.ny * (k - 1));
  // cell-centred velocities (:44-46)
  const double uc = (double(u[c - 1]) + double(u[c])) * 0.5 + u_crf;
  const double vc = (double(v[c - g.X]) + double(v[c])) * 0.5;
  const double wc = (double(w[c - g.XY]) + double(w[c])) * 0.5;
  const double pc = double(p[c]);
  const double val[kStatVars] = {uc, vc, wc, uc * uc, vc * vc, wc * wc,
                                 uc * vc, uc * wc, vc * wc, pc, pc * pc};
#pragma unroll
  for (int q = 0; q < kStatVars; ++q)
    if (sums.s[q]) sums.s[q][o] += val[q];
}

// Plane means of every sampled sum divided by the samples: out[q*nz + k-1],
// one block per (k, q); a fixed-order FP64 sum (deterministic).
__global__ void __launch_bounds__(256) k_stat_profiles(int nx, int ny, int nz, StatSums sums,
                                                       double inv_samples, double *out) {
  __shared__ double red[8];
  const int k = blockIdx.x, q = blockIdx.y;
  const double *s = sums.s[q];
  if (!s) {
    if (threadIdx.x == 0) out[q * nz + k] = 0.0;
    return;
  }
  const long long plane = (long long)nx * ny;
  double acc = 0.0;
  for (long long t = threadIdx.x; t < plane; t += blockDim.x) acc += s[(long long)k * plane + t];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w2 = 0; w2 < 8; ++w2) tot += red[w2];
    out[q * nz + k] = tot / plane * inv_samples;
  }
}

// Double-double accumulation (Knuth TwoSum): each addition's rounding error is
// carried in the low word, so the rounded total is nearly independent of the
// order of the terms (the low words' own sums still round, which can move the
// total by an ulp on ill-conditioned data).
__device__ __forceinline__ void dd_acc(double &hi, double &lo, double x) {
  const double s = hi + x;
  const double bb = s - hi;
  lo += (hi - (s - bb)) + (x - bb);
  hi = s;
}
__device__ __forceinline__ void dd_merge(double &hi, double &lo, double bhi, double blo) {
  const double s = hi + bhi;
  const double bb = s - hi;
  const double e = (hi - (s - bb)) + (bhi - bb);
  hi = s;
  lo = (lo + blo) + e;
}

// calcAndWriteSkf's plane sum (mod_monitor.cc:100-104): sum over (i,j) of
// re_inv*(vel(i,j,k_wall) + vel_crf)/dz, double-double, one block.
template <class T>
__global__ void __launch_bounds__(1024) k_wall_tau(Geo g, int k_wall, double dz, double vel_crf,
                                                   const T *__restrict__ vel, double *out) {
  __shared__ double rh[32], rl[32];
  const long long plane = (long long)g.nx * g.ny;
  double hi = 0.0, lo = 0.0;
  for (long long t = threadIdx.x; t < plane; t += blockDim.x) {
    const int j = (int)(t / g.nx) + 1, i = (int)(t % g.nx) + 1;
    dd_acc(hi, lo, g.re_inv * (double(vel[g.at(i, j, k_wall)]) + vel_crf) / dz);
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double bh = __shfl_down_sync(0xffffffffu, hi, o);
    const double bl = __shfl_down_sync(0xffffffffu, lo, o);
    dd_merge(hi, lo, bh, bl);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    rh[wid] = hi;
    rl[wid] = lo;
  }
  __syncthreads();
  if (wid == 0) {
    hi = lane < (int)(blockDim.x >> 5) ? rh[lane] : 0.0;
    lo = lane < (int)(blockDim.x >> 5) ? rl[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      const double bh = __shfl_down_sync(0xffffffffu, hi, o);
      const double bl = __shfl_down_sync(0xffffffffu, lo, o);
      dd_merge(hi, lo, bh, bl);
    }
    if (lane == 0) *out = (hi + lo) / g.nx / g.ny;
  }
}

// extractRegion (mod_monitor.cc:117-158): the box of size sz from the 1-based
// interior index st, staggered -> centred along dir (0 none, 1 x, 2 y, 3 z),
// plus `shift` (u_crf for u, mod_monitor.cc:170-177); out x fastest.
template <class T>
__global__ void k_extract_region(Geo g, const T *__restrict__ var, int dir, int3 st, int3 sz,
                                 double shift, double *__restrict__ out) {
  const long long n = (long long)sz.x * sz.y * sz.z;
  const long long d = dir == 1 ? 1 : (dir == 2 ? g.X : (dir == 3 ? g.XY : 0));
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % sz.x), j = (int)((t / sz.x) % sz.y), k = (int)(t / ((long long)sz.x * sz.y));
    const long long c = g.at(st.x + i, st.y + j, st.z + k);
    const double x = dir == 0 ? double(var[c]) : 0.5 * (double(var[c - d]) + double(var[c]));
    out[t] = shift == 0.0 ? x : x + shift;
  }
}

// Plane means of u + u_crf (instantaneous mean profile), one block per plane.
template <class T>
__global__ void __launch_bounds__(256) k_plane_mean(Geo g, const T *__restrict__ u, double u_crf,
                                                    double *__restrict__ out) {
  __shared__ double red[8];
  const int k = blockIdx.x + 1;
  double s = 0.0;
  for (int t = threadIdx.x; t < g.nx * g.ny; t += blockDim.x) {
    const int j = t / g.nx + 1, i = t % g.nx + 1;
    s += double(u[g.at(i, j, k)]);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
    out[k - 1] = tot / ((double)g.nx * g.ny) + u_crf;
  }
}

StatSums stat_sums(const plc_ctx *c) {
  StatSums s;
  for (int q = 0; q < kStatVars; ++q) s.s[q] = c->d_stat[q];
  return s;
}

template <class T>
const T *field_of(const plc_ctx *c, int f);
template <>
const double *field_of<double>(const plc_ctx *c, int f) {
  return c->d_field[f];
}
template <>
const float *field_of<float>(const plc_ctx *c, int f) {
  return c->f_field[f];
}

template <class T>
cudaError_t calc_stat_t(const plc_ctx *c) {
  dim3 grid((c->nx + BX - 1) / BX, (c->ny + BY - 1) / BY, c->nz);
  k_calc_stat<T><<<grid, dim3(BX, BY), 0, c->stream>>>(
      c->geo(), c->prm.u_crf, field_of<T>(c, PLC_U), field_of<T>(c, PLC_V), field_of<T>(c, PLC_W),
      field_of<T>(c, PLC_P), stat_sums(c));
  return cudaGetLastError();
}

template <class T>
cudaError_t wall_tau_t(const plc_ctx *c, int k_wall, double dz, double *d_out) {
  k_wall_tau<T><<<1, 1024, 0, c->stream>>>(c->geo(), k_wall, dz, c->prm.u_crf,
                                            field_of<T>(c, PLC_U), d_out);
  return cudaGetLastError();
}

template <class T>
cudaError_t extract_t(const plc_ctx *c, int field, int dir, int3 st, int3 sz, double shift,
                      double *d_out) {
  const long long n = (long long)sz.x * sz.y * sz.z;
  long long nb = (n + 255) / 256;
  if (nb > 16ll * c->num_sms) nb = 16ll * c->num_sms;
  k_extract_region<T><<<(unsigned)(nb < 1 ? 1 : nb), 256, 0, c->stream>>>(
      c->geo(), field_of<T>(c, field), dir, st, sz, shift, d_out);
  return cudaGetLastError();
}

#define PLC_CHECK_CTX(c) \
  if (!(c)) return plc::set_error(nullptr, PLC_ERR_ARG, "null context")
#define PLC_NEED_STAT(c) \
  if (!(c)->stat_ready) return set_error(c, PLC_ERR_STATE, "statistics not initialised (plc_stat_init)")

}  // namespace
}  // namespace plc

using namespace plc;

extern "C" {

// ---- mod_statistics -------------------------------------------------------
int plc_stat_init(plc_ctx *c) {
  PLC_CHECK_CTX(c);
  plc_stat_free(c);
  const size_t n = (size_t)c->nx * c->ny * c->nz;
  // allocStat (mod_statistics.cc:7-13): the enabled sums, zeroed
  for (int q = 0; q < kStatVars; ++q)
    if (c->prm.stat_which_var[q]) {
      if (cudaMalloc(&c->d_stat[q], n * sizeof(double)) != cudaSuccess) {
        plc_stat_free(c);
        return set_error(c, PLC_ERR_NOMEM, "cudaMalloc statistics");
      }
      PLC_CUDA(c, cudaMemsetAsync(c->d_stat[q], 0, n * sizeof(double), c->stream));
    }
  // initStat (mod_statistics.cc:23-28)
  c->stat_nts = c->prm.nt_init_stat + 1;
  c->stat_nte = c->prm.nt_init_stat;
  c->stat_nspl = 0;
  c->stat_ready = true;
  PLC_CUDA(c, cudaStreamSynchronize(c->stream));
  return PLC_OK;
}

int plc_stat_free(plc_ctx *c) {
  PLC_CHECK_CTX(c);
  for (auto &s : c->d_stat) {
    cudaFree(s);
    s = nullptr;
  }
  c->stat_ready = false;
  return PLC_OK;
}

int plc_calc_stat(plc_ctx *c, int nt) {
  PLC_CHECK_CTX(c);
  PLC_NEED_STAT(c);
  const int si = c->prm.sample_interval;
  if (si <= 0) return set_error(c, PLC_ERR_ARG, "sample_interval must be positive");
  // the sampling rule of calcStat (mod_statistics.cc:33-35)
  if ((nt - c->prm.nt_init_stat) % si != 0) return PLC_OK;
  c->stat_nte += si;
  c->stat_nspl += 1;
  PLC_CUDA(c, c->mixed ? calc_stat_t<float>(c) : calc_stat_t<double>(c));
  return PLC_OK;
}

int plc_stat_info(const plc_ctx *c, int *nts, int *nte, int *nspl) {
  if (!c) return set_error(nullptr, PLC_ERR_ARG, "null context");
  if (nts) *nts = c->stat_nts;
  if (nte) *nte = c->stat_nte;
  if (nspl) *nspl = c->stat_nspl;
  return PLC_OK;
}

int plc_stat_download(plc_ctx *c, int which, double *h_dst) {
  PLC_CHECK_CTX(c);
  PLC_NEED_STAT(c);
  if (which < 0 || which >= kStatVars || !c->d_stat[which] || !h_dst)
    return set_error(c, PLC_ERR_ARG, "statistic not sampled, or null destination");
  const size_t n = (size_t)c->nx * c->ny * c->nz;
  PLC_CUDA(c, cudaMemcpyAsync(h_dst, c->d_stat[which], n * sizeof(double), cudaMemcpyDeviceToHost,
                              c->stream));
  PLC_CUDA(c, cudaStreamSynchronize(c->stream));
  return PLC_OK;
}

int plc_stat_upload(plc_ctx *c, int which, const double *h_src, int nts, int nte, int nspl) {
  PLC_CHECK_CTX(c);
  PLC_NEED_STAT(c);
  if (which < 0 || which >= kStatVars || !c->d_stat[which] || !h_src)
    return set_error(c, PLC_ERR_ARG, "statistic not sampled, or null source");
  const size_t n = (size_t)c->nx * c->ny * c->nz;
  PLC_CUDA(c, cudaMemcpyAsync(c->d_stat[which], h_src, n * sizeof(double), cudaMemcpyHostToDevice,
                              c->stream));
  PLC_CUDA(c, cudaStreamSynchronize(c->stream));
  // inputStatData restores the sample counters with the sums (mod_dataIO.cc:232-252)
  c->stat_nts = nts;
  c->stat_nte = nte;
  c->stat_nspl = nspl;
  return PLC_OK;
}

int plc_stat_profiles(plc_ctx *c, double *h_prof) {
  PLC_CHECK_CTX(c);
  PLC_NEED_STAT(c);
  if (!h_prof) return set_error(c, PLC_ERR_ARG, "null destination");
  const size_t n = (size_t)kStatVars * c->nz;
  double *d = nullptr;
  PLC_CUDA(c, cudaMallocAsync(&d, n * sizeof(double), c->stream));
  k_stat_profiles<<<dim3(c->nz, kStatVars), 256, 0, c->stream>>>(
      c->nx, c->ny, c->nz, stat_sums(c), c->stat_nspl > 0 ? 1.0 / c->stat_nspl : 0.0, d);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h_prof, d, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  const cudaError_t ef = cudaFreeAsync(d, c->stream);
  if (e == cudaSuccess) e = ef;
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_status(c, e, "plc_stat_profiles");
  return PLC_OK;
}

int plc_mean_profile(plc_ctx *c, double *h_prof) {
  PLC_CHECK_CTX(c);
  if (!h_prof) return set_error(c, PLC_ERR_ARG, "null destination");
  double *d = nullptr;
  PLC_CUDA(c, cudaMallocAsync(&d, c->nz * sizeof(double), c->stream));
  if (c->mixed)
    k_plane_mean<float><<<c->nz, 256, 0, c->stream>>>(c->geo(), c->f_field[PLC_U], c->prm.u_crf, d);
  else
    k_plane_mean<double><<<c->nz, 256, 0, c->stream>>>(c->geo(), c->d_field[PLC_U], c->prm.u_crf, d);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h_prof, d, c->nz * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  const cudaError_t ef = cudaFreeAsync(d, c->stream);
  if (e == cudaSuccess) e = ef;
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_status(c, e, "plc_mean_profile");
  return PLC_OK;
}

// ---- mod_monitor ----------------------------------------------------------
int plc_monitor_skf(plc_ctx *c, int wall, double *u_tau, double *cf) {
  PLC_CHECK_CTX(c);
  if (wall != 0 && wall != 1) return set_error(c, PLC_ERR_ARG, "wall must be 0 (bottom) or 1 (top)");
  // outputMonitor (mod_monitor.cc:318-323): k_wall = 1 or nz, dz = dzf(k_wall)/2
  const int k_wall = wall == 0 ? 1 : c->nz;
  const double dz = 0.5 * c->h_dzf[k_wall];
  double *d = c->d_partials;  // scratch word
  PLC_CUDA(c, c->mixed ? wall_tau_t<float>(c, k_wall, dz, d) : wall_tau_t<double>(c, k_wall, dz, d));
  PLC_CUDA(c, cudaMemcpyAsync(c->h_scal, d, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  PLC_CUDA(c, cudaStreamSynchronize(c->stream));
  const double tau_w = c->h_scal[0];
  // mod_monitor.cc:107-109
  if (u_tau) *u_tau = std::sqrt(tau_w);
  if (cf) *cf = tau_w / (0.5 * c->prm.u_ref * c->prm.u_ref);
  return PLC_OK;
}

int plc_monitor_probe(plc_ctx *c, int ig, int jg, int kg, double *out4) {
  PLC_CHECK_CTX(c);
  if (!out4 || ig < 1 || ig > c->nx || jg < 1 || jg > c->ny || kg < 1 || kg > c->nz)
    return set_error(c, PLC_ERR_ARG, "probe point outside the interior, or null output");
  // extractAndWriteProbePoint (mod_monitor.cc:77-91): u + u_crf, v, w, p
  const long long idx = c->geo().at(ig, jg, kg);
  const int fields[4] = {PLC_U, PLC_V, PLC_W, PLC_P};
  for (int q = 0; q < 4; ++q) {
    if (c->mixed) {
      float x = 0.f;
      PLC_CUDA(c, cudaMemcpyAsync(&x, c->f_field[fields[q]] + idx, sizeof(float),
                                  cudaMemcpyDeviceToHost, c->stream));
      PLC_CUDA(c, cudaStreamSynchronize(c->stream));
      out4[q] = x;
    } else {
      PLC_CUDA(c, cudaMemcpyAsync(out4 + q, c->d_field[fields[q]] + idx, sizeof(double),
                                  cudaMemcpyDeviceToHost, c->stream));
    }
  }
  PLC_CUDA(c, cudaStreamSynchronize(c->stream));
  out4[0] += c->prm.u_crf;
  return PLC_OK;
}

int plc_monitor_forcing(plc_ctx *c, double *vel_mean3) {
  PLC_CHECK_CTX(c);
  if (!vel_mean3) return set_error(c, PLC_ERR_ARG, "null output");
  // calcAndWriteForcing (mod_monitor.cc:57-75): Mean of each forced component
  // (u shifted by u_crf); 0 for the others
  for (int d = 0; d < 3; ++d) {
    vel_mean3[d] = 0.0;
    if (!c->prm.is_forced[d]) continue;
    if (c->mixed)
      PLC_CUDA(c, launch_mean(c, 0, c->nx, c->ny, c->f_field[d], c->stream));
    else
      PLC_CUDA(c, launch_mean(c, 0, c->nx, c->ny, c->d_field[d], c->stream));
    PLC_CUDA(c, cudaMemcpyAsync(c->h_scal, reinterpret_cast<char *>(c->d_sc) + offsetof(StepConst, mean),
                                sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PLC_CUDA(c, cudaStreamSynchronize(c->stream));
    vel_mean3[d] = c->h_scal[0];
  }
  vel_mean3[0] += c->prm.u_crf;
  return PLC_OK;
}

int plc_extract_region(plc_ctx *c, const int *region_ijk, int field, double *h_dst) {
  PLC_CHECK_CTX(c);
  if (!region_ijk || !h_dst) return set_error(c, PLC_ERR_ARG, "null argument");
  if (field != PLC_U && field != PLC_V && field != PLC_W && field != PLC_P)
    return set_error(c, PLC_ERR_ARG, "region extracts are of u, v, w or p");
  // initMonitor clips the region to the domain (mod_monitor.cc:273-279)
  int r[6] = {region_ijk[0], region_ijk[1], region_ijk[2], region_ijk[3], region_ijk[4],
              region_ijk[5]};
  r[0] = r[0] < 1 ? 1 : r[0];
  r[1] = r[1] > c->nx ? c->nx : r[1];
  r[2] = r[2] < 1 ? 1 : r[2];
  r[3] = r[3] > c->ny ? c->ny : r[3];
  r[4] = r[4] < 1 ? 1 : r[4];
  r[5] = r[5] > c->nz ? c->nz : r[5];
  if (r[1] < r[0] || r[3] < r[2] || r[5] < r[4]) return set_error(c, PLC_ERR_ARG, "empty region");
  const int3 st = make_int3(r[0], r[2], r[4]);
  const int3 sz = make_int3(r[1] - r[0] + 1, r[3] - r[2] + 1, r[5] - r[4] + 1);
  // extractAndWriteRegion (mod_monitor.cc:160-205): u, v, w centred along
  // their own direction, u shifted by u_crf; p as stored
  const int dir = field == PLC_U ? 1 : (field == PLC_V ? 2 : (field == PLC_W ? 3 : 0));
  const double shift = field == PLC_U ? c->prm.u_crf : 0.0;
  const size_t n = (size_t)sz.x * sz.y * sz.z;
  double *d = nullptr;
  PLC_CUDA(c, cudaMallocAsync(&d, n * sizeof(double), c->stream));
  cudaError_t e = c->mixed ? extract_t<float>(c, field, dir, st, sz, shift, d)
                           : extract_t<double>(c, field, dir, st, sz, shift, d);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h_dst, d, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  const cudaError_t ef = cudaFreeAsync(d, c->stream);
  if (e == cudaSuccess) e = ef;
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_status(c, e, "plc_extract_region");
  return PLC_OK;
}

}  // extern "C"
