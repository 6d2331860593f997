// CPU oracle for the PowerLLEL_Channel DNS time step -- TEST INFRASTRUCTURE.
//
// Plain FP64 restatement of the reference's hot path; see oracle.h for the
// layout conventions and the parity status (pinned to the reference's own
// modules compiled for the CPU, except for oneMKL's DFT).  Compiled with
// -ffp-contract=off so that every expression is evaluated exactly in the
// order written, which follows the reference expression by expression.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.

#include "oracle.h"

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using cplx = std::complex<double>;

struct Idx {
  int X, Y;  // halo'd x and y lengths
  long long operator()(int i, int j, int k) const {
    return (long long)i + (long long)X * ((long long)j + (long long)Y * k);
  }
};

inline Idx make_idx(const orc_grid *g) { return Idx{g->nx + 2, g->ny + 2}; }

// Double-double accumulation: (hi, lo) += x with Knuth's error-free TwoSum.
inline void two_sum_acc(double &hi, double &lo, double x) {
  const double s = hi + x;
  const double bb = s - hi;
  const double e = (hi - (s - bb)) + (x - bb);
  hi = s;
  lo += e;
}

// ---------------------------------------------------------------------------
// Mixed-radix complex DFT (recursive decimation in time by the smallest prime
// factor).  Independent of the GPU implementation, which uses a Stockham
// formulation with a two-for-one real packing.
// ---------------------------------------------------------------------------
struct FftPlan {
  int n;
  std::vector<cplx> w;  // w[t] = exp(-2 pi i t / n)
};

int smallest_factor(int n) {
  for (int r = 2; r * r <= n; ++r)
    if (n % r == 0) return r;
  return n;
}

std::mutex g_plan_mu;
std::map<int, std::shared_ptr<FftPlan>> g_plans;

std::shared_ptr<FftPlan> get_plan(int n) {
  std::lock_guard<std::mutex> lk(g_plan_mu);
  auto it = g_plans.find(n);
  if (it != g_plans.end()) return it->second;
  auto p = std::make_shared<FftPlan>();
  p->n = n;
  p->w.resize(n);
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int t = 0; t < n; ++t) {
    long double ang = -two_pi * (long double)t / (long double)n;
    p->w[t] = cplx((double)cosl(ang), (double)sinl(ang));
  }
  g_plans[n] = p;
  return p;
}

// X[0..n) = sum_t x[t*s] * W^(t*k), W = exp(sign*2*pi*i/n), sign = -1 for
// forward and +1 (conj twiddles) for inverse.  tmp holds at least n entries.
void dft_rec(const cplx *x, long s, cplx *X, int n, const FftPlan &P,
             bool inverse, cplx *tmp) {
  if (n == 1) {
    X[0] = x[0];
    return;
  }
  const int N = P.n;
  const int r = smallest_factor(n);
  const int m = n / r;
  for (int q = 0; q < r; ++q) dft_rec(x + q * s, s * r, X + q * m, m, P, inverse, tmp);
  const int scale = N / n;
  for (int k = 0; k < m; ++k) {
    for (int p = 0; p < r; ++p) {
      const int kk = k + p * m;
      cplx acc(0.0, 0.0);
      for (int q = 0; q < r; ++q) {
        const long e = ((long)q * kk) % n;
        cplx tw = P.w[e * scale];
        if (inverse) tw = std::conj(tw);
        acc += tw * X[q * m + k];
      }
      tmp[kk] = acc;
    }
  }
  for (int t = 0; t < n; ++t) X[t] = tmp[t];
}

void cdft(int n, const cplx *x, cplx *X, bool inverse, std::vector<cplx> &tmp) {
  auto P = get_plan(n);
  if ((int)tmp.size() < n) tmp.resize(n);
  dft_rec(x, 1, X, n, *P, inverse, tmp.data());
}

void rfft_packed_impl(int n, const double *in, double *out,
                      std::vector<cplx> &a, std::vector<cplx> &b,
                      std::vector<cplx> &tmp) {
  a.resize(n);
  b.resize(n);
  for (int t = 0; t < n; ++t) a[t] = cplx(in[t], 0.0);
  cdft(n, a.data(), b.data(), false, tmp);
  // packed real layout: mod_fft.cc:79-86 (idx_m = num for i == 1)
  out[0] = b[0].real();
  out[1] = b[n / 2].real();
  for (int m = 1; m < n / 2; ++m) {
    out[2 * m] = b[m].real();
    out[2 * m + 1] = b[m].imag();
  }
}

void irfft_packed_impl(int n, const double *in, double *out,
                       std::vector<cplx> &a, std::vector<cplx> &b,
                       std::vector<cplx> &tmp) {
  a.resize(n);
  b.resize(n);
  // mod_fft.cc:94-104: the CCE buffer is zeroed, then Re parts of k=0 and
  // k=n/2 and the (Re, Im) pairs of 1..n/2-1 are scattered into it.
  a[0] = cplx(in[0], 0.0);
  a[n / 2] = cplx(in[1], 0.0);
  for (int m = 1; m < n / 2; ++m) {
    a[m] = cplx(in[2 * m], in[2 * m + 1]);
    a[n - m] = std::conj(a[m]);
  }
  cdft(n, a.data(), b.data(), true, tmp);
  for (int t = 0; t < n; ++t) out[t] = b[t].real();
}

// ---------------------------------------------------------------------------
// Halo rules (mod_updateBound.cc).  At p_row = p_col = 1 the y halo comes from
// the MPI self-exchange (mod_type.hh:219-289 + mod_updateBound.cc:11-30) over
// all x and z indices, then x is made periodic over all y and z indices
// (:32-73), then the z planes are overwritten by the wall rules (:75-180).
// ---------------------------------------------------------------------------
void halo_y_periodic(const orc_grid *g, double *var) {
  const Idx I = make_idx(g);
  const int nx = g->nx, ny = g->ny, nz = g->nz;
#pragma omp parallel for
  for (int k = 0; k <= nz + 1; ++k)
    for (int i = 0; i <= nx + 1; ++i) {
      double south = var[I(i, ny, k)];  // gathered row j = ny
      double north = var[I(i, 1, k)];   // gathered row j = 1
      var[I(i, 0, k)] = south;
      var[I(i, ny + 1, k)] = north;
    }
}

void halo_x_periodic(const orc_grid *g, double *var) {
  const Idx I = make_idx(g);
  const int nx = g->nx, ny = g->ny, nz = g->nz;
#pragma omp parallel for
  for (int k = 0; k <= nz + 1; ++k)
    for (int j = 0; j <= ny + 1; ++j) var[I(0, j, k)] = var[I(nx, j, k)];
#pragma omp parallel for
  for (int k = 0; k <= nz + 1; ++k)
    for (int j = 0; j <= ny + 1; ++j) var[I(nx + 1, j, k)] = var[I(1, j, k)];
}

// imposeNoSlipBC, mod_updateBound.cc:75-144
void noslip_z(const orc_grid *g, double *var, bool centered, double bcvalue) {
  const Idx I = make_idx(g);
  const int nx = g->nx, ny = g->ny, n = g->nz;
  for (int j = 0; j <= ny + 1; ++j)
    for (int i = 0; i <= nx + 1; ++i) {
      if (centered)
        var[I(i, j, 0)] = 2.0 * bcvalue - var[I(i, j, 1)];
      else
        var[I(i, j, 0)] = bcvalue;
    }
  for (int j = 0; j <= ny + 1; ++j)
    for (int i = 0; i <= nx + 1; ++i) {
      if (centered) {
        var[I(i, j, n + 1)] = 2.0 * bcvalue - var[I(i, j, n)];
      } else {
        var[I(i, j, n)] = bcvalue;
        var[I(i, j, n + 1)] = bcvalue;
      }
    }
}

// imposeZeroGradBC, mod_updateBound.cc:146-180
void zerograd_z(const orc_grid *g, double *var) {
  const Idx I = make_idx(g);
  const int nx = g->nx, ny = g->ny, n = g->nz;
  for (int j = 0; j <= ny + 1; ++j)
    for (int i = 0; i <= nx + 1; ++i) var[I(i, j, 0)] = var[I(i, j, 1)];
  for (int j = 0; j <= ny + 1; ++j)
    for (int i = 0; i <= nx + 1; ++i) var[I(i, j, n + 1)] = var[I(i, j, n)];
}

}  // namespace

struct orc_poisson {
  int nx, ny, nz;
  double normfactor;
  std::vector<double> var;  // nx*ny*nz spectral work array
  std::vector<double> a, c;  // nz
  std::vector<double> b;     // nx*ny*nz pre-factored diagonal
};

extern "C" {

// ---------------------------------------------------------------------------
// mod_statistics::calcStat, src/mod_statistics.cc:30-106: one sample.  The
// cell-centred velocities are (q(i-1) + q(i)) * 0.5 (+ u_crf for u) (:44-46);
// each sum adds the value or the product of two of them (:50-99).
// ---------------------------------------------------------------------------
void orc_calc_stat_sample(const orc_grid *g, double u_crf, const double *u, const double *v,
                          const double *w, const double *p, double *const *sums) {
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  const long X = nx + 2, XY = X * (ny + 2);
#pragma omp parallel for
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        const long c = i + X * j + XY * k;
        const long o = (i - 1) + (long)nx * ((j - 1) + (long)ny * (k - 1));
        const double uc = (u[c - 1] + u[c]) * 0.5 + u_crf;
        const double vc = (v[c - X] + v[c]) * 0.5;
        const double wc = (w[c - XY] + w[c]) * 0.5;
        const double pc = p[c];
        const double val[11] = {uc, vc, wc, uc * uc, vc * vc, wc * wc,
                                uc * vc, uc * wc, vc * wc, pc, pc * pc};
        for (int q = 0; q < 11; ++q)
          if (sums[q]) sums[q][o] += val[q];
      }
}

// ---------------------------------------------------------------------------
// mod_monitor::calcAndWriteSkf, src/mod_monitor.cc:93-113: the plane mean of
// re_inv * (vel + vel_crf) / dz at k_wall.  The reference's sum runs in
// (j, i) order with an MPI_Reduce over ranks; here it is double-double, so the
// rounded total does not depend on the order.
// ---------------------------------------------------------------------------
double orc_wall_tau(const orc_grid *g, int k_wall, double dz, const double *vel,
                    double vel_crf) {
  const int nx = g->nx, ny = g->ny;
  const long X = nx + 2, XY = X * (ny + 2);
  double hi = 0.0, lo = 0.0;
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i)
      two_sum_acc(hi, lo, g->re_inv * (vel[i + X * j + XY * k_wall] + vel_crf) / dz);
  return (hi + lo) / nx / ny;
}

// ---------------------------------------------------------------------------
// mod_monitor::extractRegion, src/mod_monitor.cc:117-158.
// ---------------------------------------------------------------------------
void orc_extract_region(const orc_grid *g, const double *var, int offset_dir,
                        const int *reg_st, const int *reg_sz, double *out) {
  const long X = g->nx + 2, XY = X * (g->ny + 2);
  const int is = reg_st[0] - 1, js = reg_st[1] - 1, ks = reg_st[2] - 1;
  const long d = offset_dir == 1 ? 1 : (offset_dir == 2 ? X : (offset_dir == 3 ? XY : 0));
  for (int k = 1; k <= reg_sz[2]; ++k)
    for (int j = 1; j <= reg_sz[1]; ++j)
      for (int i = 1; i <= reg_sz[0]; ++i) {
        const long c = (i + is) + X * (j + js) + XY * (k + ks);
        const long o = (i - 1) + (long)reg_sz[0] * ((j - 1) + (long)reg_sz[1] * (k - 1));
        out[o] = offset_dir == 0 ? var[c] : 0.5 * (var[c - d] + var[c]);
      }
}

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int orc_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// ---------------------------------------------------------------------------
// Mesh: mod_mesh.cc:95-125 (initMeshByFunc) and :13-76 (initMesh)
// ---------------------------------------------------------------------------
void orc_mesh_by_func(int mesh_type, int stretch_func, double stretch_ratio,
                      int nz, double lz, double *dzf_global) {
  const double pi = M_PI;
  if (stretch_ratio == 0.0 || mesh_type == 0) {
    for (int k = 0; k <= nz + 1; ++k) dzf_global[k] = lz / nz;
    return;
  }
  std::vector<double> zf(nz + 2, 0.0);
  zf[0] = 0.0;
  if (stretch_func == 0) {
    for (int k = 1; k <= nz; ++k) {
      double z0 = k / (1.0 * nz);
      zf[k] = 0.5 * (1.0 + tanh((z0 - 0.5) * stretch_ratio) /
                               tanh(stretch_ratio / 2.0));
    }
  } else {
    for (int k = 1; k <= nz; ++k) {
      double z0 = k / (1.0 * nz);
      zf[k] = 0.5 * (1.0 + sin((z0 - 0.5) * stretch_ratio * pi) /
                               sin(stretch_ratio * pi / 2.0));
    }
  }
  for (int k = 1; k <= nz; ++k) dzf_global[k] = lz * (zf[k] - zf[k - 1]);
  dzf_global[0] = dzf_global[1];
  dzf_global[nz + 1] = dzf_global[nz];
}

void orc_mesh_derived(int nz, double lz, const double *dzf_global, double *dzf,
                      double *dzf_inv, double *dzc, double *dzc_inv,
                      double *dzflzi, double *zc_global) {
  for (int k = 0; k <= nz + 1; ++k) {
    dzc[k] = 0.0;
    dzc_inv[k] = 0.0;
  }
  if (zc_global) {
    zc_global[0] = -0.5 * dzf_global[0];
    for (int k = 1; k <= nz + 1; ++k)
      zc_global[k] = zc_global[k - 1] + 0.5 * (dzf_global[k - 1] + dzf_global[k]);
  }
  for (int k = 0; k <= nz + 1; ++k) {
    dzf[k] = dzf_global[k];
    dzf_inv[k] = 1.0 / dzf[k];
  }
  for (int k = 0; k <= nz; ++k) {
    dzc[k] = 0.5 * (dzf[k] + dzf[k + 1]);
    dzc_inv[k] = 1.0 / dzc[k];
  }
  for (int k = 0; k <= nz + 1; ++k) dzflzi[k] = dzf[k] / lz;
}

// ---------------------------------------------------------------------------
// mod_calcVel.cc
// ---------------------------------------------------------------------------
void orc_transform2crf(const orc_grid *g, double vel_crf, double *vel,
                       double *vel_force) {
  // mod_calcVel.cc:13-25 (the SYCL range covers the interior only)
  if (vel_crf != 0) {
    const Idx I = make_idx(g);
#pragma omp parallel for
    for (int k = 1; k <= g->nz; ++k)
      for (int j = 1; j <= g->ny; ++j)
        for (int i = 1; i <= g->nx; ++i) vel[I(i, j, k)] -= vel_crf;
    *vel_force -= vel_crf;
  }
}

namespace {
// F(q) of mod_calcVel.cc:61-125 evaluated at (i,j,k); returns the three
// components of (visc - conv).
struct Rhs3 {
  double u, v, w;
};

inline Rhs3 momentum_rhs(const orc_grid *g, const Idx &I, double u_crf,
                         const double *_u, const double *_v, const double *_w,
                         int i, int j, int k) {
  const double _dx_inv = g->dx_inv, _dy_inv = g->dy_inv, _re_inv = g->re_inv;
  const double *_dzf = g->dzf, *_dzf_inv = g->dzf_inv, *_dzc_inv = g->dzc_inv;
#define U(a, b, c) _u[I(a, b, c)]
#define V(a, b, c) _v[I(a, b, c)]
#define W(a, b, c) _w[I(a, b, c)]
  double uw, ue, us, un, ub, ut;
  double ww, we, ws, wn, wb, wt;
  double vw, ve, vs, vn, vb, vt;
  double dqw, dqe, dqs, dqn, dqb, dqt;
  double conv, visc;
  Rhs3 r;
  // u component, mod_calcVel.cc:61-81
  ue = (U(i, j, k) + U(i + 1, j, k));
  uw = (U(i - 1, j, k) + U(i, j, k));
  un = (U(i, j, k) + U(i, j + 1, k));
  us = (U(i, j - 1, k) + U(i, j, k));
  ut = (U(i, j, k) * _dzf[k + 1] + U(i, j, k + 1) * _dzf[k]) * _dzc_inv[k];
  ub = (U(i, j, k) * _dzf[k - 1] + U(i, j, k - 1) * _dzf[k]) * _dzc_inv[k - 1];
  vn = (V(i, j, k) + V(i + 1, j, k));
  vs = (V(i, j - 1, k) + V(i + 1, j - 1, k));
  wt = (W(i, j, k) + W(i + 1, j, k));
  wb = (W(i, j, k - 1) + W(i + 1, j, k - 1));
  dqe = (U(i + 1, j, k) - U(i, j, k)) * _dx_inv;
  dqw = (U(i, j, k) - U(i - 1, j, k)) * _dx_inv;
  dqn = (U(i, j + 1, k) - U(i, j, k)) * _dy_inv;
  dqs = (U(i, j, k) - U(i, j - 1, k)) * _dy_inv;
  dqt = (U(i, j, k + 1) - U(i, j, k)) * _dzc_inv[k];
  dqb = (U(i, j, k) - U(i, j, k - 1)) * _dzc_inv[k - 1];
  conv = 0.25 * ((ue * ue - uw * uw) * _dx_inv + (un * vn - us * vs) * _dy_inv +
                 (ut * wt - ub * wb) * _dzf_inv[k]);
  conv = conv + 0.5 * u_crf * (ue - uw) * _dx_inv;
  visc = ((dqe - dqw) * _dx_inv + (dqn - dqs) * _dy_inv +
          (dqt - dqb) * _dzf_inv[k]) * _re_inv;
  r.u = visc - conv;
  // v component, mod_calcVel.cc:83-103
  ve = (V(i, j, k) + V(i + 1, j, k));
  vw = (V(i - 1, j, k) + V(i, j, k));
  vn = (V(i, j, k) + V(i, j + 1, k));
  vs = (V(i, j - 1, k) + V(i, j, k));
  vt = (V(i, j, k) * _dzf[k + 1] + V(i, j, k + 1) * _dzf[k]) * _dzc_inv[k];
  vb = (V(i, j, k) * _dzf[k - 1] + V(i, j, k - 1) * _dzf[k]) * _dzc_inv[k - 1];
  ue = (U(i, j, k) + U(i, j + 1, k));
  uw = (U(i - 1, j, k) + U(i - 1, j + 1, k));
  wt = (W(i, j, k) + W(i, j + 1, k));
  wb = (W(i, j, k - 1) + W(i, j + 1, k - 1));
  dqe = (V(i + 1, j, k) - V(i, j, k)) * _dx_inv;
  dqw = (V(i, j, k) - V(i - 1, j, k)) * _dx_inv;
  dqn = (V(i, j + 1, k) - V(i, j, k)) * _dy_inv;
  dqs = (V(i, j, k) - V(i, j - 1, k)) * _dy_inv;
  dqt = (V(i, j, k + 1) - V(i, j, k)) * _dzc_inv[k];
  dqb = (V(i, j, k) - V(i, j, k - 1)) * _dzc_inv[k - 1];
  conv = 0.25 * ((ue * ve - uw * vw) * _dx_inv + (vn * vn - vs * vs) * _dy_inv +
                 (wt * vt - wb * vb) * _dzf_inv[k]);
  conv = conv + 0.5 * u_crf * (ve - vw) * _dx_inv;
  visc = ((dqe - dqw) * _dx_inv + (dqn - dqs) * _dy_inv +
          (dqt - dqb) * _dzf_inv[k]) * _re_inv;
  r.v = visc - conv;
  // w component, mod_calcVel.cc:105-125
  we = (W(i, j, k) + W(i + 1, j, k));
  ww = (W(i - 1, j, k) + W(i, j, k));
  wn = (W(i, j, k) + W(i, j + 1, k));
  ws = (W(i, j - 1, k) + W(i, j, k));
  wt = (W(i, j, k) + W(i, j, k + 1));
  wb = (W(i, j, k) + W(i, j, k - 1));
  ue = (U(i, j, k) * _dzf[k + 1] + U(i, j, k + 1) * _dzf[k]) * _dzc_inv[k];
  uw = (U(i - 1, j, k) * _dzf[k + 1] + U(i - 1, j, k + 1) * _dzf[k]) * _dzc_inv[k];
  vn = (V(i, j, k) * _dzf[k + 1] + V(i, j, k + 1) * _dzf[k]) * _dzc_inv[k];
  vs = (V(i, j - 1, k) * _dzf[k + 1] + V(i, j - 1, k + 1) * _dzf[k]) * _dzc_inv[k];
  dqe = (W(i + 1, j, k) - W(i, j, k)) * _dx_inv;
  dqw = (W(i, j, k) - W(i - 1, j, k)) * _dx_inv;
  dqn = (W(i, j + 1, k) - W(i, j, k)) * _dy_inv;
  dqs = (W(i, j, k) - W(i, j - 1, k)) * _dy_inv;
  dqt = (W(i, j, k + 1) - W(i, j, k)) * _dzf_inv[k + 1];
  dqb = (W(i, j, k) - W(i, j, k - 1)) * _dzf_inv[k];
  conv = 0.25 * ((ue * we - uw * ww) * _dx_inv + (vn * wn - vs * ws) * _dy_inv +
                 (wt * wt - wb * wb) * _dzc_inv[k]);
  conv = conv + 0.5 * u_crf * (we - ww) * _dx_inv;
  visc = ((dqe - dqw) * _dx_inv + (dqn - dqs) * _dy_inv +
          (dqt - dqb) * _dzc_inv[k]) * _re_inv;
  r.w = visc - conv;
#undef U
#undef V
#undef W
  return r;
}
}  // namespace

void orc_time_int_vel_rk1(const orc_grid *g, double u_crf, const double *u,
                          const double *v, const double *w, double *u1,
                          double *v1, double *w1) {
  // mod_calcVel.cc:27-129: u1 = u + dt*(visc - conv) on the interior
  const Idx I = make_idx(g);
  const double _dt = g->dt;
#pragma omp parallel for
  for (int k = 1; k <= g->nz; ++k)
    for (int j = 1; j <= g->ny; ++j)
      for (int i = 1; i <= g->nx; ++i) {
        Rhs3 r = momentum_rhs(g, I, u_crf, u, v, w, i, j, k);
        long long c = I(i, j, k);
        u1[c] = u[c] + _dt * r.u;
        v1[c] = v[c] + _dt * r.v;
        w1[c] = w[c] + _dt * r.w;
      }
}

void orc_time_int_vel_rk2(const orc_grid *g, double u_crf, double *u,
                          double *v, double *w, const double *u1,
                          const double *v1, const double *w1) {
  // mod_calcVel.cc:140-242: u = (u1 + dt*(visc - conv)(u1) + u) * 0.5
  const Idx I = make_idx(g);
  const double _dt = g->dt;
#pragma omp parallel for
  for (int k = 1; k <= g->nz; ++k)
    for (int j = 1; j <= g->ny; ++j)
      for (int i = 1; i <= g->nx; ++i) {
        Rhs3 r = momentum_rhs(g, I, u_crf, u1, v1, w1, i, j, k);
        long long c = I(i, j, k);
        u[c] = (u1[c] + _dt * r.u + u[c]) * 0.5;
        v[c] = (v1[c] + _dt * r.v + v[c]) * 0.5;
        w[c] = (w1[c] + _dt * r.w + w[c]) * 0.5;
      }
}

void orc_correct_vel(const orc_grid *g, const double *p, double *u, double *v,
                     double *w) {
  // mod_calcVel.cc:253-278
  const Idx I = make_idx(g);
  const double dtdxi = g->dt * g->dx_inv;
  const double dtdyi = g->dt * g->dy_inv;
  const double _dt = g->dt;
#pragma omp parallel for
  for (int k = 1; k <= g->nz; ++k)
    for (int j = 1; j <= g->ny; ++j)
      for (int i = 1; i <= g->nx; ++i) {
        long long c = I(i, j, k);
        u[c] -= (p[I(i + 1, j, k)] - p[c]) * dtdxi;
        v[c] -= (p[I(i, j + 1, k)] - p[c]) * dtdyi;
        w[c] -= (p[I(i, j, k + 1)] - p[c]) * _dt * g->dzc_inv[k];
      }
}

double orc_mean(const orc_grid *g, int nx_global, int ny_global,
                const double *var) {
  // mod_utils.cc:30-51.  The reference sums var*dzflzi with sycl::reduction in
  // an unspecified order.  Here every product var*dzflzi is rounded to double
  // (as in the reference) and the products are accumulated in double-double
  // (error-free TwoSum), which makes the rounded total independent of the
  // summation order; the GPU reduction uses the same accumulation and so
  // reproduces this value exactly.
  const Idx I = make_idx(g);
  std::vector<double> plane_hi(g->nz + 2, 0.0), plane_lo(g->nz + 2, 0.0);
#pragma omp parallel for
  for (int k = 1; k <= g->nz; ++k) {
    double hi = 0.0, lo = 0.0;
    for (int j = 1; j <= g->ny; ++j)
      for (int i = 1; i <= g->nx; ++i) {
        const double x = var[I(i, j, k)] * g->dzflzi[k];
        two_sum_acc(hi, lo, x);
      }
    plane_hi[k] = hi;
    plane_lo[k] = lo;
  }
  double hi = 0.0, lo = 0.0;
  for (int k = 1; k <= g->nz; ++k) {
    two_sum_acc(hi, lo, plane_hi[k]);
    lo += plane_lo[k];
  }
  const double mean = hi + lo;
  return mean / nx_global / ny_global;
}

void orc_force_vel(const orc_grid *g, double *u, double *v, double *w,
                   double *force_out) {
  // mod_calcVel.cc:280-320
  double *vel[3] = {u, v, w};
  double mean[3] = {0.0, 0.0, 0.0};
  for (int d = 0; d < 3; ++d)
    if (g->is_forced[d]) mean[d] = orc_mean(g, g->nx, g->ny, vel[d]);
  const Idx I = make_idx(g);
  for (int d = 0; d < 3; ++d) {
    double f = 0.0;
    if (g->is_forced[d]) {
      f = g->vel_force[d] - mean[d];
      double *q = vel[d];
#pragma omp parallel for
      for (int k = 1; k <= g->nz; ++k)
        for (int j = 1; j <= g->ny; ++j)
          for (int i = 1; i <= g->nx; ++i) q[I(i, j, k)] += f;
    }
    if (force_out) force_out[d] = f;
  }
}

// ---------------------------------------------------------------------------
// mod_calcRHS.cc:7-33
// ---------------------------------------------------------------------------
void orc_calc_rhs(const orc_grid *g, const double *u, const double *v,
                  const double *w, double *rhs) {
  const Idx I = make_idx(g);
  const double dti = 1.0 / g->dt;
  const double dtidxi = dti * g->dx_inv;
  const double dtidyi = dti * g->dy_inv;
#pragma omp parallel for
  for (int k = 1; k <= g->nz; ++k)
    for (int j = 1; j <= g->ny; ++j)
      for (int i = 1; i <= g->nx; ++i) {
        rhs[I(i, j, k)] = (u[I(i, j, k)] - u[I(i - 1, j, k)]) * dtidxi +
                          (v[I(i, j, k)] - v[I(i, j - 1, k)]) * dtidyi +
                          (w[I(i, j, k)] - w[I(i, j, k - 1)]) * dti * g->dzf_inv[k];
      }
}

// ---------------------------------------------------------------------------
// mod_updateBound.cc:217-296
// ---------------------------------------------------------------------------
void orc_update_bound_vel(const orc_grid *g, double u_crf, double *u, double *v,
                          double *w) {
  double *vel[3] = {u, v, w};
  for (int d = 0; d < 3; ++d) halo_y_periodic(g, vel[d]);
  for (int d = 0; d < 3; ++d) halo_x_periodic(g, vel[d]);
  // imposeBCVel z branch, mod_updateBound.cc:247-260
  const double bc_u = 0.0 - u_crf;
  noslip_z(g, u, true, bc_u);
  noslip_z(g, v, true, 0.0);
  noslip_z(g, w, false, 0.0);
}

void orc_update_bound_p(const orc_grid *g, double *p) {
  halo_y_periodic(g, p);
  halo_x_periodic(g, p);
  zerograd_z(g, p);
}

// ---------------------------------------------------------------------------
// mod_utils.cc:77-217
// ---------------------------------------------------------------------------
int orc_check_nan(const orc_grid *g, const double *var) {
  const long long n = (long long)(g->nx + 2) * (g->ny + 2) * (g->nz + 2);
  for (long long t = 0; t < n; ++t)
    if (std::isnan(var[t])) return 0;
  return 1;
}

void orc_calc_max_cfl(const orc_grid *g, const double *u, const double *v,
                      const double *w, orc_value_index *out) {
  const Idx I = make_idx(g);
  double best = 0.0;
  int bi = 1, bj = 1, bk = 1;
  for (int k = 1; k <= g->nz; ++k)
    for (int j = 1; j <= g->ny; ++j)
      for (int i = 1; i <= g->nx; ++i) {
        double cfl_tmp = fabs((u[I(i, j, k)] + u[I(i - 1, j, k)]) * 0.5) * g->dx_inv +
                         fabs((v[I(i, j, k)] + v[I(i, j - 1, k)]) * 0.5) * g->dy_inv +
                         fabs((w[I(i, j, k)] + w[I(i, j, k - 1)]) * 0.5) * g->dzf_inv[k];
        if (cfl_tmp > best) {
          best = cfl_tmp;
          bi = i;
          bj = j;
          bk = k;
        }
      }
  out->value = best * g->dt;
  out->ig = bi;
  out->jg = bj;
  out->kg = bk;
}

void orc_calc_max_div(const orc_grid *g, const double *u, const double *v,
                      const double *w, orc_value_index *out) {
  const Idx I = make_idx(g);
  double best = 0.0;
  int bi = 1, bj = 1, bk = 1;
  for (int k = 1; k <= g->nz; ++k)
    for (int j = 1; j <= g->ny; ++j)
      for (int i = 1; i <= g->nx; ++i) {
        double div_tmp = fabs((u[I(i, j, k)] - u[I(i - 1, j, k)]) * g->dx_inv +
                              (v[I(i, j, k)] - v[I(i, j - 1, k)]) * g->dy_inv +
                              (w[I(i, j, k)] - w[I(i, j, k - 1)]) * g->dzf_inv[k]);
        if (div_tmp > best) {
          best = div_tmp;
          bi = i;
          bj = j;
          bk = k;
        }
      }
  out->value = best;
  out->ig = bi;
  out->jg = bj;
  out->kg = bk;
}

// ---------------------------------------------------------------------------
// mod_fft.cc
// ---------------------------------------------------------------------------
void orc_rfft_packed(int n, const double *in, double *out) {
  std::vector<cplx> a, b, tmp;
  rfft_packed_impl(n, in, out, a, b, tmp);
}

void orc_irfft_packed(int n, const double *in, double *out) {
  std::vector<cplx> a, b, tmp;
  irfft_packed_impl(n, in, out, a, b, tmp);
}

void orc_get_eigen_values(int ist, int isz, int isz_global, double *lambda) {
  // mod_fft.cc:196-222 ("PP" only)
  const double pi = acos(-1.0);
  const int ien = ist + isz - 1;
  const int n = isz_global;
  std::vector<double> lambda_glb(n), lambda_aux(n);
  for (int i = 0; i < n; i++) lambda_aux[i] = 2.0 * (cos(2.0 * pi * (i - 0.0) / n) - 1.0);
  lambda_glb[0] = lambda_aux[0];
  lambda_glb[1] = lambda_aux[n / 2];
  for (int i = 2; i < n; i++) lambda_glb[i] = lambda_aux[i / 2];
  for (int i = ist; i <= ien; i++) lambda[i - ist] = lambda_glb[i - 1];
}

// ---------------------------------------------------------------------------
// mod_poisson_solver.cc
// ---------------------------------------------------------------------------
orc_poisson *orc_poisson_init(int nx, int ny, int nz, double dx, double dy,
                              const double *dzf_global) {
  auto *ps = new orc_poisson;
  ps->nx = nx;
  ps->ny = ny;
  ps->nz = nz;
  ps->normfactor = 1.0 / (nx * ny);  // mod_fft.cc:57
  ps->var.assign((size_t)nx * ny * nz, 0.0);
  // eigenvalues, mod_poisson_solver.cc:231-246
  std::vector<double> lambdax(nx), lambday(ny), lambdaxy((size_t)nx * ny);
  orc_get_eigen_values(1, nx, nx, lambdax.data());
  for (int i = 0; i < nx; i++) lambdax[i] /= (dx * dx);
  orc_get_eigen_values(1, ny, ny, lambday.data());
  for (int i = 0; i < ny; i++) lambday[i] /= (dy * dy);
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) lambdaxy[i + (size_t)j * nx] = lambdax[i] + lambday[j];
  // set_trid_coeff(nz, dzf, "NN", 'c', PROC_NULL x2), mod_poisson_solver.cc:35-98
  ps->a.assign(nz, 0.0);
  ps->c.assign(nz, 0.0);
  std::vector<double> b_tmp(nz);
  const double *dzf = dzf_global;  // st_trid[2] = 1, :261-263
  const int dzf_st = -1;
  for (int k = 0; k < nz; k++) {
    ps->a[k] = 2.0 / (dzf[k - dzf_st] * (dzf[k - 1 - dzf_st] + dzf[k - dzf_st]));
    ps->c[k] = 2.0 / (dzf[k - dzf_st] * (dzf[k + 1 - dzf_st] + dzf[k - dzf_st]));
  }
  for (int i = 0; i < nz; i++) b_tmp[i] = -ps->a[i] - ps->c[i];
  {
    const double factor = 1.0;  // 'N'
    b_tmp[0] += factor * ps->a[0];
    ps->a[0] *= fabs(factor) - 1.0;
    b_tmp[nz - 1] += factor * ps->c[nz - 1];
    ps->c[nz - 1] *= fabs(factor) - 1.0;
  }
  // b = b_tmp + lambdaxy, then pre-eliminated over k, :265-282
  ps->b.assign((size_t)nx * ny * nz, 0.0);
  const size_t plane = (size_t)nx * ny;
  for (int k = 0; k < nz; k++)
    for (size_t t = 0; t < plane; t++) ps->b[t + k * plane] = b_tmp[k] + lambdaxy[t];
  for (int k = 1; k < nz; k++) {
#pragma omp parallel for
    for (long long t = 0; t < (long long)plane; t++) {
      double a_tmp = ps->a[k] / ps->b[t + (k - 1) * plane];
      ps->b[t + k * plane] -= (a_tmp * ps->c[k - 1]);
    }
  }
  return ps;
}

void orc_poisson_free(orc_poisson *ps) { delete ps; }
double *orc_poisson_work(orc_poisson *ps) { return ps->var.data(); }
const double *orc_poisson_b(const orc_poisson *ps) { return ps->b.data(); }
const double *orc_poisson_a(const orc_poisson *ps) { return ps->a.data(); }
const double *orc_poisson_c(const orc_poisson *ps) { return ps->c.data(); }

void orc_fft_fwd_xpen(orc_poisson *ps, const double *p, double *var) {
  // mod_fft.cc:60-88: copy interior line, forward real DFT, packed layout
  const int nx = ps->nx, ny = ps->ny, nz = ps->nz;
  const int X = nx + 2, Y = ny + 2;
#pragma omp parallel
  {
    std::vector<cplx> a, b, tmp;
    std::vector<double> line(nx);
#pragma omp for collapse(2)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j) {
        const double *src = p + (size_t)X * ((j + 1) + (size_t)Y * (k + 1)) + 1;
        for (int i = 0; i < nx; ++i) line[i] = src[i];
        rfft_packed_impl(nx, line.data(), var + ((size_t)k * ny + j) * nx, a, b, tmp);
      }
  }
}

void orc_fft_bwd_xpen(orc_poisson *ps, const double *var, double *p) {
  // mod_fft.cc:90-120: inverse real DFT, scaled by 1/(nx*ny), into the interior
  const int nx = ps->nx, ny = ps->ny, nz = ps->nz;
  const int X = nx + 2, Y = ny + 2;
  const double nf = ps->normfactor;
#pragma omp parallel
  {
    std::vector<cplx> a, b, tmp;
    std::vector<double> line(nx);
#pragma omp for collapse(2)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j) {
        irfft_packed_impl(nx, var + ((size_t)k * ny + j) * nx, line.data(), a, b, tmp);
        double *dst = p + (size_t)X * ((j + 1) + (size_t)Y * (k + 1)) + 1;
        for (int i = 0; i < nx; ++i) dst[i] = nf * line[i];
      }
  }
}

void orc_fft_fwd_ypen(orc_poisson *ps, double *var) {
  // mod_fft.cc:122-153: real DFT along y of every packed-x column
  const int nx = ps->nx, ny = ps->ny, nz = ps->nz;
#pragma omp parallel
  {
    std::vector<cplx> a, b, tmp;
    std::vector<double> line(ny), out(ny);
#pragma omp for collapse(2)
    for (int k = 0; k < nz; ++k)
      for (int i = 0; i < nx; ++i) {
        double *base = var + (size_t)k * nx * ny + i;
        for (int j = 0; j < ny; ++j) line[j] = base[(size_t)j * nx];
        rfft_packed_impl(ny, line.data(), out.data(), a, b, tmp);
        for (int j = 0; j < ny; ++j) base[(size_t)j * nx] = out[j];
      }
  }
}

void orc_fft_bwd_ypen(orc_poisson *ps, double *var) {
  // mod_fft.cc:155-187
  const int nx = ps->nx, ny = ps->ny, nz = ps->nz;
#pragma omp parallel
  {
    std::vector<cplx> a, b, tmp;
    std::vector<double> line(ny), out(ny);
#pragma omp for collapse(2)
    for (int k = 0; k < nz; ++k)
      for (int i = 0; i < nx; ++i) {
        double *base = var + (size_t)k * nx * ny + i;
        for (int j = 0; j < ny; ++j) line[j] = base[(size_t)j * nx];
        irfft_packed_impl(ny, line.data(), out.data(), a, b, tmp);
        for (int j = 0; j < ny; ++j) base[(size_t)j * nx] = out[j];
      }
  }
}

void orc_ssolve_trid(orc_poisson *ps, double *var) {
  // mod_poisson_solver.cc:317-357 (Thomas with the pre-factored b; a zero
  // final pivot sets the last unknown to zero)
  const int ie = ps->nx, je = ps->ny, ke = ps->nz;
  const size_t plane = (size_t)ie * je;
  const double *_a = ps->a.data(), *_b = ps->b.data(), *_c = ps->c.data();
#pragma omp parallel for
  for (long long t = 0; t < (long long)plane; ++t) {
    for (int k = 1; k < ke; ++k) {
      double var_up = var[(k - 1) * plane + t];
      double bv = _b[(k - 1) * plane + t];
      double a_tmp = _a[k] / bv;
      var[k * plane + t] -= a_tmp * var_up;
    }
    double b_val = _b[(ke - 1) * plane + t];
    double &var_p = var[(ke - 1) * plane + t];
    if (b_val != 0)
      var_p /= b_val;
    else
      var_p = 0;
    for (int k = ke - 2; k >= 0; k--) {
      double &var_down = var[k * plane + t];
      double var_up = var[(k + 1) * plane + t];
      double bv = _b[k * plane + t];
      double cv = _c[k];
      var_down = (var_down - cv * var_up) / bv;
    }
  }
}

void orc_poisson_execute(orc_poisson *ps, double *p) {
  // mod_poisson_solver.cc:454-510 at p_row = p_col = 1 (all transposes alias)
  double *var = ps->var.data();
  orc_fft_fwd_xpen(ps, p, var);
  orc_fft_fwd_ypen(ps, var);
  orc_ssolve_trid(ps, var);
  orc_fft_bwd_ypen(ps, var);
  orc_fft_bwd_xpen(ps, var, p);
}

// ---------------------------------------------------------------------------
// mod_initFlow.cc
// ---------------------------------------------------------------------------
double orc_noise_uniform(int seed, long long offset) {
  const uint64_t m = 2147483647ull, a = 48271ull;
  uint64_t x = (uint64_t)((long long)seed % (long long)m);
  if (x == 0) x = 1;
  // x_{offset+1} = a^(offset+1) * x0 mod m
  uint64_t e = (uint64_t)offset + 1ull, base = a, mult = 1ull;
  while (e) {
    if (e & 1ull) mult = (mult * base) % m;
    base = (base * base) % m;
    e >>= 1;
  }
  x = (x * mult) % m;
  return (double)(x - 1ull) / (double)(m - 1ull);
}

void orc_init_flow(const orc_grid *g, int initial_field, double u0,
                   double u_ref, double re, int init_with_noise,
                   double noise_intensity, const double *zc_global, double *u,
                   double *v, double *w) {
  const Idx I = make_idx(g);
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  std::vector<double> u_prof(nz + 1, 0.0);
  bool is_mean = false;
  if (initial_field == 0) {  // "uni", :70-74
    for (int k = 1; k <= nz; ++k) u_prof[k] = u0;
    is_mean = false;
  } else if (initial_field == 1) {  // "poi", :75-80 and :16-21
    for (int k = 1; k <= nz; ++k) {
      double z = zc_global[k] / g->lz;
      u_prof[k] = 6.0 * (1.0 - z) * z * u_ref;
    }
    is_mean = true;
  } else if (initial_field == 2) {  // "log", :81-86 and :23-30
    double retau = 0.09 * pow(re, 0.88);
    for (int k = 1; k <= nz; ++k) {
      double zn = zc_global[k] / g->lz;
      double z = fmin(zn, 1.0 - zn) * 2.0 * retau;
      u_prof[k] = (z <= 11.6 ? z : 2.5 * log(z) + 5.5);
    }
    is_mean = true;
  }
#pragma omp parallel for
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) u[I(i, j, k)] = u_prof[k];
  if (init_with_noise) {  // :102-106, addNoise :31-44
    const int seeds[3] = {123, 456, 789};
    double *vel[3] = {u, v, w};
    for (int d = 0; d < 3; ++d) {
      double *q = vel[d];
#pragma omp parallel for
      for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
          for (int i = 1; i <= nx; ++i) {
            long long offset = ((long long)(k - 1) * ny + (j - 1)) * nx + (i - 1);
            q[I(i, j, k)] += 2.0 * (orc_noise_uniform(seeds[d], offset) - 0.5) * noise_intensity;
          }
    }
  }
  if (is_mean) {
    // :108-118; the reference passes (nz, ny) as the global sizes here
    double meanold = orc_mean(g, nz, ny, u);
    if (meanold != 0.0) {
      double multiplier = 1.0 / (meanold * u_ref);
#pragma omp parallel for
      for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
          for (int i = 1; i <= nx; ++i) u[I(i, j, k)] *= multiplier;
    }
  }
}

// ---------------------------------------------------------------------------
// main.cc:116-154
// ---------------------------------------------------------------------------
// The CFL rate max(|u_c|/dx + |v_c|/dy + |w_c|/dzf) of calcMaxCFL
// (mod_utils.cc:108-150) before its multiplication by dt: each point's value
// is the reference's expression, and the maximum does not depend on the
// order, so threads split the planes.
static double cfl_rate(const orc_grid *g, const double *u, const double *v, const double *w) {
  const Idx I = make_idx(g);
  double best = 0.0;
#pragma omp parallel for reduction(max : best)
  for (int k = 1; k <= g->nz; ++k)
    for (int j = 1; j <= g->ny; ++j)
      for (int i = 1; i <= g->nx; ++i) {
        const double cfl_tmp = fabs((u[I(i, j, k)] + u[I(i - 1, j, k)]) * 0.5) * g->dx_inv +
                               fabs((v[I(i, j, k)] + v[I(i, j - 1, k)]) * 0.5) * g->dy_inv +
                               fabs((w[I(i, j, k)] + w[I(i, j, k - 1)]) * 0.5) * g->dzf_inv[k];
        if (cfl_tmp > best) best = cfl_tmp;
      }
  return best;
}

void orc_run_cfl(const orc_grid *g0, orc_poisson *ps, int nsteps, int nt_check,
                 double cfl_target, double *u, double *v, double *w, double *u1,
                 double *v1, double *w1, double *p, double *dt_used) {
  // The time step of the main loop (main.cc:114-178) under a CFL target:
  // dt = cfl_target / rate, where rate * dt is calcMaxCFL's value
  // (mod_utils.cc:122-144), evaluated before the first step, after steps
  // 1, 2, 4, 8, ... below nt_check (the first forcing step moves the bulk
  // velocity from the initial field's rescaled value to vel_force), and
  // after every nt_check-th step, where main.cc:156-178 runs its checks.
  orc_grid g = *g0;
  auto retune = [&]() {
    const double rate = cfl_rate(&g, u, v, w);
    if (rate > 0.0) g.dt = cfl_target / rate;
  };
  if (cfl_target > 0.0) retune();
  for (int s = 1; s <= nsteps; ++s) {
    if (dt_used) dt_used[s - 1] = g.dt;
    orc_step(&g, ps, 1, u, v, w, u1, v1, w1, p);
    if (cfl_target <= 0.0) continue;
    if (s < nt_check && (s & (s - 1)) == 0)
      retune();
    else if (nt_check > 0 && s % nt_check == 0)
      retune();
  }
  if (dt_used) dt_used[nsteps] = g.dt;
}

void orc_step(const orc_grid *g, orc_poisson *ps, int nsteps, double *u,
              double *v, double *w, double *u1, double *v1, double *w1,
              double *p) {
  for (int s = 0; s < nsteps; ++s) {
    orc_time_int_vel_rk1(g, g->u_crf, u, v, w, u1, v1, w1);
    orc_update_bound_vel(g, g->u_crf, u1, v1, w1);
    orc_time_int_vel_rk2(g, g->u_crf, u, v, w, u1, v1, w1);
    orc_update_bound_vel(g, g->u_crf, u, v, w);
    orc_calc_rhs(g, u, v, w, p);
    orc_poisson_execute(ps, p);
    orc_update_bound_p(g, p);
    orc_correct_vel(g, p, u, v, w);
    orc_force_vel(g, u, v, w, nullptr);
    orc_update_bound_vel(g, g->u_crf, u, v, w);
  }
}

}  // extern "C"
