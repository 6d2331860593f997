// TEST INFRASTRUCTURE ONLY.
//
// A stand-in for the oneMKL DFT interface that the reference's mod_fft.cc
// uses (descriptor<DOUBLE, REAL>, set_value, commit, compute_forward,
// compute_backward), so that its unmodified source runs on the CPU.  oneMKL
// itself is closed source and absent here; this computes the transforms its
// documentation defines, for the configuration the reference sets:
//  * forward (real -> complex, in place): for each of NUMBER_OF_TRANSFORMS
//    sequences, x_j = data[b * FWD_DISTANCE + j] (j < n, unit stride) gives
//    z_k = sum_j x_j exp(-2 pi i j k / n), k = 0 .. n/2, stored as
//    (re, im) pairs from data[b * 2 * BWD_DISTANCE] on (the CCE layout);
//  * backward (complex -> real): the inverse sum with exp(+2 pi i j k / n)
//    over the Hermitian-extended z (z_{n-k} = conj z_k), unscaled, the
//    imaginary parts of z_0 and z_{n/2} not used;
//  * strides other than {0, 1} and odd n are refused.
// Each real sequence of even length n is transformed as one complex
// sequence of length n/2 (x_{2m} + i x_{2m+1}) by a recursive mixed-radix
// (4, 2, 3, then any factor) decimation-in-time FFT, followed by the
// standard split into the real spectrum; twiddles are cos/sin of 2 pi j / n
// evaluated directly.  Sequences are spread over OpenMP threads.
#pragma once

#include <CL/sycl.hpp>

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

typedef long long MKL_LONG;

namespace oneapi {
namespace mkl {
namespace dft {

enum class precision { SINGLE, DOUBLE };
enum class domain { REAL, COMPLEX };
enum class config_param {
  NUMBER_OF_TRANSFORMS,
  INPUT_STRIDES,
  OUTPUT_STRIDES,
  FWD_DISTANCE,
  BWD_DISTANCE,
  FORWARD_SCALE,
  BACKWARD_SCALE,
  PLACEMENT
};

namespace shim {

using cplx = std::complex<double>;

inline void fail(const char *what) {
  std::fprintf(stderr, "oneMKL DFT shim: %s\n", what);
  std::abort();
}

// out[k] = sum_m in[m * stride] W_L^{m k}, k < L, with W_L^e = tw[e * (N / L)]
// and tw[e] = exp(-+ 2 pi i e / N) (the sign is in the table).
inline void fft_rec(const cplx *in, long stride, cplx *out, int L, const cplx *tw, int N,
                    cplx *scratch) {
  if (L == 1) {
    out[0] = in[0];
    return;
  }
  int r = 0;
  if (L % 4 == 0)
    r = 4;
  else if (L % 2 == 0)
    r = 2;
  else if (L % 3 == 0)
    r = 3;
  else {
    for (int f = 5; f * f <= L; f += 2)
      if (L % f == 0) {
        r = f;
        break;
      }
    if (!r) r = L;
  }
  const int M = L / r;
  if (M == 1) {  // a direct DFT of length r
    for (int k = 0; k < L; ++k) {
      cplx acc = 0.0;
      for (int m = 0; m < L; ++m) acc += in[m * stride] * tw[(long)((m * (long)k) % L) * (N / L)];
      out[k] = acc;
    }
    return;
  }
  // sub-transforms of the r decimated sequences into out[q * M ...]
  for (int q = 0; q < r; ++q) fft_rec(in + q * stride, stride * r, out + q * M, M, tw, N, scratch);
  // butterflies: X[k + M s] = sum_q W_L^{q k} W_r^{q s} Y_q[k]
  const long wl = N / L;
  for (int k = 0; k < M; ++k) {
    cplx y[64];
    cplx *yy = r <= 64 ? y : scratch;
    for (int q = 0; q < r; ++q) yy[q] = out[q * M + k] * tw[(long)q * k * wl % N];
    for (int s = 0; s < r; ++s) {
      cplx acc = 0.0;
      for (int q = 0; q < r; ++q) acc += yy[q] * tw[((long)q * s % r) * (N / r)];
      scratch[r + s] = acc;
    }
    for (int s = 0; s < r; ++s) out[k + M * s] = scratch[r + s];
  }
}

}  // namespace shim

template <precision P, domain D>
class descriptor {
 public:
  explicit descriptor(std::int64_t n) : n_(n) {
    static_assert(P == precision::DOUBLE && D == domain::REAL, "DOUBLE/REAL only");
  }
  template <class T>
  void set_value(config_param p, T v) {
    if constexpr (std::is_pointer_v<T> || std::is_array_v<T>) {
      if (v[0] != 0 || v[1] != 1) shim::fail("strides other than {0, 1}");
    } else {
      switch (p) {
        case config_param::NUMBER_OF_TRANSFORMS: howmany_ = (long)v; break;
        case config_param::FWD_DISTANCE: fwd_ = (long)v; break;
        case config_param::BWD_DISTANCE: bwd_ = (long)v; break;
        default: shim::fail("unsupported configuration parameter");
      }
    }
  }
  void commit(sycl::queue &) {
    if (n_ < 2 || n_ % 2) shim::fail("odd or short length");
    const int L = (int)(n_ / 2);
    twf_.resize(L);
    twb_.resize(L);
    for (int e = 0; e < L; ++e) {
      const double a = 2.0 * M_PI * (double)e / (double)L;
      twf_[e] = shim::cplx(std::cos(a), -std::sin(a));
      twb_[e] = std::conj(twf_[e]);
    }
    split_.resize(L + 1);
    for (int k = 0; k <= L; ++k) {
      const double a = 2.0 * M_PI * (double)k / (double)n_;
      split_[k] = shim::cplx(std::cos(a), -std::sin(a));  // exp(-2 pi i k / n)
    }
  }

  void forward(double *data) const {
    const int L = (int)(n_ / 2);
#pragma omp parallel
    {
      std::vector<shim::cplx> c(L), C(L), scratch(2 * L + 2);
#pragma omp for schedule(static)
      for (long b = 0; b < howmany_; ++b) {
        double *x = data + b * fwd_;
        for (int m = 0; m < L; ++m) c[m] = shim::cplx(x[2 * m], x[2 * m + 1]);
        shim::fft_rec(c.data(), 1, C.data(), L, twf_.data(), L, scratch.data());
        double *z = data + b * 2 * bwd_;
        // z_k = E_k + W^k O_k with E_k = (C_k + conj C_{L-k}) / 2,
        // O_k = (C_k - conj C_{L-k}) / (2 i)
        for (int k = 0; k <= L; ++k) {
          const shim::cplx Ck = C[k % L], Cm = std::conj(C[(L - k) % L]);
          const shim::cplx E = 0.5 * (Ck + Cm);
          const shim::cplx O = shim::cplx(0.0, -0.5) * (Ck - Cm);
          const shim::cplx zk = E + split_[k] * O;
          scratch[k] = zk;
        }
        for (int k = 0; k <= L; ++k) {
          z[2 * k] = scratch[k].real();
          z[2 * k + 1] = scratch[k].imag();
        }
      }
    }
  }

  void backward(double *data) const {
    const int L = (int)(n_ / 2);
#pragma omp parallel
    {
      std::vector<shim::cplx> c(L), C(L), scratch(2 * L + 2), z(L + 1);
#pragma omp for schedule(static)
      for (long b = 0; b < howmany_; ++b) {
        const double *zp = data + b * 2 * bwd_;
        for (int k = 0; k <= L; ++k) z[k] = shim::cplx(zp[2 * k], zp[2 * k + 1]);
        z[0] = shim::cplx(z[0].real(), 0.0);
        z[L] = shim::cplx(z[L].real(), 0.0);
        // C_k = E_k + i conj(W^k) ... the inverse of the forward split:
        // E_k = (z_k + conj z_{L-k}) / 2, O_k = (z_k - conj z_{L-k}) conj(W^k) / 2,
        // C_k = E_k + i O_k (times 2 for the unscaled length-n inverse)
        for (int k = 0; k < L; ++k) {
          const shim::cplx zk = z[k], zm = std::conj(z[L - k]);
          const shim::cplx E = zk + zm;
          const shim::cplx O = (zk - zm) * std::conj(split_[k]);
          c[k] = E + shim::cplx(0.0, 1.0) * O;
        }
        shim::fft_rec(c.data(), 1, C.data(), L, twb_.data(), L, scratch.data());
        double *x = data + b * fwd_;
        for (int m = 0; m < L; ++m) {
          x[2 * m] = C[m].real();
          x[2 * m + 1] = C[m].imag();
        }
      }
    }
  }

 private:
  long n_ = 0, howmany_ = 1, fwd_ = 0, bwd_ = 0;
  std::vector<shim::cplx> twf_, twb_, split_;
};

template <class Desc>
sycl::event compute_forward(Desc &desc, double *inout, const std::vector<sycl::event> & = {}) {
  desc.forward(inout);
  return sycl::event{};
}

template <class Desc>
sycl::event compute_backward(Desc &desc, double *inout, const std::vector<sycl::event> & = {}) {
  desc.backward(inout);
  return sycl::event{};
}

}  // namespace dft
}  // namespace mkl
}  // namespace oneapi
