// Batched real FFTs and the wall-normal tridiagonal solve of the Poisson
// projection, in FP64 (the reference's arithmetic) and in FP32 storage for
// the mixed-precision form.
//
// The reference (mod_fft.cc) copies p into a padded buffer, calls oneMKL's
// batched real DFT and repacks the result; the y transform goes through an
// explicit transpose.  Here each transform is ONE pass over HBM:
//
//  * Two real lines a, b are transformed together as z = a + i*b with a
//    complex FFT held in shared memory; A_m = (Z_m + conj Z_{n-m})/2 and
//    B_m = (Z_m - conj Z_{n-m})/(2i) are written directly in the packed real
//    layout of the reference (index 0 = Re X_0, 1 = Re X_{n/2},
//    2m / 2m+1 = Re / Im X_m; mod_fft.cc:79-86).
//  * x lines pair the rows j, j+1 of one z plane (contiguous loads); the
//    forward x transform of the fused step evaluates div(u)/dt while loading
//    (calcRHS fused, mod_calcRHS.cc:23-30).
//  * y lines pair adjacent packed-x columns i, i+1 and are read and written in
//    place with x-contiguous row segments: no transpose buffer.
//  * The complex FFT is a mixed-radix (16, 8, 4, 2, 3) Stockham transform between
//    two shared-memory buffers, one butterfly per thread and pass; element e
//    of a line lives at e + e/8 (FP64) or e + e/16 (FP32) to spread the
//    strided accesses over the banks.
//  * Both transforms are unscaled; the backward x transform multiplies by
//    1/(nx*ny) (mod_fft.cc:57,116-117) and, in the fused step, also writes
//    the pressure halos (updateBoundP, mod_updateBound.cc:287-330).
//
// Every kernel is a template on the storage type T (double, float); the
// transform arithmetic runs in T with twiddles rounded once from long double.
//
// The tridiagonal solve (ssolve_trid, mod_poisson_solver.cc:317-357) is a
// Thomas sweep per (kx,ky) system, one thread per system, coalesced over kx,
// with the pre-factored reciprocal pivots read from a table indexed by the
// distinct wavenumber pair.  In the mixed form the systems of the lowest
// wavenumbers sweep in FP64 (pivots, arithmetic and intermediate values), the
// others in FP32.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <type_traits>
#include <vector>

#include "plc_device.cuh"
#include "plc_internal.h"

namespace plc {

namespace {

template <class T>
struct Cx;
template <>
struct Cx<double> {
  using V = double2;
  static constexpr int kPadShift = 3;  // one pad element per 128 bytes
};
template <>
struct Cx<float> {
  using V = float2;
  static constexpr int kPadShift = 4;
};
template <class V>
using ScalarOf = decltype(V::x);
template <class V>
constexpr int pad_shift() {
  return Cx<ScalarOf<V>>::kPadShift;
}

template <class V>
__device__ __forceinline__ V mk(ScalarOf<V> x, ScalarOf<V> y) {
  V r;
  r.x = x;
  r.y = y;
  return r;
}

template <class V>
struct FftDev {
  int n, npass;
  unsigned long long radices;  // radix - 1, 4 bits per pass, pass 0 in the low bits
  const V *tw;
};

template <class V>
__device__ __forceinline__ int padi(int e) {
  return e + (e >> pad_shift<V>());
}

template <class V>
__host__ __device__ __forceinline__ constexpr int line_stride(int n) {
  return n + (n >> pad_shift<V>()) + 1;
}

template <class V>
__device__ __forceinline__ V cmul(V a, V b) {
  return mk<V>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <class V>
__device__ __forceinline__ V cmulc(V a, V b) {
  return mk<V>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <class V>
__device__ __forceinline__ V cadd(V a, V b) {
  return mk<V>(a.x + b.x, a.y + b.y);
}
template <class V>
__device__ __forceinline__ V csub(V a, V b) {
  return mk<V>(a.x - b.x, a.y - b.y);
}
// FP32 complex arithmetic on Blackwell's packed FP32x2 instructions (FADD2,
// FMUL2, FFMA2): a complex add or subtract is one instruction, a complex
// product two, instead of two and four scalar ones.  The FFT butterflies are
// mostly these operations; FP64 keeps the scalar forms above.
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
  return __ffma2_rn(b, make_float2(-1.f, -1.f), a);  // exact product, one rounding
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  const float2 t = __fmul2_rn(make_float2(a.x, a.x), b);  // (ax bx, ax by)
  return __ffma2_rn(make_float2(-a.y, a.y), make_float2(b.y, b.x), t);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
  const float2 t = __fmul2_rn(a, make_float2(b.x, b.x));      // (ax bx, ay bx)
  return __ffma2_rn(make_float2(a.y, -a.x), make_float2(b.y, b.y), t);
}
// multiply by -i (forward) or +i (inverse)
template <bool INV, class V>
__device__ __forceinline__ V rot90(V a) {
  return INV ? mk<V>(-a.y, a.x) : mk<V>(a.y, -a.x);
}

template <int R, bool INV>
struct Dft;

template <bool INV>
struct Dft<2, INV> {
  template <class V>
  __device__ __forceinline__ static void run(V (&v)[2]) {
    const V a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <bool INV>
struct Dft<4, INV> {
  template <class V>
  __device__ __forceinline__ static void run(V (&v)[4]) {
    const V t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    const V t2 = cadd(v[1], v[3]), t3 = rot90<INV>(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  }
};

template <bool INV>
struct Dft<8, INV> {
  template <class V>
  __device__ __forceinline__ static void run(V (&v)[8]) {
    using S = ScalarOf<V>;
    const S s = S(0.70710678118654752440);  // 1/sqrt(2)
    V e[4] = {v[0], v[2], v[4], v[6]};
    V o[4] = {v[1], v[3], v[5], v[7]};
    Dft<4, INV>::run(e);
    Dft<4, INV>::run(o);
    // o[m] *= W8^m, W8 = exp(-+ i pi/4)
    V x = o[1];
    o[1] = INV ? mk<V>(s * (x.x - x.y), s * (x.x + x.y)) : mk<V>(s * (x.x + x.y), s * (x.y - x.x));
    o[2] = rot90<INV>(o[2]);
    x = o[3];
    o[3] = INV ? mk<V>(-s * (x.x + x.y), s * (x.x - x.y))
               : mk<V>(s * (x.y - x.x), -s * (x.x + x.y));
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      v[m] = cadd(e[m], o[m]);
      v[m + 4] = csub(e[m], o[m]);
    }
  }
};

template <bool INV>
struct Dft<16, INV> {
  template <class V>
  __device__ __forceinline__ static void run(V (&v)[16]) {
    // radix-2 step over two 8-point transforms: X_k = E_k + W16^k O_k,
    // X_{k+8} = E_k - W16^k O_k, W16 = exp(-+ 2 pi i / 16)
    using S = ScalarOf<V>;
    const S c1 = S(0.92387953251128675613);  // cos(pi/8)
    const S s1 = S(0.38268343236508977173);  // sin(pi/8)
    const S h = S(0.70710678118654752440);   // 1/sqrt(2)
    V e[8], o[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      e[m] = v[2 * m];
      o[m] = v[2 * m + 1];
    }
    Dft<8, INV>::run(e);
    Dft<8, INV>::run(o);
    const V w[8] = {mk<V>(S(1), S(0)), mk<V>(c1, -s1), mk<V>(h, -h),   mk<V>(s1, -c1),
                    mk<V>(S(0), S(-1)), mk<V>(-s1, -c1), mk<V>(-h, -h), mk<V>(-c1, -s1)};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const V t = INV ? cmulc(o[k], w[k]) : cmul(o[k], w[k]);
      v[k] = cadd(e[k], t);
      v[k + 8] = csub(e[k], t);
    }
  }
};

// 32 points: a radix-2 step over two 16-point transforms, X_k = E_k + W32^k O_k,
// X_{k+16} = E_k - W32^k O_k, W32 = exp(-+ 2 pi i / 32)
template <bool INV>
struct Dft<32, INV> {
  template <class V>
  __device__ __forceinline__ static void run(V (&v)[32]) {
    using S = ScalarOf<V>;
    // cos and sin of j pi / 16, j = 0 .. 7
    const S c[8] = {S(1),
                    S(0.98078528040323044913),
                    S(0.92387953251128675613),
                    S(0.83146961230254523708),
                    S(0.70710678118654752440),
                    S(0.55557023301960222474),
                    S(0.38268343236508977173),
                    S(0.19509032201612826785)};
    V e[16], o[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) {
      e[m] = v[2 * m];
      o[m] = v[2 * m + 1];
    }
    Dft<16, INV>::run(e);
    Dft<16, INV>::run(o);
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      // W32^k = cos(k pi/16) - i sin(k pi/16); for k >= 8, -i W32^(k-8)
      const V w = k < 8 ? mk<V>(c[k], k == 0 ? S(0) : -c[8 - k])
                        : mk<V>(k == 8 ? S(0) : -c[16 - k], -c[k - 8]);
      const V t = k == 0 ? o[0] : (INV ? cmulc(o[k], w) : cmul(o[k], w));
      v[k] = cadd(e[k], t);
      v[k + 16] = csub(e[k], t);
    }
  }
};

template <bool INV>
struct Dft<3, INV> {
  template <class V>
  __device__ __forceinline__ static void run(V (&v)[3]) {
    using S = ScalarOf<V>;
    const S h = S(0.86602540378443864676);  // sqrt(3)/2
    const V t1 = cadd(v[1], v[2]);
    const V t2 = mk<V>(v[0].x - S(0.5) * t1.x, v[0].y - S(0.5) * t1.y);
    const V d = csub(v[1], v[2]);
    const V t3 = INV ? mk<V>(-h * d.y, h * d.x) : mk<V>(h * d.y, -h * d.x);
    v[0] = cadd(v[0], t1);
    v[1] = cadd(t2, t3);
    v[2] = csub(t2, t3);
  }
};

// 24-point DFT as three 8-point DFTs of the interleaved subsequences
// x[3m + r], the twiddles W24^(r k), and eight 3-point DFTs across r:
// X[k + 8q] = sum_r W3^(r q) W24^(r k) Y_r[k] (Cooley-Tukey with n = 3m + r,
// k' = k + 8q).  The twiddles W24^j = cos(15 j deg) -+ i sin(15 j deg) that are
// not trivial are applied by complex multiplication; j = 6 is a rotation by
// 90 degrees and j = 3 a scaled sum and difference.
template <bool INV>
struct Dft<24, INV> {
  template <class V>
  __device__ __forceinline__ static void run(V (&v)[24]) {
    using S = ScalarOf<V>;
    // cos and sin of 15 j degrees, j = 0 .. 14
    const S c[15] = {S(1),
                     S(0.96592582628906828675),
                     S(0.86602540378443864676),
                     S(0.70710678118654752440),
                     S(0.5),
                     S(0.25881904510252076235),
                     S(0),
                     S(-0.25881904510252076235),
                     S(-0.5),
                     S(-0.70710678118654752440),
                     S(-0.86602540378443864676),
                     S(-0.96592582628906828675),
                     S(-1),
                     S(-0.96592582628906828675),
                     S(-0.86602540378443864676)};
    const S sn[15] = {S(0),
                      S(0.25881904510252076235),
                      S(0.5),
                      S(0.70710678118654752440),
                      S(0.86602540378443864676),
                      S(0.96592582628906828675),
                      S(1),
                      S(0.96592582628906828675),
                      S(0.86602540378443864676),
                      S(0.70710678118654752440),
                      S(0.5),
                      S(0.25881904510252076235),
                      S(0),
                      S(-0.25881904510252076235),
                      S(-0.5)};
    V y[3][8];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
#pragma unroll
      for (int m = 0; m < 8; ++m) y[r][m] = v[3 * m + r];
      Dft<8, INV>::run(y[r]);
    }
#pragma unroll
    for (int r = 1; r < 3; ++r)
#pragma unroll
      for (int k = 1; k < 8; ++k) {
        const int j = r * k;
        const V x = y[r][k];
        if (j == 6) {
          y[r][k] = rot90<INV>(x);
        } else if (j == 3) {  // W24^3 = (1 -+ i)/sqrt(2)
          const S h = c[3];
          y[r][k] = INV ? mk<V>(h * (x.x - x.y), h * (x.x + x.y))
                        : mk<V>(h * (x.x + x.y), h * (x.y - x.x));
        } else {
          const V w = mk<V>(c[j], -sn[j]);  // W24^j, forward sign
          y[r][k] = INV ? cmulc(x, w) : cmul(x, w);
        }
      }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      V t[3] = {y[0][k], y[1][k], y[2][k]};
      Dft<3, INV>::run(t);
      v[k] = t[0];
      v[k + 8] = t[1];
      v[k + 16] = t[2];
    }
  }
};

// One Stockham pass of radix R over nl lines of length n (line stride LS).
template <int R, bool INV, class V>
__device__ __forceinline__ void fft_pass(const V *__restrict__ src, V *__restrict__ dst, int nl,
                                         int n, int LS, int Ns, const V *__restrict__ tw) {
  const int nb = n / R;
  const int tot = nl * nb;
  const int tws = n / (Ns * R);
  for (int b = threadIdx.x; b < tot; b += blockDim.x) {
    const int l = b / nb;
    const int j = b - l * nb;
    const V *s = src + l * LS;
    V *d = dst + l * LS;
    const int jm = j % Ns;
    V v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = s[padi<V>(j + r * nb)];
    if (jm != 0) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        const V w = __ldg(tw + r * jm * tws);
        v[r] = INV ? cmulc(v[r], w) : cmul(v[r], w);
      }
    }
    Dft<R, INV>::run(v);
    const int idxD = (j / Ns) * Ns * R + jm;
#pragma unroll
    for (int r = 0; r < R; ++r) d[padi<V>(idxD + r * Ns)] = v[r];
  }
}

// Complex FFT of nl lines held in A; returns the buffer holding the result.
template <bool INV, class V>
__device__ V *fft_run(V *A, V *B, int nl, int LS, const FftDev<V> &P) {
  int Ns = 1;
  for (int p = 0; p < P.npass; ++p) {
    const int R = (int)((P.radices >> (4 * p)) & 15ull) + 1;
    switch (R) {
      case 16: fft_pass<16, INV>(A, B, nl, P.n, LS, Ns, P.tw); break;
      case 8: fft_pass<8, INV>(A, B, nl, P.n, LS, Ns, P.tw); break;
      case 4: fft_pass<4, INV>(A, B, nl, P.n, LS, Ns, P.tw); break;
      case 2: fft_pass<2, INV>(A, B, nl, P.n, LS, Ns, P.tw); break;
      default: fft_pass<3, INV>(A, B, nl, P.n, LS, Ns, P.tw); break;
    }
    __syncthreads();
    V *t = A;
    A = B;
    B = t;
    Ns *= R;
  }
  return A;
}

// ---------------------------------------------------------------------------
// Compile-time plans.  For the line lengths of the supported grids the radix
// sequence (the rule of host_fft_factor: 16s, then one 8/4/2, then 3s) and
// all index arithmetic are constants, the passes are unrolled and the
// integer divisions become multiplications; N = 0 selects the runtime plan.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int count2(int n) {
  int a = 0;
  while (n > 0 && n % 2 == 0) {
    n /= 2;
    ++a;
  }
  return a;
}
__host__ __device__ constexpr int count3(int n) {
  int b = 0;
  while (n > 0 && n % 3 == 0) {
    n /= 3;
    ++b;
  }
  return b;
}
// Two plan families.  Family 0: 16s, then one 8/4/2, then 3s.  Family 1 (W24),
// for lengths 3 * 2^a with 3 <= a <= 7 (24 .. 384): two passes, radix 2^(a-3)
// and then 24 (one pass for 24 itself).  Each context's autotuner times both
// families where a length has two (with the tile sizes) and keeps the faster
// per direction: in FP32 the radix-24 family wins for the y lines of the
// 768 x 384 x 256 case; in FP64 its 24 complex values per butterfly need about
// 156 registers, which halves the resident blocks.
__host__ __device__ constexpr bool plan_has24(int n) {
  const int a = count2(n);
  return (n >> a) == 3 && a >= 3 && a <= 7;
}
template <bool W24>
__host__ __device__ constexpr int plan_npass(int n) {
  const int a = count2(n), b = count3(n >> a);
  if (W24 && plan_has24(n)) return a == 3 ? 1 : 2;
  return a / 4 + (a % 4 != 0 ? 1 : 0) + b;
}
template <bool W24>
__host__ __device__ constexpr int plan_radix(int n, int p) {
  const int a = count2(n);
  if (W24 && plan_has24(n)) return (a == 3 || p == 1) ? 24 : (1 << (a - 3));
  if (p < a / 4) return 16;
  p -= a / 4;
  if (a % 4 != 0) {
    if (p == 0) return a % 4 == 3 ? 8 : (a % 4 == 2 ? 4 : 2);
    p -= 1;
  }
  return 3;
}

// Shared-memory index of element e0 + r*stride of a line when e0 >= 0 and
// stride is a multiple of the padding period P = 2^pad_shift: padi(e0) plus
// the constant r*(stride + stride/P), so that all R accesses of a butterfly
// are one base register plus immediate offsets.
template <class V, int STRIDE>
__device__ __forceinline__ constexpr bool pad_linear() {
  return STRIDE % (1 << pad_shift<V>()) == 0;
}

template <int R, bool INV, int N, int NS, class V>
__device__ __forceinline__ void fft_pass_t(const V *__restrict__ src, V *__restrict__ dst, int nl,
                                           const V *__restrict__ tw) {
  constexpr int nb = N / R, LS = line_stride<V>(N), tws = N / (NS * R);
  constexpr int P = 1 << pad_shift<V>();
  const int tot = nl * nb;
  for (int b = threadIdx.x; b < tot; b += blockDim.x) {
    const int l = b / nb;
    const int j = b - l * nb;
    const V *s = src + l * LS;
    V *d = dst + l * LS;
    const int jm = j % NS;
    V v[R];
    if constexpr (pad_linear<V, nb>()) {
      const V *sb = s + padi<V>(j);
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = sb[r * (nb + nb / P)];
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = s[padi<V>(j + r * nb)];
    }
    if (NS > 1 && jm != 0) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        const V w = __ldg(tw + r * jm * tws);
        v[r] = INV ? cmulc(v[r], w) : cmul(v[r], w);
      }
    }
    Dft<R, INV>::run(v);
    if constexpr (pad_linear<V, NS>()) {
      V *db = d + padi<V>((j / NS) * NS * R + jm);
#pragma unroll
      for (int r = 0; r < R; ++r) db[r * (NS + NS / P)] = v[r];
    } else if constexpr (NS == 1 && R % P == 0) {
      // first pass: idxD = j*R, a multiple of P; offsets r < R
      V *db = d + j * (R + R / P);
#pragma unroll
      for (int r = 0; r < R; ++r) db[r + r / P] = v[r];
    } else {
      const int idxD = (j / NS) * NS * R + jm;
#pragma unroll
      for (int r = 0; r < R; ++r) d[padi<V>(idxD + r * NS)] = v[r];
    }
  }
}

template <int N, int NS, int P, bool INV, int PL, class V>
__device__ __forceinline__ void passes_t(V *&A, V *&B, int nl, const V *__restrict__ tw) {
  constexpr bool W24 = PL == 1;
  if constexpr (P < plan_npass<W24>(N)) {
    constexpr int R = plan_radix<W24>(N, P);
    fft_pass_t<R, INV, N, NS>(A, B, nl, tw);
    __syncthreads();
    V *t = A;
    A = B;
    B = t;
    passes_t<N, NS * R, P + 1, INV, PL>(A, B, nl, tw);
  }
}

// Complex FFT of nl lines held in A (compile-time plan of family PL for
// N > 0).
template <int N, bool INV, int PL, class V>
__device__ __forceinline__ V *fft_run_n(V *A, V *B, int nl, int LS, const FftDev<V> &P) {
  if constexpr (N > 0) {
    passes_t<N, 1, 0, INV, PL>(A, B, nl, P.tw);
    return A;
  } else {
    return fft_run<INV>(A, B, nl, LS, P);
  }
}

// The four packed outputs owned by the conjugate pair (m, n-m), 0 <= m < n/2:
// packed indices q0 = 2m and q1 = 2m+1 (q0 = 0 and q1 = 1 for m = 0, i.e.
// X_0 and X_{n/2}), for the sequence a (real parts) and b (imaginary parts).
// A_m = (Z_m + conj Z_{n-m})/2, B_m = (Z_m - conj Z_{n-m})/(2i).
template <class V>
__device__ __forceinline__ void unpack_four(const V *Z, int n, int m, V &a, V &b) {
  using S = ScalarOf<V>;
  const S half = S(0.5);
  if (m == 0) {
    const V z0 = Z[0], zh = Z[padi<V>(n >> 1)];
    a = mk<V>((z0.x + z0.x) * half, (zh.x + zh.x) * half);
    b = mk<V>((z0.y + z0.y) * half, (zh.y + zh.y) * half);
  } else {
    const V zm = Z[padi<V>(m)], zc = Z[padi<V>(n - m)];
    a = mk<V>((zm.x + zc.x) * half, (zm.y - zc.y) * half);
    b = mk<V>((zm.y + zc.y) * half, (zc.x - zm.x) * half);
  }
}

// Builds Z_m and Z_{n-m} (0 <= m <= n/2) of the pair whose packed spectra are
// those of the real sequences a and b (Z = A + iB), reading them with vector
// loads.  Rows: the packed spectra of a and b lie in rows ra and rb, (Re, Im)
// of mode m adjacent at 2m (x lines: one load gives Re and Im).  Columns: a
// and b are adjacent columns, element k of both at ab[k*st] (y lines: one
// load gives a and b).
template <class V>
__device__ __forceinline__ void pack_pair_rows(V *Z, int n, int m, const ScalarOf<V> *ra,
                                               const ScalarOf<V> *rb) {
  using S = ScalarOf<V>;
  S reA, imA, reB, imB;
  if (m == 0) {
    reA = ra[0];
    reB = rb[0];
    imA = imB = S(0);
  } else if (m == (n >> 1)) {
    reA = ra[1];
    reB = rb[1];
    imA = imB = S(0);
  } else {
    const V a = reinterpret_cast<const V *>(ra)[m], b = reinterpret_cast<const V *>(rb)[m];
    reA = a.x;
    imA = a.y;
    reB = b.x;
    imB = b.y;
  }
  Z[padi<V>(m)] = mk<V>(reA - imB, imA + reB);
  if (m != 0 && m != (n >> 1)) Z[padi<V>(n - m)] = mk<V>(reA + imB, reB - imA);
}
// The column form with scalar loads: element k of a at ab[k * st], of b at
// ab[k * st + 1].
template <class V>
__device__ __forceinline__ void pack_pair_cols_scalar(V *Z, int n, int m,
                                                      const ScalarOf<V> *ab, int st) {
  using S = ScalarOf<V>;
  S reA, imA, reB, imB;
  if (m == 0) {
    reA = ab[0];
    reB = ab[1];
    imA = imB = S(0);
  } else if (m == (n >> 1)) {
    reA = ab[st];
    reB = ab[st + 1];
    imA = imB = S(0);
  } else {
    reA = ab[(2 * m) * st];
    reB = ab[(2 * m) * st + 1];
    imA = ab[(2 * m + 1) * st];
    imB = ab[(2 * m + 1) * st + 1];
  }
  Z[padi<V>(m)] = mk<V>(reA - imB, imA + reB);
  if (m != 0 && m != (n >> 1)) Z[padi<V>(n - m)] = mk<V>(reA + imB, reB - imA);
}
template <class V>
__device__ __forceinline__ void pack_pair_cols(V *Z, int n, int m, const V *ab, int st) {
  using S = ScalarOf<V>;
  S reA, imA, reB, imB;
  if (m == 0) {
    const V r = ab[0];
    reA = r.x;
    reB = r.y;
    imA = imB = S(0);
  } else if (m == (n >> 1)) {
    const V r = ab[st];
    reA = r.x;
    reB = r.y;
    imA = imB = S(0);
  } else {
    const V re = ab[(2 * m) * st], im = ab[(2 * m + 1) * st];
    reA = re.x;
    reB = re.y;
    imA = im.x;
    imB = im.y;
  }
  Z[padi<V>(m)] = mk<V>(reA - imB, imA + reB);
  if (m != 0 && m != (n >> 1)) Z[padi<V>(n - m)] = mk<V>(reA + imB, reB - imA);
}

// div(u)/dt at halo'd index c exactly as calcRHS evaluates it
// (mod_calcRHS.cc:27-29), every operation rounded separately (no contraction)
// so that the value is bit-identical to the reference expression.
__device__ __forceinline__ double div_dt(const double *__restrict__ u,
                                         const double *__restrict__ v,
                                         const double *__restrict__ w, long long c, int X,
                                         long long XY, double dtidxi, double dtidyi, double dti,
                                         double dzfi) {
  const double tx = __dmul_rn(__dsub_rn(u[c], u[c - 1]), dtidxi);
  const double ty = __dmul_rn(__dsub_rn(v[c], v[c - X]), dtidyi);
  const double tz = __dmul_rn(__dmul_rn(__dsub_rn(w[c], w[c - XY]), dti), dzfi);
  return __dadd_rn(__dadd_rn(tx, ty), tz);
}
// the mixed form: FP32 operands and arithmetic
__device__ __forceinline__ float div_dt(const float *__restrict__ u, const float *__restrict__ v,
                                        const float *__restrict__ w, long long c, int X,
                                        long long XY, float dtidxi, float dtidyi, float dti,
                                        float dzfi) {
  return (u[c] - u[c - 1]) * dtidxi + (v[c] - v[c - X]) * dtidyi + (w[c] - w[c - XY]) * (dti * dzfi);
}

// Forward x transform fused with calcRHS, one tile per block: rows
// (j0+2l, j0+2l+1) of plane k are div(u)/dt evaluated from global memory while
// loading (many resident blocks hide the load latency), then transformed.
template <class T, int N, bool FUSED, int PL>
__global__ void __launch_bounds__(256) k_fft_x_fwd_div(Geo g, FftDev<typename Cx<T>::V> P, int nl,
                                                       const StepConst *__restrict__ sc,
                                                       const T *__restrict__ p,
                                                       const T *__restrict__ u,
                                                       const T *__restrict__ v,
                                                       const T *__restrict__ w,
                                                       T *__restrict__ var) {
  using V = typename Cx<T>::V;
  extern __shared__ __align__(16) unsigned char fft_smem[];
  V *smem = reinterpret_cast<V *>(fft_smem);
  const int n = N > 0 ? N : g.nx, LS = line_stride<V>(n);
  V *A = smem, *B = smem + nl * LS;
  const int j0 = blockIdx.x * 2 * nl;  // 0-based row in the plane
  const int k = blockIdx.y;            // 0-based plane
  T dti = 0, dtidxi = 0, dtidyi = 0, dzfi = 0;
  if (FUSED) {
    dti = T(sc->dti);
    dtidxi = T(sc->dtidxi);
    dtidyi = T(sc->dtidyi);
    dzfi = T(__ldg(g.dzf_inv + k + 1));
  }
  for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
    const int l = e / n, t = e - l * n;
    const long long ca = g.at(t + 1, j0 + 2 * l + 1, k + 1);
    const long long cb = ca + g.X;
    T a, b;
    if (FUSED) {
      a = div_dt(u, v, w, ca, g.X, g.XY, dtidxi, dtidyi, dti, dzfi);
      b = div_dt(u, v, w, cb, g.X, g.XY, dtidxi, dtidyi, dti, dzfi);
    } else {
      a = p[ca];
      b = p[cb];
    }
    A[l * LS + padi<V>(t)] = mk<V>(a, b);
  }
  __syncthreads();
  const V *Z = fft_run_n<N, false, PL>(A, B, nl, LS, P);
  const int half = n >> 1;
  for (int e = threadIdx.x; e < nl * half; e += blockDim.x) {
    const int l = e / half, m = e - l * half;
    V a, b;
    unpack_four(Z + l * LS, n, m, a, b);
    const long long row = (long long)k * g.ny + j0 + 2 * l;
    reinterpret_cast<V *>(var + row * n)[m] = a;
    reinterpret_cast<V *>(var + (row + 1) * n)[m] = b;
  }
}

// The same for one block of a batched launch over several channels (the
// block's coordinates from the work list).  The single-channel kernel keeps
// its own copy of these lines: a body shared between the two changed the
// single-channel kernel's code generation and made it slower.
template <class T, int N, bool FUSED, int PL>
__device__ __forceinline__ void fft_x_fwd_div_body(Geo g, FftDev<typename Cx<T>::V> P,
                                                   int nl, const StepConst *__restrict__ sc,
                                                   const T *__restrict__ p,
                                                   const T *__restrict__ u,
                                                   const T *__restrict__ v,
                                                   const T *__restrict__ w,
                                                   T *__restrict__ var, VBlk vb) {
  using V = typename Cx<T>::V;
  extern __shared__ __align__(16) unsigned char fft_smem[];
  V *smem = reinterpret_cast<V *>(fft_smem);
  const int n = N > 0 ? N : g.nx, LS = line_stride<V>(n);
  V *A = smem, *B = smem + nl * LS;
  const int j0 = vb.x() * 2 * nl;  // 0-based row in the plane
  const int k = vb.y();            // 0-based plane
  T dti = 0, dtidxi = 0, dtidyi = 0, dzfi = 0;
  if (FUSED) {
    dti = T(sc->dti);
    dtidxi = T(sc->dtidxi);
    dtidyi = T(sc->dtidyi);
    dzfi = T(__ldg(g.dzf_inv + k + 1));
  }
  for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
    const int l = e / n, t = e - l * n;
    const long long ca = g.at(t + 1, j0 + 2 * l + 1, k + 1);
    const long long cb = ca + g.X;
    T a, b;
    if (FUSED) {
      a = div_dt(u, v, w, ca, g.X, g.XY, dtidxi, dtidyi, dti, dzfi);
      b = div_dt(u, v, w, cb, g.X, g.XY, dtidxi, dtidyi, dti, dzfi);
    } else {
      a = p[ca];
      b = p[cb];
    }
    A[l * LS + padi<V>(t)] = mk<V>(a, b);
  }
  __syncthreads();
  const V *Z = fft_run_n<N, false, PL>(A, B, nl, LS, P);
  const int half = n >> 1;
  for (int e = threadIdx.x; e < nl * half; e += blockDim.x) {
    const int l = e / half, m = e - l * half;
    V a, b;
    unpack_four(Z + l * LS, n, m, a, b);
    const long long row = (long long)k * g.ny + j0 + 2 * l;
    reinterpret_cast<V *>(var + row * n)[m] = a;
    reinterpret_cast<V *>(var + (row + 1) * n)[m] = b;
  }
}

// ---------------------------------------------------------------------------
// Persistent transform kernels.  Each block takes tiles t = blockIdx.x,
// blockIdx.x + gridDim.x, ...; the raw rows of the next tile are copied into
// a staging buffer S with cp.async (16-byte chunks, L2 only) as soon as the
// current tile has been packed into the FFT buffers, so the copy overlaps the
// radix passes and the stores of the current tile.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                   static_cast<unsigned>(__cvta_generic_to_shared(smem))),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// Copies `rows` rows of `len` elements (len a multiple of 16 bytes, 16-byte
// aligned rows) from src (row stride `stride` elements) to dst (row stride
// `len`); fcpr divides by the chunks per row, len / (16 / sizeof(T)).
template <class T>
__device__ __forceinline__ void stage_rows(T *dst, const T *src, int rows, int len,
                                           long long stride, const FastDiv &fcpr) {
  constexpr int per = 16 / sizeof(T);  // elements per 16-byte chunk
  const int cpr = len / per;           // chunks per row
  for (int e = threadIdx.x; e < rows * cpr; e += blockDim.x) {
    const int r = fcpr.div(e), ch = e - r * cpr;
    cp_async16(dst + r * len + per * ch, src + r * stride + per * ch);
  }
}

// Forward x transform (persistent): rows (j0+2l, j0+2l+1) of p at plane k ->
// packed spectra.  The halo'd rows are staged whole (16-byte aligned).
template <class T, int N, int PL>
__global__ void __launch_bounds__(128) k_fft_x_fwd(Geo g, FftDev<typename Cx<T>::V> P, int nl,
                                                   const T *__restrict__ p, T *__restrict__ var) {
  using V = typename Cx<T>::V;
  extern __shared__ __align__(16) unsigned char fft_smem[];
  V *smem = reinterpret_cast<V *>(fft_smem);
  const int n = N > 0 ? N : g.nx, LS = line_stride<V>(n), X = g.X, R = 2 * nl;
  V *A = smem, *B = smem + nl * LS;
  T *S = reinterpret_cast<T *>(B + nl * LS);  // R halo'd rows
  const int tiles_y = g.ny / R;
  const int ntiles = tiles_y * g.nz;
  const FastDiv fcpr(X / (16 / sizeof(T)));
  auto issue = [&](int tile) {
    const int j0 = (tile % tiles_y) * R, k = tile / tiles_y;  // 0-based
    stage_rows(S, p + g.at(0, j0 + 1, k + 1), R, X, X, fcpr);
    cp_async_commit();
  };
  int tile = blockIdx.x;
  if (tile < ntiles) issue(tile);
  for (; tile < ntiles; tile += gridDim.x) {
    const int j0 = (tile % tiles_y) * R, k = tile / tiles_y;
    cp_async_wait_all();
    __syncthreads();
    for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
      const int l = e / n, t = e - l * n;
      A[l * LS + padi<V>(t)] = mk<V>(S[(2 * l) * X + t + 1], S[(2 * l + 1) * X + t + 1]);
    }
    __syncthreads();
    if (tile + (int)gridDim.x < ntiles) issue(tile + gridDim.x);
    const V *Z = fft_run_n<N, false, PL>(A, B, nl, LS, P);
    const int half = n >> 1;
    for (int e = threadIdx.x; e < nl * half; e += blockDim.x) {
      const int l = e / half, m = e - l * half;
      V a, b;
      unpack_four(Z + l * LS, n, m, a, b);
      const long long row = (long long)k * g.ny + j0 + 2 * l;
      reinterpret_cast<V *>(var + row * n)[m] = a;
      reinterpret_cast<V *>(var + (row + 1) * n)[m] = b;
    }
  }
}

// Backward x transform: packed spectra -> p interior scaled by nf; with
// FUSE_BC the pressure halos are written as well (updateBoundP).
template <class T, int N, bool FUSE_BC, int PL>
__global__ void __launch_bounds__(128) k_fft_x_bwd(Geo g, FftDev<typename Cx<T>::V> P, int nl,
                                                   double nf, const T *__restrict__ var, T *p,
                                                   int rev) {
  using V = typename Cx<T>::V;
  extern __shared__ __align__(16) unsigned char fft_smem[];
  V *smem = reinterpret_cast<V *>(fft_smem);
  const int n = N > 0 ? N : g.nx, LS = line_stride<V>(n), R = 2 * nl;
  V *A = smem, *B = smem + nl * LS;
  T *S = reinterpret_cast<T *>(B + nl * LS);  // R rows of n elements
  const int tiles_y = g.ny / R;
  const int ntiles = tiles_y * g.nz;
  const T scale = T(nf);
  const FastDiv fcpr(n / (16 / sizeof(T)));
  auto issue = [&](int tile) {
    const int tt = rev ? ntiles - 1 - tile : tile;  // plane order
    const int j0 = (tt % tiles_y) * R, k = tt / tiles_y;
    stage_rows(S, var + ((long long)k * g.ny + j0) * n, R, n, n, fcpr);
    cp_async_commit();
  };
  int tile = blockIdx.x;
  if (tile < ntiles) issue(tile);
  const int half = n >> 1;
  for (; tile < ntiles; tile += gridDim.x) {
    const int tt = rev ? ntiles - 1 - tile : tile;
    const int j0 = (tt % tiles_y) * R, k = tt / tiles_y;
    cp_async_wait_all();
    __syncthreads();
    for (int e = threadIdx.x; e < nl * (half + 1); e += blockDim.x) {
      const int l = e / (half + 1), m = e - l * (half + 1);
      pack_pair_rows(A + l * LS, n, m, S + (2 * l) * n, S + (2 * l + 1) * n);
    }
    __syncthreads();
    if (tile + (int)gridDim.x < ntiles) issue(tile + gridDim.x);
    V *Z = fft_run_n<N, true, PL>(A, B, nl, LS, P);
    // rows j = j0 + 2l + 1 (a) and j + 1 (b) of plane k + 1
    const int kk = k + 1;
    // FP32 with the pressure halos (updateBoundP) and rows shorter than a
    // line of the FFT buffer the last pass left free (n >= 64): the scaled
    // rows are laid out whole there -- x images and row padding included --
    // then stored as float4, each row once more to its y image row and z
    // ghost plane where it has one.  Rows start on 16-byte boundaries (the
    // pitch is a multiple of 4); the free buffer's start is rounded up to 16
    // bytes (it is 8-byte aligned), which the slack of at least 2*nl elements
    // covers.  (The FP64 kernel measured slower this way, 0.58 against 0.46 ms
    // at 768 x 384 x 256: it keeps the element loop below.)
    if (FUSE_BC && sizeof(T) == 4 && g.X < LS &&
        (reinterpret_cast<unsigned long long>(p) & 15ull) == 0) {
      using T16 = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
      constexpr int VW = 16 / sizeof(T);
      const int X = g.X, nq = X / VW;
      const FastDiv fnq(nq);
      // line l: rows a, b at 2*l*X
      T *O = reinterpret_cast<T *>(
          (reinterpret_cast<unsigned long long>(Z == A ? B : A) + 15ull) & ~15ull);
      for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
        const int l = e / n, t = e - l * n;
        const V z = Z[l * LS + padi<V>(t)];
        T *oa = O + 2 * l * X, *ob = oa + X;
        const T a = scale * z.x, b = scale * z.y;
        oa[t + 1] = a;
        ob[t + 1] = b;
        if (t == 0) {  // x image of i = 1
          oa[n + 1] = a;
          ob[n + 1] = b;
        }
        if (t == n - 1) {  // x image of i = n
          oa[0] = a;
          ob[0] = b;
        }
      }
      for (int e = threadIdx.x; e < nl * 2 * (X - n - 2); e += blockDim.x) {
        const int r = e / (X - n - 2);  // row padding
        O[r * X + n + 2 + (e - r * (X - n - 2))] = T(0);
      }
      __syncthreads();
      const int kimg = kk == 1 ? 0 : (kk == g.nz ? g.nz + 1 : -1);
      for (int e = threadIdx.x; e < 2 * nl * nq; e += blockDim.x) {
        const int r = fnq.div(e), q = e - r * nq;  // r = 2l + h
        const T16 val = reinterpret_cast<const T16 *>(O + r * X)[q];
        const int j = j0 + r + 1;
        const int jimg = j == g.ny ? 0 : (j == 1 ? g.ny + 1 : -1);
        auto row = [&](int jj, int kq) {
          reinterpret_cast<T16 *>(p + (long long)jj * X + (long long)kq * g.XY)[q] = val;
        };
        row(j, kk);
        if (jimg >= 0) row(jimg, kk);
        if (kimg >= 0) {
          row(j, kimg);
          if (jimg >= 0) row(jimg, kimg);
        }
      }
    } else {
      // element by element; with FUSE_BC also the periodic images (x ends of
      // each row, the y image row) and the zero-gradient ghost plane, decided
      // per row
      const int kimg = !FUSE_BC ? -1 : (kk == 1 ? 0 : (kk == g.nz ? g.nz + 1 : -1));
      for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
        const int l = e / n, t = e - l * n;
        const V z = Z[l * LS + padi<V>(t)];
        const T ab[2] = {scale * z.x, scale * z.y};
        const int i = t + 1;
        const int iimg = !FUSE_BC ? -1 : (i == g.nx ? 0 : (i == 1 ? g.nx + 1 : -1));
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int j = j0 + 2 * l + 1 + h;
          const int jimg = !FUSE_BC ? -1 : (j == g.ny ? 0 : (j == 1 ? g.ny + 1 : -1));
          const T v = ab[h];
          auto row = [&](int jj, int kq) {
            T *r = p + (long long)jj * g.X + (long long)kq * g.XY;
            r[i] = v;
            if (iimg >= 0) r[iimg] = v;
          };
          row(j, kk);
          if (jimg >= 0) row(jimg, kk);
          if (kimg >= 0) {
            row(j, kimg);
            if (jimg >= 0) row(jimg, kimg);
          }
        }
      }
    }
  }
}

// The same for one block of a batched launch over several channels (the
// block's coordinates from the work list).  The single-channel kernel keeps
// its own copy of these lines: a body shared between the two changed the
// single-channel kernel's code generation and made it slower.
template <class T, int N, bool FUSE_BC, int PL>
__device__ __forceinline__ void fft_x_bwd_body(Geo g, FftDev<typename Cx<T>::V> P,
                                               int nl, double nf, const T *__restrict__ var, T *p,
                                               int rev, VBlk vb) {
  using V = typename Cx<T>::V;
  extern __shared__ __align__(16) unsigned char fft_smem[];
  V *smem = reinterpret_cast<V *>(fft_smem);
  const int n = N > 0 ? N : g.nx, LS = line_stride<V>(n), R = 2 * nl;
  V *A = smem, *B = smem + nl * LS;
  T *S = reinterpret_cast<T *>(B + nl * LS);  // R rows of n elements
  const int tiles_y = g.ny / R;
  const int ntiles = tiles_y * g.nz;
  const T scale = T(nf);
  const FastDiv fcpr(n / (16 / sizeof(T)));
  auto issue = [&](int tile) {
    const int tt = rev ? ntiles - 1 - tile : tile;  // plane order
    const int j0 = (tt % tiles_y) * R, k = tt / tiles_y;
    stage_rows(S, var + ((long long)k * g.ny + j0) * n, R, n, n, fcpr);
    cp_async_commit();
  };
  int tile = vb.x();
  if (tile < ntiles) issue(tile);
  const int half = n >> 1;
  for (; tile < ntiles; tile += vb.gx()) {
    const int tt = rev ? ntiles - 1 - tile : tile;
    const int j0 = (tt % tiles_y) * R, k = tt / tiles_y;
    cp_async_wait_all();
    __syncthreads();
    for (int e = threadIdx.x; e < nl * (half + 1); e += blockDim.x) {
      const int l = e / (half + 1), m = e - l * (half + 1);
      pack_pair_rows(A + l * LS, n, m, S + (2 * l) * n, S + (2 * l + 1) * n);
    }
    __syncthreads();
    if (tile + vb.gx() < ntiles) issue(tile + vb.gx());
    V *Z = fft_run_n<N, true, PL>(A, B, nl, LS, P);
    // rows j = j0 + 2l + 1 (a) and j + 1 (b) of plane k + 1
    const int kk = k + 1;
    // FP32 with the pressure halos (updateBoundP) and rows shorter than a
    // line of the FFT buffer the last pass left free (n >= 64): the scaled
    // rows are laid out whole there -- x images and row padding included --
    // then stored as float4, each row once more to its y image row and z
    // ghost plane where it has one.  Rows start on 16-byte boundaries (the
    // pitch is a multiple of 4); the free buffer's start is rounded up to 16
    // bytes (it is 8-byte aligned), which the slack of at least 2*nl elements
    // covers.  (The FP64 kernel measured slower this way, 0.58 against 0.46 ms
    // at 768 x 384 x 256: it keeps the element loop below.)
    if (FUSE_BC && sizeof(T) == 4 && g.X < LS &&
        (reinterpret_cast<unsigned long long>(p) & 15ull) == 0) {
      using T16 = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
      constexpr int VW = 16 / sizeof(T);
      const int X = g.X, nq = X / VW;
      const FastDiv fnq(nq);
      // line l: rows a, b at 2*l*X
      T *O = reinterpret_cast<T *>(
          (reinterpret_cast<unsigned long long>(Z == A ? B : A) + 15ull) & ~15ull);
      for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
        const int l = e / n, t = e - l * n;
        const V z = Z[l * LS + padi<V>(t)];
        T *oa = O + 2 * l * X, *ob = oa + X;
        const T a = scale * z.x, b = scale * z.y;
        oa[t + 1] = a;
        ob[t + 1] = b;
        if (t == 0) {  // x image of i = 1
          oa[n + 1] = a;
          ob[n + 1] = b;
        }
        if (t == n - 1) {  // x image of i = n
          oa[0] = a;
          ob[0] = b;
        }
      }
      for (int e = threadIdx.x; e < nl * 2 * (X - n - 2); e += blockDim.x) {
        const int r = e / (X - n - 2);  // row padding
        O[r * X + n + 2 + (e - r * (X - n - 2))] = T(0);
      }
      __syncthreads();
      const int kimg = kk == 1 ? 0 : (kk == g.nz ? g.nz + 1 : -1);
      for (int e = threadIdx.x; e < 2 * nl * nq; e += blockDim.x) {
        const int r = fnq.div(e), q = e - r * nq;  // r = 2l + h
        const T16 val = reinterpret_cast<const T16 *>(O + r * X)[q];
        const int j = j0 + r + 1;
        const int jimg = j == g.ny ? 0 : (j == 1 ? g.ny + 1 : -1);
        auto row = [&](int jj, int kq) {
          reinterpret_cast<T16 *>(p + (long long)jj * X + (long long)kq * g.XY)[q] = val;
        };
        row(j, kk);
        if (jimg >= 0) row(jimg, kk);
        if (kimg >= 0) {
          row(j, kimg);
          if (jimg >= 0) row(jimg, kimg);
        }
      }
    } else {
      // element by element; with FUSE_BC also the periodic images (x ends of
      // each row, the y image row) and the zero-gradient ghost plane, decided
      // per row
      const int kimg = !FUSE_BC ? -1 : (kk == 1 ? 0 : (kk == g.nz ? g.nz + 1 : -1));
      for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
        const int l = e / n, t = e - l * n;
        const V z = Z[l * LS + padi<V>(t)];
        const T ab[2] = {scale * z.x, scale * z.y};
        const int i = t + 1;
        const int iimg = !FUSE_BC ? -1 : (i == g.nx ? 0 : (i == 1 ? g.nx + 1 : -1));
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int j = j0 + 2 * l + 1 + h;
          const int jimg = !FUSE_BC ? -1 : (j == g.ny ? 0 : (j == 1 ? g.ny + 1 : -1));
          const T v = ab[h];
          auto row = [&](int jj, int kq) {
            T *r = p + (long long)jj * g.X + (long long)kq * g.XY;
            r[i] = v;
            if (iimg >= 0) r[iimg] = v;
          };
          row(j, kk);
          if (jimg >= 0) row(jimg, kk);
          if (kimg >= 0) {
            row(j, kimg);
            if (jimg >= 0) row(jimg, kimg);
          }
        }
      }
    }
  }
}

// y transform in place on the spectral array: tile = columns i0..i0+2nl-1 of
// plane k (TX = 2nl x-contiguous elements per row, row stride nx).
template <class T, int N, bool INV, int PL>
__global__ void __launch_bounds__(256) k_fft_y(int nx, int ny, int nz,
                                               FftDev<typename Cx<T>::V> P, int nl,
                                               T *__restrict__ var, int rev) {
  using V = typename Cx<T>::V;
  extern __shared__ __align__(16) unsigned char fft_smem[];
  V *smem = reinterpret_cast<V *>(fft_smem);
  const int n = N > 0 ? N : ny, LS = line_stride<V>(n), TX = 2 * nl;
  V *A = smem, *B = smem + nl * LS;
  T *S = reinterpret_cast<T *>(B + nl * LS);  // n rows of TX elements
  const int tiles_x = nx / TX;
  const int ntiles = tiles_x * nz;
  const FastDiv fcpr(TX / (16 / sizeof(T))), fnl(nl);
  auto issue = [&](int tile) {
    const int tt = rev ? ntiles - 1 - tile : tile;  // plane order
    const int i0 = (tt % tiles_x) * TX, k = tt / tiles_x;
    stage_rows(S, var + (long long)k * nx * ny + i0, n, TX, nx, fcpr);
    cp_async_commit();
  };
  int tile = blockIdx.x;
  if (tile < ntiles) issue(tile);
  const int half = n >> 1;
  for (; tile < ntiles; tile += gridDim.x) {
    const int tt = rev ? ntiles - 1 - tile : tile;
    const int i0 = (tt % tiles_x) * TX, k = tt / tiles_x;
    T *plane = var + (long long)k * nx * ny + i0;
    cp_async_wait_all();
    __syncthreads();
    if (!INV) {
      // columns 2l, 2l+1 of row t form element t of line l: one vector
      // load and store per pair
      for (int e = threadIdx.x; e < n * nl; e += blockDim.x) {
        const int t = fnl.div(e), l = e - t * nl;
        A[l * LS + padi<V>(t)] = reinterpret_cast<const V *>(S + t * TX)[l];
      }
    } else {
      // consecutive threads take consecutive column pairs l: their reads of
      // the staged rows are adjacent (a stride of 2*TX elements between
      // threads would put every lane in one bank)
      for (int e = threadIdx.x; e < nl * (half + 1); e += blockDim.x) {
        const int m = fnl.div(e), l = e - m * nl;
        if constexpr (sizeof(T) == 4)
          pack_pair_cols(A + l * LS, n, m, reinterpret_cast<const V *>(S) + l, nl);
        else  // FP64: scalar loads (16-byte ones measured 3% slower)
          pack_pair_cols_scalar(A + l * LS, n, m, S + 2 * l, TX);
      }
    }
    __syncthreads();
    if (tile + (int)gridDim.x < ntiles) issue(tile + gridDim.x);
    const V *Z = fft_run_n<N, INV, PL>(A, B, nl, LS, P);
    if (!INV) {
      for (int e = threadIdx.x; e < half * nl; e += blockDim.x) {
        const int m = fnl.div(e), l = e - m * nl;
        V a, b;
        unpack_four(Z + l * LS, n, m, a, b);
        const int q0 = (m == 0) ? 0 : 2 * m;
        // row q0: (A, B) of columns 2l, 2l+1; row q0+1 likewise
        reinterpret_cast<V *>(plane + (long long)q0 * nx)[l] = mk<V>(a.x, b.x);
        reinterpret_cast<V *>(plane + (long long)(q0 + 1) * nx)[l] = mk<V>(a.y, b.y);
      }
    } else {
      for (int e = threadIdx.x; e < n * nl; e += blockDim.x) {
        const int t = fnl.div(e), l = e - t * nl;
        reinterpret_cast<V *>(plane + (long long)t * nx)[l] = Z[l * LS + padi<V>(t)];
      }
    }
  }
}

// The same for one block of a batched launch over several channels (the
// block's coordinates from the work list).  The single-channel kernel keeps
// its own copy of these lines: a body shared between the two changed the
// single-channel kernel's code generation and made it slower.
template <class T, int N, bool INV, int PL>
__device__ __forceinline__ void fft_y_body(int nx, int ny, int nz,
                                           FftDev<typename Cx<T>::V> P, int nl,
                                           T *__restrict__ var, int rev, VBlk vb) {
  using V = typename Cx<T>::V;
  extern __shared__ __align__(16) unsigned char fft_smem[];
  V *smem = reinterpret_cast<V *>(fft_smem);
  const int n = N > 0 ? N : ny, LS = line_stride<V>(n), TX = 2 * nl;
  V *A = smem, *B = smem + nl * LS;
  T *S = reinterpret_cast<T *>(B + nl * LS);  // n rows of TX elements
  const int tiles_x = nx / TX;
  const int ntiles = tiles_x * nz;
  const FastDiv fcpr(TX / (16 / sizeof(T))), fnl(nl);
  auto issue = [&](int tile) {
    const int tt = rev ? ntiles - 1 - tile : tile;  // plane order
    const int i0 = (tt % tiles_x) * TX, k = tt / tiles_x;
    stage_rows(S, var + (long long)k * nx * ny + i0, n, TX, nx, fcpr);
    cp_async_commit();
  };
  int tile = vb.x();
  if (tile < ntiles) issue(tile);
  const int half = n >> 1;
  for (; tile < ntiles; tile += vb.gx()) {
    const int tt = rev ? ntiles - 1 - tile : tile;
    const int i0 = (tt % tiles_x) * TX, k = tt / tiles_x;
    T *plane = var + (long long)k * nx * ny + i0;
    cp_async_wait_all();
    __syncthreads();
    if (!INV) {
      // columns 2l, 2l+1 of row t form element t of line l: one vector
      // load and store per pair
      for (int e = threadIdx.x; e < n * nl; e += blockDim.x) {
        const int t = fnl.div(e), l = e - t * nl;
        A[l * LS + padi<V>(t)] = reinterpret_cast<const V *>(S + t * TX)[l];
      }
    } else {
      // consecutive threads take consecutive column pairs l: their reads of
      // the staged rows are adjacent (a stride of 2*TX elements between
      // threads would put every lane in one bank)
      for (int e = threadIdx.x; e < nl * (half + 1); e += blockDim.x) {
        const int m = fnl.div(e), l = e - m * nl;
        if constexpr (sizeof(T) == 4)
          pack_pair_cols(A + l * LS, n, m, reinterpret_cast<const V *>(S) + l, nl);
        else  // FP64: scalar loads (16-byte ones measured 3% slower)
          pack_pair_cols_scalar(A + l * LS, n, m, S + 2 * l, TX);
      }
    }
    __syncthreads();
    if (tile + vb.gx() < ntiles) issue(tile + vb.gx());
    const V *Z = fft_run_n<N, INV, PL>(A, B, nl, LS, P);
    if (!INV) {
      for (int e = threadIdx.x; e < half * nl; e += blockDim.x) {
        const int m = fnl.div(e), l = e - m * nl;
        V a, b;
        unpack_four(Z + l * LS, n, m, a, b);
        const int q0 = (m == 0) ? 0 : 2 * m;
        // row q0: (A, B) of columns 2l, 2l+1; row q0+1 likewise
        reinterpret_cast<V *>(plane + (long long)q0 * nx)[l] = mk<V>(a.x, b.x);
        reinterpret_cast<V *>(plane + (long long)(q0 + 1) * nx)[l] = mk<V>(a.y, b.y);
      }
    } else {
      for (int e = threadIdx.x; e < n * nl; e += blockDim.x) {
        const int t = fnl.div(e), l = e - t * nl;
        reinterpret_cast<V *>(plane + (long long)t * nx)[l] = Z[l * LS + padi<V>(t)];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Warp-line transforms (plan family 2).  A warp owns L complex lines (2L
// real lines) and transforms them with no block barrier: the first radix
// pass loads its inputs straight from global memory into registers (a
// Stockham pass of radix R reads the elements j + r N/R of a line, which are
// consecutive over the lanes), the passes in between exchange through the
// warp's own shared-memory lines under __syncwarp, and the last pass of an
// inverse transform stores its outputs (the elements j + r N/R again)
// straight to global memory; a forward transform separates the two real
// spectra from the warp's shared memory after its last pass.  The plans
// below give every lane the same number of butterflies in every pass, so
// each lane holds L N / 32 complex values throughout.
// ---------------------------------------------------------------------------

// Prime-factor (Good-Thomas) 6- and 12-point DFTs: N = 3 N2 with N2 = 2 or 4
// coprime to 3; x[(N2 n1 + 3 n2) mod N] -> 3-point DFTs over n1, then
// N2-point DFTs over n2, with no twiddles; the output of (k1, k2) is
// X[(N2 c k1 + 3 d k2) mod N], c = N2^-1 mod 3, d = 3^-1 mod N2
// (W_N^(n k) = W_3^(n1 k1) W_N2^(n2 k2) for these index maps).
template <bool INV>
struct Dft<6, INV> {
  template <class V>
  __device__ __forceinline__ static void run(V (&v)[6]) {
    // n = (2 n1 + 3 n2) mod 6, k = (4 k1 + 3 k2) mod 6
    V a[3] = {v[0], v[2], v[4]};
    V b[3] = {v[3], v[5], v[1]};
    Dft<3, INV>::run(a);
    Dft<3, INV>::run(b);
#pragma unroll
    for (int k1 = 0; k1 < 3; ++k1) {
      V t[2] = {a[k1], b[k1]};
      Dft<2, INV>::run(t);
      v[(4 * k1) % 6] = t[0];
      v[(4 * k1 + 3) % 6] = t[1];
    }
  }
};

template <bool INV>
struct Dft<12, INV> {
  template <class V>
  __device__ __forceinline__ static void run(V (&v)[12]) {
    // n = (4 n1 + 3 n2) mod 12, k = (4 k1 + 9 k2) mod 12
    V y[4][3];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
#pragma unroll
      for (int n1 = 0; n1 < 3; ++n1) y[n2][n1] = v[(4 * n1 + 3 * n2) % 12];
      Dft<3, INV>::run(y[n2]);
    }
#pragma unroll
    for (int k1 = 0; k1 < 3; ++k1) {
      V t[4] = {y[0][k1], y[1][k1], y[2][k1], y[3][k1]};
      Dft<4, INV>::run(t);
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) v[(4 * k1 + 9 * k2) % 12] = t[k2];
    }
  }
};

// Lines per group and radices of the warp-line plans (0: no plan).  A group
// of G warps owns L complex lines; the passes need not give every lane the
// same number of butterflies (the lanes past the last one idle).
__host__ __device__ constexpr int wp_base_lines(int n) {
  return (n == 768 || n == 512)               ? 1
         : (n == 384 || n == 256 || n == 192) ? 2
         : (n == 128 || n == 96 || n == 64)   ? 4
         : (n == 48 || n == 32)               ? 8
                                              : 0;
}
// warps per line group: four, so that a lane holds a quarter of L N / 32
// values and the registers leave room for more resident warps
__host__ __device__ constexpr int wp_group(int n) { return wp_base_lines(n) > 0 ? 4 : 0; }
// lines per group: the y transforms of FP32 take twice the lines, so that a
// warp's row segments span whole 32-byte sectors
__host__ __device__ constexpr int wp_lines(int n, bool f32_y) {
  return wp_base_lines(n) * (f32_y ? 2 : 1);
}
// Radices of the plans; with L lines per group of 128 lanes, the passes
// give the lanes equal shares where L N / R allows (the first pass of a
// length-768 line idles half of them, its later passes a quarter).
__host__ __device__ constexpr int wp_npass(int n, int L) {
  return L == 0 ? 0
         : (n == 768 || n == 512 || n == 384 || n == 192 || n == 96) ? 3
         : (n == 256 || n == 128 || n == 64 || n == 48 || n == 32)   ? 2
                                                                     : 0;
}
__host__ __device__ constexpr int wp_radix(int n, int L, int p) {
  return n == 768   ? (p == 0 ? 12 : 8)                    // 12 8 8
         : n == 512 ? 8                                     // 8 8 8
         : n == 384 ? (p == 0 ? 12 : (p == 1 ? 8 : 4))     // 12 8 4
         : n == 256 ? 16                                    // 16 16
         : n == 192 ? (p == 0 ? 12 : 4)                     // 12 4 4
         : n == 128 ? (p == 0 ? 8 : 16)                     // 8 16
         : n == 96  ? (p == 0 ? 12 : (p == 1 ? 4 : 2))      // 12 4 2
         : n == 64  ? 8                                     // 8 8
         : n == 48  ? (p == 0 ? 12 : 4)                     // 12 4
         : n == 32  ? (p == 0 ? 8 : 4)                      // 8 4
                    : 0;
}
__host__ __device__ constexpr bool wp_radix_ok(int r) {
  return r == 2 || r == 3 || r == 4 || r == 6 || r == 8 || r == 12 || r == 16;
}

// Butterfly b of a pass (L lines of NB butterflies): line l, butterfly j.
// LFAST puts the lines of a butterfly on adjacent lanes (the y lines, whose
// lines are adjacent columns), otherwise a line's butterflies are.
template <int L, int NB, bool LFAST>
__device__ __forceinline__ void wp_bfly(int b, int &l, int &j) {
  if constexpr (L == 1) {
    l = 0;
    j = b;
  } else if constexpr (LFAST) {
    l = b % L;
    j = b / L;
  } else {
    l = b / NB;
    j = b - l * NB;
  }
}

// Barrier of one line group (G warps): __syncwarp for one warp, else the
// named barrier 1 + grp over its 32 G threads.
template <int G>
__device__ __forceinline__ void wp_sync(int grp) {
  if constexpr (G == 1)
    __syncwarp();
  else
    asm volatile("bar.sync %0, %1;" ::"r"(1 + grp), "r"(32 * G) : "memory");
}

// One Stockham pass of radix R (NS = product of the earlier radices) over the
// group's L lines; gl is the thread's index in its group.  GIN: inputs from
// ld(l, e) instead of the shared lines; GOUT (last pass): outputs to
// st(l, e, z) instead of the shared lines.
template <int R, bool INV, int N, int L, int G, int NS, bool GIN, bool GOUT, bool LFAST, class V,
          class Ld, class St>
__device__ __forceinline__ void wp_pass(V *buf, const V *__restrict__ tw, int gl, int grp,
                                        const Ld &ld, const St &st) {
  constexpr int NB = N / R, TOT = L * NB, GT = 32 * G, T = (TOT + GT - 1) / GT;
  constexpr int LS = line_stride<V>(N), tws = N / (NS * R);
  constexpr bool FULL = TOT % GT == 0;
  constexpr bool LF = (GIN || GOUT) && LFAST;
  V v[T][R];
#pragma unroll
  for (int t = 0; t < T; ++t) {
    const int b = gl + GT * t;
    if (FULL || b < TOT) {
      int l, j;
      wp_bfly<L, NB, LF>(b, l, j);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if constexpr (GIN)
          v[t][r] = ld(l, j + r * NB);
        else
          v[t][r] = buf[l * LS + padi<V>(j + r * NB)];
      }
    }
  }
  if constexpr (!GIN) wp_sync<G>(grp);  // all reads of the lines precede the writes
#pragma unroll
  for (int t = 0; t < T; ++t) {
    const int b = gl + GT * t;
    if (FULL || b < TOT) {
      int l, j;
      wp_bfly<L, NB, LF>(b, l, j);
      const int jm = NS == 1 ? 0 : j % NS;
      if constexpr (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          const V w = __ldg(tw + r * jm * tws);
          v[t][r] = INV ? cmulc(v[t][r], w) : cmul(v[t][r], w);
        }
      }
      Dft<R, INV>::run(v[t]);
      if constexpr (GOUT) {
        // NS * R = N: output r of butterfly j is element j + r N/R
#pragma unroll
        for (int r = 0; r < R; ++r) st(l, j + r * NB, v[t][r]);
      } else {
        const int base = (j / NS) * NS * R + jm;
#pragma unroll
        for (int r = 0; r < R; ++r) buf[l * LS + padi<V>(base + r * NS)] = v[t][r];
      }
    }
  }
  if constexpr (!GOUT) wp_sync<G>(grp);
}

// The passes of the plan; GIN_FIRST: the first pass loads through ld (else
// the lines are already in the shared buffer, natural order); GOUT_LAST:
// the last pass stores through st (else to the shared buffer).
template <int N, int L, int G, int P, int NS, bool INV, bool GIN_FIRST, bool GOUT_LAST,
          bool LFAST, class V, class Ld, class St>
__device__ __forceinline__ void wp_passes(V *buf, const V *__restrict__ tw, int gl, int grp,
                                          const Ld &ld, const St &st) {
  static_assert(wp_npass(N, L) > 0, "a plan for this length");
  if constexpr (P < wp_npass(N, L)) {
    constexpr int R = wp_radix(N, L, P);
    static_assert(wp_radix_ok(R), "radix of the plan");
    constexpr bool last = P + 1 == wp_npass(N, L);
    wp_pass<R, INV, N, L, G, NS, P == 0 && GIN_FIRST, last && GOUT_LAST, LFAST>(buf, tw, gl, grp,
                                                                                ld, st);
    wp_passes<N, L, G, P + 1, NS * R, INV, GIN_FIRST, GOUT_LAST, LFAST>(buf, tw, gl, grp, ld, st);
  }
}

// line groups per block for a group count along the line-pair axis: the
// largest of 8/G, 4/G, 2/G, 1 that divides it
inline int wp_groups_per_block(int groups, int G) {
  for (int w : {8, 4, 2, 1})
    if (w % G == 0 && groups % (w / G) == 0) return w / G;
  return 1;
}

// y transform in place: group grp of block (bx, k) owns the column pairs
// c0 .. c0 + 2L - 1, c0 = (bx GPB + grp) 2L, of plane k.
template <class T, int N, bool INV>
__global__ void __launch_bounds__(256) k_wfft_y(int nx, int ny, int nz,
                                                const typename Cx<T>::V *__restrict__ tw,
                                                T *__restrict__ var, int rev) {
  using V = typename Cx<T>::V;
  using S = T;
  constexpr int G = wp_group(N), L = wp_lines(N, sizeof(T) == 4), LS = line_stride<V>(N);
  constexpr int H = N / 2;
  extern __shared__ __align__(16) unsigned char fft_smem[];
  const int gl = threadIdx.x % (32 * G), grp = threadIdx.x / (32 * G);
  const int GPB = blockDim.x / (32 * G);
  V *buf = reinterpret_cast<V *>(fft_smem) + grp * L * LS;
  const int c0 = (blockIdx.x * GPB + grp) * 2 * L;
  const int k = rev ? nz - 1 - (int)blockIdx.y : (int)blockIdx.y;
  T *plane = var + (long long)k * nx * ny + c0;
  auto nost = [](int, int, V) {};
  if (!INV) {
    // rows e of the column pair (2l, 2l+1) as one complex line a + i b
    auto ld = [&](int l, int e) -> V {
      return *reinterpret_cast<const V *>(plane + (long long)e * nx + 2 * l);
    };
    wp_passes<N, L, G, 0, 1, false, true, false, true>(buf, tw, gl, grp, ld, nost);
    // separate the spectra: row q0 gets (A, B) real parts of mode m, q0 + 1
    // the imaginary parts (mod_fft.cc:144-151, packed order)
#pragma unroll 4
    for (int b = gl; b < L * H; b += 32 * G) {
      const int l = b % L, m = b / L;
      V a, bb;
      unpack_four(buf + l * LS, N, m, a, bb);
      const int q0 = m == 0 ? 0 : 2 * m;
      *reinterpret_cast<V *>(plane + (long long)q0 * nx + 2 * l) = mk<V>(a.x, bb.x);
      *reinterpret_cast<V *>(plane + (long long)(q0 + 1) * nx + 2 * l) = mk<V>(a.y, bb.y);
    }
  } else {
    // Z_e of the pair from the packed spectra of columns 2l, 2l+1
    auto ld = [&](int l, int e) -> V {
      const int m = e <= H ? e : N - e;
      const T *col = plane + 2 * l;
      S reA, reB, imA = S(0), imB = S(0);
      if (m == 0 || m == H) {
        const V r = *reinterpret_cast<const V *>(col + (m == 0 ? 0 : nx));
        reA = r.x;
        reB = r.y;
      } else {
        const V re = *reinterpret_cast<const V *>(col + (long long)(2 * m) * nx);
        const V im = *reinterpret_cast<const V *>(col + (long long)(2 * m + 1) * nx);
        reA = re.x;
        reB = re.y;
        imA = im.x;
        imB = im.y;
      }
      return e <= H ? mk<V>(reA - imB, imA + reB) : mk<V>(reA + imB, reB - imA);
    };
    auto st = [&](int l, int e, V z) {
      *reinterpret_cast<V *>(plane + (long long)e * nx + 2 * l) = z;
    };
    wp_passes<N, L, G, 0, 1, true, true, true, true>(buf, tw, gl, grp, ld, st);
  }
}

// Forward x transform: group grp of block (bx, k) owns rows j0 .. j0 + 2L - 1,
// j0 = (bx GPB + grp) 2L (0-based), of plane k, lines (j0 + 2l, j0 + 2l + 1);
// FUSED evaluates div(u)/dt while loading (calcRHS), else reads p.
template <class T, int N, bool FUSED>
__global__ void __launch_bounds__(256) k_wfft_x_fwd(Geo g, const typename Cx<T>::V *__restrict__ tw,
                                                    const StepConst *__restrict__ sc,
                                                    const T *__restrict__ p,
                                                    const T *__restrict__ u,
                                                    const T *__restrict__ v,
                                                    const T *__restrict__ w,
                                                    T *__restrict__ var) {
  using V = typename Cx<T>::V;
  constexpr int G = wp_group(N), L = wp_lines(N, false), LS = line_stride<V>(N), H = N / 2;
  extern __shared__ __align__(16) unsigned char fft_smem[];
  const int gl = threadIdx.x % (32 * G), grp = threadIdx.x / (32 * G);
  const int GPB = blockDim.x / (32 * G);
  V *buf = reinterpret_cast<V *>(fft_smem) + grp * L * LS;
  const int j0 = (blockIdx.x * GPB + grp) * 2 * L;
  const int k = blockIdx.y;
  T dti = 0, dtidxi = 0, dtidyi = 0, dzfi = 0;
  if (FUSED) {
    dti = T(sc->dti);
    dtidxi = T(sc->dtidxi);
    dtidyi = T(sc->dtidyi);
    dzfi = T(__ldg(g.dzf_inv + k + 1));
  }
  const long long c00 = g.at(1, j0 + 1, k + 1);
  auto ld = [&](int l, int e) -> V {
    const long long ca = c00 + e + 2LL * l * g.X, cb = ca + g.X;
    if (FUSED)
      return mk<V>(div_dt(u, v, w, ca, g.X, g.XY, dtidxi, dtidyi, dti, dzfi),
                   div_dt(u, v, w, cb, g.X, g.XY, dtidxi, dtidyi, dti, dzfi));
    else
      return mk<V>(p[ca], p[cb]);
  };
  auto nost = [](int, int, V) {};
  // div(u)/dt (or p) of the group's 2L rows into the shared lines, spread
  // evenly over the group's lanes (each value costs six loads), then the
  // passes from shared memory
#pragma unroll 4
  for (int b = gl; b < L * N; b += 32 * G) {
    const int l = b / N, e = b - l * N;
    buf[l * LS + padi<V>(e)] = ld(l, e);
  }
  wp_sync<G>(grp);
  wp_passes<N, L, G, 0, 1, false, false, false, false>(buf, tw, gl, grp, ld, nost);
#pragma unroll 4
  for (int b = gl; b < L * H; b += 32 * G) {
    const int l = b / H, m = b - l * H;
    V a, bb;
    unpack_four(buf + l * LS, N, m, a, bb);
    const long long row = (long long)k * g.ny + j0 + 2 * l;
    reinterpret_cast<V *>(var + row * N)[m] = a;
    reinterpret_cast<V *>(var + (row + 1) * N)[m] = bb;
  }
}

// Backward x transform: packed spectra -> p interior scaled by nf; with
// FUSE_BC also the pressure halos (updateBoundP).
template <class T, int N, bool FUSE_BC>
__global__ void __launch_bounds__(256) k_wfft_x_bwd(Geo g, const typename Cx<T>::V *__restrict__ tw,
                                                    double nf, const T *__restrict__ var, T *p,
                                                    int rev) {
  using V = typename Cx<T>::V;
  using S = T;
  constexpr int G = wp_group(N), L = wp_lines(N, false), LS = line_stride<V>(N), H = N / 2;
  extern __shared__ __align__(16) unsigned char fft_smem[];
  const int gl = threadIdx.x % (32 * G), grp = threadIdx.x / (32 * G);
  const int GPB = blockDim.x / (32 * G);
  V *buf = reinterpret_cast<V *>(fft_smem) + grp * L * LS;
  const int j0 = (blockIdx.x * GPB + grp) * 2 * L;
  const int k = rev ? g.nz - 1 - (int)blockIdx.y : (int)blockIdx.y;
  const T scale = T(nf);
  const T *rows = var + ((long long)k * g.ny + j0) * N;
  auto ld = [&](int l, int e) -> V {
    const int m = e <= H ? e : N - e;
    const T *ra = rows + (long long)(2 * l) * N, *rb = ra + N;
    S reA, reB, imA = S(0), imB = S(0);
    if (m == 0 || m == H) {
      reA = ra[m == 0 ? 0 : 1];
      reB = rb[m == 0 ? 0 : 1];
    } else {
      const V a = reinterpret_cast<const V *>(ra)[m], b = reinterpret_cast<const V *>(rb)[m];
      reA = a.x;
      imA = a.y;
      reB = b.x;
      imB = b.y;
    }
    return e <= H ? mk<V>(reA - imB, imA + reB) : mk<V>(reA + imB, reB - imA);
  };
  const int kk = k + 1;
  const int kimg = !FUSE_BC ? -1 : (kk == 1 ? 0 : (kk == g.nz ? g.nz + 1 : -1));
  auto st = [&](int l, int e, V z) {
    const T ab[2] = {scale * z.x, scale * z.y};
    const int i = e + 1;
    const int iimg = !FUSE_BC ? -1 : (i == g.nx ? 0 : (i == 1 ? g.nx + 1 : -1));
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int j = j0 + 2 * l + 1 + h;
      const int jimg = !FUSE_BC ? -1 : (j == g.ny ? 0 : (j == 1 ? g.ny + 1 : -1));
      const T val = ab[h];
      auto row = [&](int jj, int kq) {
        T *r = p + (long long)jj * g.X + (long long)kq * g.XY;
        r[i] = val;
        if (iimg >= 0) r[iimg] = val;
      };
      row(j, kk);
      if (jimg >= 0) row(jimg, kk);
      if (kimg >= 0) {
        row(j, kimg);
        if (jimg >= 0) row(jimg, kimg);
      }
    }
  };
  wp_passes<N, L, G, 0, 1, true, true, true, false>(buf, tw, gl, grp, ld, st);
}

// ---------------------------------------------------------------------------
// Two-pass y transforms (plan family 3).  A line of length N = R1 * R2 is
// transformed as X[k1 + R1 k2] = sum_n2 W_N^(n2 k1) W_R2^(n2 k2)
// sum_n1 x[R2 n1 + n2] W_R1^(n1 k1): the first pass loads the R1 elements
// x[R2 n1 + n2] of one (line, n2) straight from global memory into
// registers, transforms them, applies the twiddles W_N^(n2 k1) and writes the
// result to shared memory; after one barrier the second pass reads the R2
// values of one (line, k1) into registers and transforms them.  The inverse
// stores its outputs from there; the forward transform writes them back to
// shared memory (every thread holds at most one second-pass task: the
// block has L R1 threads) and, after one more barrier, separates the two
// real spectra of each complex line while storing them.  A block holds
// L complex lines (2L adjacent columns of one plane): with the line index
// fastest in shared memory ([row][line]), every global access of a warp is
// two whole 128-byte row segments and every shared-memory access runs at
// full width.  Two or three barriers per tile instead of one per Stockham
// pass, and no staging buffer.
// ---------------------------------------------------------------------------
// first-pass radix R1 of the plans (0: no plan)
__host__ __device__ constexpr int y2_r1(int n) {
  return n == 384 ? 16 : n == 256 ? 16 : n == 192 ? 8 : n == 128 ? 8 : n == 96 ? 4
       : n == 64 ? 8 : n == 48 ? 4 : n == 32 ? 4 : 0;
}
// complex lines per block: two 128-byte row segments per warp access
template <class T>
__host__ __device__ constexpr int y2_lines() {
  return sizeof(T) == 4 ? 16 : 8;
}

template <class T, int N, bool INV>
__device__ __forceinline__ void fft_y2_body(int nx, int ny, int nz,
                                            const typename Cx<T>::V *__restrict__ tw,
                                            T *__restrict__ var, int rev, int tile) {
  using V = typename Cx<T>::V;
  using S = T;
  constexpr int R1 = y2_r1(N), R2 = N / R1, L = y2_lines<T>(), H = N / 2;
  extern __shared__ __align__(16) unsigned char fft_smem[];
  V *Y = reinterpret_cast<V *>(fft_smem);  // [row][line]
  const int tiles_x = nx / (2 * L);
  const int k = rev ? nz - 1 - tile / tiles_x : tile / tiles_x;
  const int i0 = (tile % tiles_x) * 2 * L;
  T *plane = var + (long long)k * nx * ny + i0;
  auto row = [&](int t) { return reinterpret_cast<V *>(plane + (long long)t * nx); };
  // pass 1: (line l, n2) tasks, R1 elements each
  for (int task = threadIdx.x; task < L * R2; task += blockDim.x) {
    const int l = task % L, n2 = task / L;
    V v[R1];
    if (!INV) {
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) v[n1] = row(R2 * n1 + n2)[l];
    } else {
      // element e of line l from the packed spectra of columns 2l, 2l+1
      // (rows 2m, 2m+1 of mode m; rows 0 and 1 the real modes 0 and N/2)
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) {
        const int e = R2 * n1 + n2;
        if (e == 0 || e == H) {
          v[n1] = row(e == 0 ? 0 : 1)[l];
        } else {
          const int m = e < H ? e : N - e;
          const V re = row(2 * m)[l], im = row(2 * m + 1)[l];
          v[n1] = e < H ? mk<V>(re.x - im.y, im.x + re.y) : mk<V>(re.x + im.y, re.y - im.x);
        }
      }
    }
    Dft<R1, INV>::run(v);
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
      V x = v[k1];
      if (k1 > 0 && n2 > 0) {
        const V w = __ldg(tw + n2 * k1);
        x = INV ? cmulc(x, w) : cmul(x, w);
      }
      Y[(k1 * R2 + n2) * L + l] = x;
    }
  }
  __syncthreads();
  // pass 2: (line l, k1) tasks, R2 elements each; at most one per thread
  const int l = threadIdx.x % L, k1 = threadIdx.x / L;
  V v[R2];
#pragma unroll
  for (int n2 = 0; n2 < R2; ++n2) v[n2] = Y[(k1 * R2 + n2) * L + l];
  Dft<R2, INV>::run(v);
  if (INV) {
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) row(k1 + R1 * k2)[l] = v[k2];
    return;
  }
  __syncthreads();
#pragma unroll
  for (int k2 = 0; k2 < R2; ++k2) Y[(k1 + R1 * k2) * L + l] = v[k2];
  __syncthreads();
  // the two real spectra A (column 2l) and B (column 2l+1) of each line:
  // rows 2m, 2m+1 hold (Re, Im) of mode m, rows 0 and 1 the real modes 0, N/2
  const S half = S(0.5);
  for (int task = threadIdx.x; task < L * H; task += blockDim.x) {
    const int ll = task % L, m = task / L;
    V a, b;
    if (m == 0) {
      const V z0 = Y[ll], zh = Y[H * L + ll];
      a = mk<V>((z0.x + z0.x) * half, (zh.x + zh.x) * half);
      b = mk<V>((z0.y + z0.y) * half, (zh.y + zh.y) * half);
    } else {
      const V zm = Y[m * L + ll], zc = Y[(N - m) * L + ll];
      a = mk<V>((zm.x + zc.x) * half, (zm.y - zc.y) * half);
      b = mk<V>((zm.y + zc.y) * half, (zc.x - zm.x) * half);
    }
    const int q0 = m == 0 ? 0 : 2 * m;
    row(q0)[ll] = mk<V>(a.x, b.x);
    row(q0 + 1)[ll] = mk<V>(a.y, b.y);
  }
}

template <class T, int N, bool INV>
__global__ void __launch_bounds__(y2_lines<T>() * y2_r1(N))
    k_fft_y2(int nx, int ny, int nz, const typename Cx<T>::V *__restrict__ tw,
             T *__restrict__ var, int rev) {
  fft_y2_body<T, N, INV>(nx, ny, nz, tw, var, rev, (int)blockIdx.x);
}

// The same over the mixed-form channels of an ensemble: block b works on
// tile b - start[m] of channel m (start[m] <= b < start[m + 1]).
struct Y2Member {
  int nx, ny, nz, rev;
  const float2 *tw;
  float *var;
};
struct Y2Batch {
  int n;
  int start[kBatchMax + 1];
  Y2Member m[kBatchMax];
};
template <int N, bool INV>
__global__ void __launch_bounds__(y2_lines<float>() * y2_r1(N))
    k_fft_y2_batch(const __grid_constant__ Y2Batch b) {
  batch_grid_sync();
  const int q = batch_member(b.start, b.n, (int)blockIdx.x);
  const Y2Member &a = b.m[q];
  fft_y2_body<float, N, INV>(a.nx, a.ny, a.nz, a.tw, a.var, a.rev, (int)blockIdx.x - b.start[q]);
}

// Two-pass x transforms (plan family 3 of the x lines).  The same two passes
// as k_fft_y2, along contiguous rows: a complex line is a pair of rows
// (j, j+1) of one plane, and a warp's tasks run along a line, so that its
// global accesses are consecutive elements of a row.  Shared memory holds
// each line's first-pass results as R1 rows of R2 + 1 elements and the
// second pass's as R2 rows of R1 + 1 (odd row lengths: the strided accesses
// of the other pass hit distinct banks).  The block has L R1 threads, one
// second-pass task each.  Lengths with R1, R2 <= 32.
__host__ __device__ constexpr int x2_r1(int n) {
  return n == 768 ? 32 : n == 512 ? 32 : n == 384 ? 16 : n == 256 ? 16 : n == 192 ? 8
       : n == 128 ? 8 : n == 96 ? 4 : n == 64 ? 8 : n == 48 ? 4 : n == 32 ? 4 : 0;
}
// line pairs (complex lines) per block: 256 threads, at most 16 lines
__host__ __device__ constexpr int x2_lines(int n) {
  return x2_r1(n) > 0 ? (256 / x2_r1(n) < 16 ? 256 / x2_r1(n) : 16) : 0;
}
__host__ __device__ constexpr int x2_line_elems(int n) {
  return x2_r1(n) > 0 ? ((x2_r1(n) * (n / x2_r1(n) + 1) > (n / x2_r1(n)) * (x2_r1(n) + 1))
                             ? x2_r1(n) * (n / x2_r1(n) + 1)
                             : (n / x2_r1(n)) * (x2_r1(n) + 1))
                      : 0;
}

// Forward: rows (j0 + 2l, j0 + 2l + 1) of plane k (div(u)/dt with FUSED, p
// otherwise) -> packed spectra.  Grid (ny / (2 L), nz).
template <class T, int N, bool FUSED>
__global__ void __launch_bounds__(x2_lines(N) * x2_r1(N))
    k_fft_x2_fwd(Geo g, const typename Cx<T>::V *__restrict__ tw, const StepConst *__restrict__ sc,
                 const T *__restrict__ p, const T *__restrict__ u, const T *__restrict__ v,
                 const T *__restrict__ w, T *__restrict__ var) {
  using V = typename Cx<T>::V;
  using S = T;
  constexpr int R1 = x2_r1(N), R2 = N / R1, L = x2_lines(N), E = x2_line_elems(N), H = N / 2;
  extern __shared__ __align__(16) unsigned char fft_smem[];
  V *buf = reinterpret_cast<V *>(fft_smem);
  const int j0 = blockIdx.x * 2 * L;  // 0-based row in the plane
  const int k = blockIdx.y;           // 0-based plane
  T dti = 0, dtidxi = 0, dtidyi = 0, dzfi = 0;
  if (FUSED) {
    dti = T(sc->dti);
    dtidxi = T(sc->dtidxi);
    dtidyi = T(sc->dtidyi);
    dzfi = T(__ldg(g.dzf_inv + k + 1));
  }
  // pass 1: (n2, line) tasks, n2 fastest
  for (int task = threadIdx.x; task < L * R2; task += blockDim.x) {
    const int n2 = task % R2, l = task / R2;
    const long long ca0 = g.at(1, j0 + 2 * l + 1, k + 1);
    V x[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) {
      const long long ca = ca0 + R2 * n1 + n2, cb = ca + g.X;
      T a, b;
      if (FUSED) {
        a = div_dt(u, v, w, ca, g.X, g.XY, dtidxi, dtidyi, dti, dzfi);
        b = div_dt(u, v, w, cb, g.X, g.XY, dtidxi, dtidyi, dti, dzfi);
      } else {
        a = p[ca];
        b = p[cb];
      }
      x[n1] = mk<V>(a, b);
    }
    Dft<R1, false>::run(x);
    V *Y = buf + l * E;
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
      V y = x[k1];
      if (k1 > 0 && n2 > 0) y = cmul(y, __ldg(tw + n2 * k1));
      Y[k1 * (R2 + 1) + n2] = y;
    }
  }
  __syncthreads();
  // pass 2: (k1, line) tasks, one per thread
  const int k1 = threadIdx.x % R1, l = threadIdx.x / R1;
  V *Yl = buf + l * E;
  V x[R2];
#pragma unroll
  for (int n2 = 0; n2 < R2; ++n2) x[n2] = Yl[k1 * (R2 + 1) + n2];
  Dft<R2, false>::run(x);
  __syncthreads();
  // X[k1 + R1 k2] at row k2, column k1 (rows of R1 + 1)
#pragma unroll
  for (int k2 = 0; k2 < R2; ++k2) Yl[k2 * (R1 + 1) + k1] = x[k2];
  __syncthreads();
  auto X = [&](const V *Z, int kk) { return Z[(kk / R1) * (R1 + 1) + kk % R1]; };
  const S half = S(0.5);
  for (int task = threadIdx.x; task < L * H; task += blockDim.x) {
    const int m = task % H, ll = task / H;
    const V *Z = buf + ll * E;
    V a, b;
    if (m == 0) {
      const V z0 = X(Z, 0), zh = X(Z, H);
      a = mk<V>((z0.x + z0.x) * half, (zh.x + zh.x) * half);
      b = mk<V>((z0.y + z0.y) * half, (zh.y + zh.y) * half);
    } else {
      const V zm = X(Z, m), zc = X(Z, N - m);
      a = mk<V>((zm.x + zc.x) * half, (zm.y - zc.y) * half);
      b = mk<V>((zm.y + zc.y) * half, (zc.x - zm.x) * half);
    }
    const long long row = (long long)k * g.ny + j0 + 2 * ll;
    reinterpret_cast<V *>(var + row * N)[m] = a;
    reinterpret_cast<V *>(var + (row + 1) * N)[m] = b;
  }
}

// Backward: packed spectra -> p interior scaled by nf; with FUSE_BC the
// pressure halos as well (updateBoundP).  Grid (ny / (2 L), nz).
template <class T, int N, bool FUSE_BC>
__global__ void __launch_bounds__(x2_lines(N) * x2_r1(N))
    k_fft_x2_bwd(Geo g, const typename Cx<T>::V *__restrict__ tw, double nf,
                 const T *__restrict__ var, T *p, int rev) {
  using V = typename Cx<T>::V;
  using S = T;
  constexpr int R1 = x2_r1(N), R2 = N / R1, L = x2_lines(N), E = x2_line_elems(N), H = N / 2;
  extern __shared__ __align__(16) unsigned char fft_smem[];
  V *buf = reinterpret_cast<V *>(fft_smem);
  const int j0 = blockIdx.x * 2 * L;
  const int k = rev ? g.nz - 1 - (int)blockIdx.y : (int)blockIdx.y;
  const T scale = T(nf);
  // pass 1: element e of line l from the packed spectra of rows a and b
  for (int task = threadIdx.x; task < L * R2; task += blockDim.x) {
    const int n2 = task % R2, l = task / R2;
    const T *ra = var + ((long long)k * g.ny + j0 + 2 * l) * N, *rb = ra + N;
    V x[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) {
      const int e = R2 * n1 + n2;
      const int m = e <= H ? e : N - e;
      S reA, reB, imA = S(0), imB = S(0);
      if (m == 0 || m == H) {
        reA = ra[m == 0 ? 0 : 1];
        reB = rb[m == 0 ? 0 : 1];
      } else {
        const V a = reinterpret_cast<const V *>(ra)[m], b = reinterpret_cast<const V *>(rb)[m];
        reA = a.x;
        imA = a.y;
        reB = b.x;
        imB = b.y;
      }
      x[n1] = e <= H ? mk<V>(reA - imB, imA + reB) : mk<V>(reA + imB, reB - imA);
    }
    Dft<R1, true>::run(x);
    V *Y = buf + l * E;
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
      V y = x[k1];
      if (k1 > 0 && n2 > 0) y = cmulc(y, __ldg(tw + n2 * k1));
      Y[k1 * (R2 + 1) + n2] = y;
    }
  }
  __syncthreads();
  const int k1 = threadIdx.x % R1, l = threadIdx.x / R1;
  const V *Yl = buf + l * E;
  V x[R2];
#pragma unroll
  for (int n2 = 0; n2 < R2; ++n2) x[n2] = Yl[k1 * (R2 + 1) + n2];
  Dft<R2, true>::run(x);
  // element t = k1 + R1 k2 of rows j = j0 + 2l + 1 (a) and j + 1 (b) of
  // plane k + 1, with the periodic images and the zero-gradient ghost plane
  const int kk = k + 1;
  const int kimg = !FUSE_BC ? -1 : (kk == 1 ? 0 : (kk == g.nz ? g.nz + 1 : -1));
#pragma unroll
  for (int k2 = 0; k2 < R2; ++k2) {
    const V z = x[k2];
    const T ab[2] = {scale * z.x, scale * z.y};
    const int i = k1 + R1 * k2 + 1;
    const int iimg = !FUSE_BC ? -1 : (i == g.nx ? 0 : (i == 1 ? g.nx + 1 : -1));
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int j = j0 + 2 * l + 1 + h;
      const int jimg = !FUSE_BC ? -1 : (j == g.ny ? 0 : (j == 1 ? g.ny + 1 : -1));
      const T val = ab[h];
      auto put = [&](int jj, int kq) {
        T *r = p + (long long)jj * g.X + (long long)kq * g.XY;
        r[i] = val;
        if (iimg >= 0) r[iimg] = val;
      };
      put(j, kk);
      if (jimg >= 0) put(jimg, kk);
      if (kimg >= 0) {
        put(j, kimg);
        if (jimg >= 0) put(jimg, kimg);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Thomas sweep per (i,j) system with the reciprocal pivot table
// rpiv[(k*(ny/2+1) + my)*(nx/2+1) + mx]; the reference's divisions by b
// become multiplications by 1/b (mod_poisson_solver.cc:334-354).
//
// The sweeps are sequential in k, but their loads are not: batches of PF
// planes of the right-hand side and of the pivots are loaded one batch ahead
// of the elimination, so 2*PF loads per thread are in flight.  Sys gives the
// loads and stores of one system: rhs(k), piv(k), a(k), c(k), the forward
// values fwd_put(k, x) / fwd_get(k) and the solution out(k, x); A is the
// arithmetic type.
// ---------------------------------------------------------------------------
template <class A, int PF, class Sys>
__device__ __forceinline__ void thomas_sweep(int nz, const Sys &sys) {
  A prev = sys.rhs(0);
  sys.fwd_put(0, prev);
  {
    // forward elimination over k = 1 .. nz-1
    A xn[PF], rn[PF];
    int k = 1;
#pragma unroll
    for (int s = 0; s < PF; ++s)
      if (k + s < nz) {
        xn[s] = sys.rhs(k + s);
        rn[s] = sys.piv(k + s - 1);
      }
    for (; k < nz; k += PF) {
      A x[PF], r[PF];
#pragma unroll
      for (int s = 0; s < PF; ++s) {
        x[s] = xn[s];
        r[s] = rn[s];
      }
      const int kn = k + PF;
#pragma unroll
      for (int s = 0; s < PF; ++s)
        if (kn + s < nz) {
          xn[s] = sys.rhs(kn + s);
          rn[s] = sys.piv(kn + s - 1);
        }
#pragma unroll
      for (int s = 0; s < PF; ++s)
        if (k + s < nz) {
          A cur = x[s];
          cur -= (sys.a(k + s) * r[s]) * prev;
          sys.fwd_put(k + s, cur);
          prev = cur;
        }
    }
  }
  prev *= sys.piv(nz - 1);
  sys.out(nz - 1, prev);
  {
    // back substitution over k = nz-2 .. 0
    A xn[PF], rn[PF];
    int k = nz - 2;
#pragma unroll
    for (int s = 0; s < PF; ++s)
      if (k - s >= 0) {
        xn[s] = sys.fwd_get(k - s);
        rn[s] = sys.piv(k - s);
      }
    for (; k >= 0; k -= PF) {
      A x[PF], r[PF];
#pragma unroll
      for (int s = 0; s < PF; ++s) {
        x[s] = xn[s];
        r[s] = rn[s];
      }
      const int kn = k - PF;
#pragma unroll
      for (int s = 0; s < PF; ++s)
        if (kn - s >= 0) {
          xn[s] = sys.fwd_get(kn - s);
          rn[s] = sys.piv(kn - s);
        }
#pragma unroll
      for (int s = 0; s < PF; ++s)
        if (k - s >= 0) {
          const A cur = (x[s] - sys.c(k - s) * prev) * r[s];
          sys.out(k - s, cur);
          prev = cur;
        }
    }
  }
}

// The same sweep for a system solved in place in the spectral array (data,
// pivots and coefficients of type A), with the addresses walked by pointer
// increments (one 64-bit add an access instead of a 64-bit multiply-add):
// q = right-hand side and solution (plane stride `plane`), rp = reciprocal
// pivots (stride PS), ca / cc = the 1-D sub- and super-diagonal.  Same
// operations in the same order as thomas_sweep.
// L2 priorities of the sweep's traffic: the right-hand side and the forward
// values are read for the last time (evict first); the forward values are
// stored to be read back by the back substitution (evict last).
__device__ __forceinline__ double ld_last_use(const double *p) { return __ldcs(p); }
__device__ __forceinline__ float ld_last_use(const float *p) { return __ldcs(p); }
__device__ __forceinline__ unsigned long long l2_keep_policy() {
  unsigned long long pol;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ void st_keep(double *p, double v, unsigned long long pol) {
  asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(p), "d"(v), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void st_keep(float *p, float v, unsigned long long pol) {
  asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(v), "l"(pol)
               : "memory");
}

template <class A, int PF>
__device__ __forceinline__ void thomas_inplace(int nz, A *__restrict__ q, long long plane,
                                               const A *__restrict__ rp, long long PS,
                                               const A *__restrict__ ca,
                                               const A *__restrict__ cc) {
  const unsigned long long keep = l2_keep_policy();
  A prev = q[0];
  const A *lq = q + plane;  // next right-hand side to load (k = 1)
  const A *lr = rp;         // next pivot to load (k - 1 = 0)
  A *wq = q + plane;        // next forward value to store (k = 1)
  {
    A xn[PF], rn[PF];
#pragma unroll
    for (int s = 0; s < PF; ++s)
      if (1 + s < nz) {
        xn[s] = ld_last_use(lq);
        lq += plane;
        rn[s] = __ldg(lr);
        lr += PS;
      }
    for (int k = 1; k < nz; k += PF) {
      A x[PF], r[PF];
#pragma unroll
      for (int s = 0; s < PF; ++s) {
        x[s] = xn[s];
        r[s] = rn[s];
      }
#pragma unroll
      for (int s = 0; s < PF; ++s)
        if (k + PF + s < nz) {
          xn[s] = ld_last_use(lq);
          lq += plane;
          rn[s] = __ldg(lr);
          lr += PS;
        }
#pragma unroll
      for (int s = 0; s < PF; ++s)
        if (k + s < nz) {
          A cur = x[s];
          cur -= (__ldg(ca + k + s) * r[s]) * prev;
          st_keep(wq, cur, keep);
          wq += plane;
          prev = cur;
        }
    }
  }
  // lr is at pivot nz-1, wq one plane past the last forward value
  prev *= __ldg(lr);
  wq -= plane;
  *wq = prev;
  {
    const A *bq = wq - plane;  // next forward value to load (k = nz - 2)
    const A *br = lr - PS;     // its pivot
    A *bw = wq - plane;        // next solution value to store
    A xn[PF], rn[PF];
#pragma unroll
    for (int s = 0; s < PF; ++s)
      if (nz - 2 - s >= 0) {
        xn[s] = ld_last_use(bq);
        bq -= plane;
        rn[s] = __ldg(br);
        br -= PS;
      }
    for (int k = nz - 2; k >= 0; k -= PF) {
      A x[PF], r[PF];
#pragma unroll
      for (int s = 0; s < PF; ++s) {
        x[s] = xn[s];
        r[s] = rn[s];
      }
#pragma unroll
      for (int s = 0; s < PF; ++s)
        if (k - PF - s >= 0) {
          xn[s] = ld_last_use(bq);
          bq -= plane;
          rn[s] = __ldg(br);
          br -= PS;
        }
#pragma unroll
      for (int s = 0; s < PF; ++s)
        if (k - s >= 0) {
          const A cur = (x[s] - __ldg(cc + k - s) * prev) * r[s];
          *bw = cur;
          bw -= plane;
          prev = cur;
        }
    }
  }
}

// A low-wavenumber system of the mixed form: FP32 right-hand side and
// solution, FP64 pivots and arithmetic, forward values in the FP64 buffer
// `lq` (plane stride LP).
struct LowSys {
  float *q;
  long long plane;
  double *lq;
  long long LP;
  const double *rp;
  long long PS;
  const double *ca, *cc;
  __device__ __forceinline__ double rhs(int k) const { return double(q[(long long)k * plane]); }
  __device__ __forceinline__ double piv(int k) const { return __ldg(rp + (long long)k * PS); }
  __device__ __forceinline__ double a(int k) const { return __ldg(ca + k); }
  __device__ __forceinline__ double c(int k) const { return __ldg(cc + k); }
  __device__ __forceinline__ void fwd_put(int k, double x) const { lq[k * LP] = x; }
  __device__ __forceinline__ double fwd_get(int k) const { return lq[k * LP]; }
  __device__ __forceinline__ void out(int k, double x) const {
    q[(long long)k * plane] = float(x);
  }
};

// packed indices (i, j) of system t and the offset of its pivot column
__device__ __forceinline__ void trid_index(int t, int nx, int ny, int &i, int &j,
                                           long long &pivot) {
  i = t % nx;
  j = t / nx;
  const int mx = (i == 0) ? 0 : ((i == 1) ? (nx >> 1) : (i >> 1));
  const int my = (j == 0) ? 0 : ((j == 1) ? (ny >> 1) : (j >> 1));
  pivot = (long long)my * ((nx >> 1) + 1) + mx;
}

// FP64: the reference's solve, in place.
__global__ void __launch_bounds__(128) k_trid(int nx, int ny, int nz,
                                              const double *__restrict__ rpiv,
                                              const double *__restrict__ a,
                                              const double *__restrict__ c,
                                              double *__restrict__ var) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const long long plane = (long long)nx * ny;
  if (t >= plane) return;
  int i, j;
  long long pv;
  trid_index(t, nx, ny, i, j, pv);
  const long long PS = (long long)((nx >> 1) + 1) * ((ny >> 1) + 1);
  thomas_inplace<double, 8>(nz, var + t, plane, rpiv + pv, PS, a, c);
}

// Mixed form: systems whose packed x and y indices are both below kLowModes
// (the lowest wavenumbers, with the largest amplification 1/lambda, and the
// pinned singular (0,0) mode) sweep in FP64 with FP64 pivots and FP64
// forward values in `low` [k][j][i]; all other systems sweep in FP32 in
// place with the FP32 pivot table, 24 planes of loads in flight.
__global__ void __launch_bounds__(128) k_trid_mixed(
    int nx, int ny, int nz, const float *__restrict__ rpiv32, const float *__restrict__ a32,
    const float *__restrict__ c32, const double *__restrict__ rpiv,
    const double *__restrict__ a, const double *__restrict__ c, float *__restrict__ var,
    double *__restrict__ low) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const long long plane = (long long)nx * ny;
  if (t >= plane) return;
  int i, j;
  long long pv;
  trid_index(t, nx, ny, i, j, pv);
  const long long PS = (long long)((nx >> 1) + 1) * ((ny >> 1) + 1);
  if (i < kLowModes && j < kLowModes) {
    constexpr long long LP = (long long)kLowModes * kLowModes;
    thomas_sweep<double, 8>(
        nz, LowSys{var + t, plane, low + j * kLowModes + i, LP, rpiv + pv, PS, a, c});
  } else {
    // 24 planes of loads in flight (0.238 ms against 0.252 for 16 and 0.259
    // for 8 at 768 x 384 x 256)
    thomas_inplace<float, 24>(nz, var + t, plane, rpiv32 + pv, PS, a32, c32);
  }
}

// The same for one block of a batched launch over several channels (the
// block's coordinates from the work list).  The single-channel kernel keeps
// its own copy of these lines: a body shared between the two changed the
// single-channel kernel's code generation and made it slower.
__device__ __forceinline__ void trid_mixed_body(
    int nx, int ny, int nz, const float *__restrict__ rpiv32, const float *__restrict__ a32,
    const float *__restrict__ c32, const double *__restrict__ rpiv,
    const double *__restrict__ a, const double *__restrict__ c, float *__restrict__ var,
    double *__restrict__ low, int bx) {
  const int t = bx * blockDim.x + threadIdx.x;
  const long long plane = (long long)nx * ny;
  if (t >= plane) return;
  int i, j;
  long long pv;
  trid_index(t, nx, ny, i, j, pv);
  const long long PS = (long long)((nx >> 1) + 1) * ((ny >> 1) + 1);
  if (i < kLowModes && j < kLowModes) {
    constexpr long long LP = (long long)kLowModes * kLowModes;
    thomas_sweep<double, 8>(
        nz, LowSys{var + t, plane, low + j * kLowModes + i, LP, rpiv + pv, PS, a, c});
  } else {
    // 24 planes of loads in flight (0.238 ms against 0.252 for 16 and 0.259
    // for 8 at 768 x 384 x 256)
    thomas_inplace<float, 24>(nz, var + t, plane, rpiv32 + pv, PS, a32, c32);
  }
}

// ---------------------------------------------------------------------------
// Batched launches over the mixed-form channels of an ensemble: one launch
// per stage (and line length) carries each channel's arguments in its
// parameters; block b works for channel m, start[m] <= b < start[m + 1], as
// block b - start[m] of that channel's own grid (for the persistent kernels:
// of the channel's share of the launch's blocks, vblocks).
// ---------------------------------------------------------------------------
struct XfMember {
  Geo g;
  FftDev<float2> P;
  int nl, gx, gy;
  const StepConst *sc;
  const float *u, *v, *w;
  float *var;
};
struct XfBatch {
  int n;
  int start[kBatchMax + 1];
  XfMember m[kBatchMax];
};
template <int N, int PL>
__global__ void __launch_bounds__(256) k_fft_x_fwd_div_batch(const __grid_constant__ XfBatch b) {
  batch_grid_sync();
  const int q = batch_member(b.start, b.n, (int)blockIdx.x);
  const XfMember &a = b.m[q];
  fft_x_fwd_div_body<float, N, true, PL>(a.g, a.P, a.nl, a.sc, nullptr, a.u, a.v, a.w, a.var,
                                         VBlk::of((int)blockIdx.x - b.start[q], a.gx, a.gy, 1));
}

struct YMember {
  int nx, ny, nz, nl, rev, vblocks;
  FftDev<float2> P;
  float *var;
};
struct YBatch {
  int n;
  int start[kBatchMax + 1];
  YMember m[kBatchMax];
};
template <int N, bool INV, int PL>
__global__ void __launch_bounds__(256) k_fft_y_batch(const __grid_constant__ YBatch b) {
  batch_grid_sync();
  const int q = batch_member(b.start, b.n, (int)blockIdx.x);
  const YMember &a = b.m[q];
  fft_y_body<float, N, INV, PL>(a.nx, a.ny, a.nz, a.P, a.nl, a.var, a.rev,
                                VBlk::of((int)blockIdx.x - b.start[q], a.vblocks, 1, 1));
}

struct XbMember {
  Geo g;
  FftDev<float2> P;
  int nl, rev, vblocks;
  double nf;
  const float *var;
  float *p;
};
struct XbBatch {
  int n;
  int start[kBatchMax + 1];
  XbMember m[kBatchMax];
};
template <int N, int PL>
__global__ void __launch_bounds__(128) k_fft_x_bwd_batch(const __grid_constant__ XbBatch b) {
  batch_grid_sync();
  const int q = batch_member(b.start, b.n, (int)blockIdx.x);
  const XbMember &a = b.m[q];
  fft_x_bwd_body<float, N, true, PL>(a.g, a.P, a.nl, a.nf, a.var, a.p, a.rev,
                                     VBlk::of((int)blockIdx.x - b.start[q], a.vblocks, 1, 1));
}

struct TrMember {
  int nx, ny, nz;
  const float *rpiv32, *a32, *c32;
  const double *rpiv, *a, *c;
  float *var;
  double *low;
};
struct TrBatch {
  int n;
  int start[kBatchMax + 1];
  TrMember m[kBatchMax];
};
__global__ void __launch_bounds__(128) k_trid_mixed_batch(const __grid_constant__ TrBatch b) {
  batch_grid_sync();
  const int q = batch_member(b.start, b.n, (int)blockIdx.x);
  const TrMember &a = b.m[q];
  trid_mixed_body(a.nx, a.ny, a.nz, a.rpiv32, a.a32, a.c32, a.rpiv, a.a, a.c, a.var, a.low,
                  (int)blockIdx.x - b.start[q]);
}
static_assert(sizeof(XfBatch) <= 32000 && sizeof(YBatch) <= 32000 && sizeof(XbBatch) <= 32000 &&
                  sizeof(TrBatch) <= 32000,
              "kernel parameters are limited to 32764 bytes");

// ---------------------------------------------------------------------------
// Thomas sweep with the right-hand side held on chip.  A block of 32 threads
// owns 32 consecutive systems (packed x indices i0 .. i0+31 of one packed y
// row j) and copies their whole columns -- nz rows of 32 elements, one
// 16-byte-aligned segment per plane -- into shared memory with bulk copies
// (cp.async.bulk, no multicast), in eight chunks of planes each signalling
// its own mbarrier.  The forward elimination starts on the first chunk while
// the others land, keeps the forward values in place in shared memory, and
// the back substitution writes the solution to global memory once: the
// spectral array is read once and written once (the forward values no
// longer round-trip through HBM).  Same operations in the same order as
// thomas_inplace.  Every wait is bounded: on a timeout the block records
// the error word and leaves.
// ---------------------------------------------------------------------------
constexpr int kTridChunks = 8;
constexpr long long kTridWaitLimit = 1ll << 22;

__device__ __forceinline__ unsigned trid_smem_addr(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void trid_bulk_load(void *dst, const void *src, unsigned bytes,
                                               unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(trid_smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(trid_smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ bool trid_try_wait(unsigned long long *bar) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(trid_smem_addr(bar))
      : "memory");
  return ok != 0;
}

size_t trid_tile_smem(int nz, size_t elem) { return (size_t)nz * 32 * elem + 8 * kTridChunks + 16; }

// The block's columns: systems t = blockIdx.x * 32 + lane (nx % 32 == 0, so
// one packed y row j); xs[k * 32 + lane] holds row k of the lane's system.
template <class A>
__device__ __forceinline__ void trid_tile_load(A *xs, unsigned long long *bar, const A *col,
                                               long long plane, int nz, int cp) {
  const int lane = threadIdx.x;
  if (lane == 0) {
    for (int ch = 0; ch < kTridChunks; ++ch) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(trid_smem_addr(bar + ch)));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int ch = 0; ch < kTridChunks; ++ch) {
      const int k0 = ch * cp, k1 = min(nz, k0 + cp);
      const unsigned bytes = (unsigned)(k1 > k0 ? k1 - k0 : 0) * 32u * (unsigned)sizeof(A);
      // the chunk's expected bytes (an empty chunk completes at once)
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                       trid_smem_addr(bar + ch)),
                   "r"(bytes)
                   : "memory");
    }
  }
  __syncwarp();
  for (int k = lane; k < nz; k += 32)
    trid_bulk_load(xs + k * 32, col + k * plane, 32u * (unsigned)sizeof(A), bar + k / cp);
}

// Before the block exits: every chunk has landed (returns at once when the
// sweep waited for them all; bounded when a wait gave up, so that no copy
// into this block's shared memory is still in flight when it leaves).
__device__ __forceinline__ void trid_drain(unsigned long long *bar, int *err) {
  for (int ch = 0; ch < kTridChunks; ++ch) {
    bool done = false;
    for (long long it = 0; it < kTridWaitLimit && !done; ++it) done = trid_try_wait(bar + ch);
    if (!done) atomicOr(err, 4);
  }
}

__device__ __forceinline__ bool trid_wait_chunk(unsigned long long *bar, int ch, int *err) {
  for (long long it = 0; it < kTridWaitLimit; ++it)
    if (trid_try_wait(bar + ch)) return true;
  atomicOr(err, 4);
  return false;
}

// The sweep of one lane's system: xs column (stride 32), pivots rp (stride
// PS), 1-D coefficients ca, cc; solution stored to q (plane stride).
template <class A>
__device__ __forceinline__ void trid_tile_sweep(A *xs, int nz, int cp,
                                                unsigned long long *bar, const A *__restrict__ rp,
                                                long long PS, const A *__restrict__ ca,
                                                const A *__restrict__ cc, A *q, long long plane,
                                                int *err, bool &ok) {
  const int lane = threadIdx.x;
  constexpr int PF = 8;
  if (!trid_wait_chunk(bar, 0, err)) {
    ok = false;
    return;
  }
  A prev = xs[lane];
  // forward elimination, pivots of PF planes loaded one batch ahead
  A rn[PF];
#pragma unroll
  for (int s = 0; s < PF; ++s)
    if (s < nz - 1) rn[s] = __ldg(rp + (long long)s * PS);
  int next_chunk = 1;
  for (int k = 1; k < nz; k += PF) {
    A r[PF];
#pragma unroll
    for (int s = 0; s < PF; ++s) r[s] = rn[s];
#pragma unroll
    for (int s = 0; s < PF; ++s)
      if (k + PF + s - 1 <= nz - 2) rn[s] = __ldg(rp + (long long)(k + PF + s - 1) * PS);
#pragma unroll
    for (int s = 0; s < PF; ++s) {
      const int kk = k + s;
      if (kk < nz) {
        while (next_chunk < kTridChunks && kk >= next_chunk * cp) {
          if (!trid_wait_chunk(bar, next_chunk, err)) {
            ok = false;
            return;
          }
          ++next_chunk;
        }
        A cur = xs[kk * 32 + lane];
        cur -= (__ldg(ca + kk) * r[s]) * prev;
        xs[kk * 32 + lane] = cur;
        prev = cur;
      }
    }
  }
  prev *= __ldg(rp + (long long)(nz - 1) * PS);
  q[(long long)(nz - 1) * plane] = prev;
  // back substitution
#pragma unroll
  for (int s = 0; s < PF; ++s)
    if (nz - 2 - s >= 0) rn[s] = __ldg(rp + (long long)(nz - 2 - s) * PS);
  for (int k = nz - 2; k >= 0; k -= PF) {
    A r[PF];
#pragma unroll
    for (int s = 0; s < PF; ++s) r[s] = rn[s];
#pragma unroll
    for (int s = 0; s < PF; ++s)
      if (k - PF - s >= 0) rn[s] = __ldg(rp + (long long)(k - PF - s) * PS);
#pragma unroll
    for (int s = 0; s < PF; ++s) {
      const int kk = k - s;
      if (kk >= 0) {
        const A cur = (xs[kk * 32 + lane] - __ldg(cc + kk) * prev) * r[s];
        q[(long long)kk * plane] = cur;
        prev = cur;
      }
    }
  }
}

// FP64: the reference's solve with the columns on chip.
__global__ void __launch_bounds__(32) k_trid_tile(int nx, int ny, int nz,
                                                  const double *__restrict__ rpiv,
                                                  const double *__restrict__ a,
                                                  const double *__restrict__ c,
                                                  double *__restrict__ var, int *err) {
  extern __shared__ __align__(128) unsigned char trid_smem[];
  double *xs = reinterpret_cast<double *>(trid_smem);
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(xs + (size_t)nz * 32);
  const int lane = threadIdx.x;
  const long long plane = (long long)nx * ny;
  const long long t0 = (long long)blockIdx.x * 32;
  const int cp = (nz + kTridChunks - 1) / kTridChunks;
  trid_tile_load(xs, bar, var + t0, plane, nz, cp);
  int i, j;
  long long pv;
  trid_index((int)(t0 + lane), nx, ny, i, j, pv);
  const long long PS = (long long)((nx >> 1) + 1) * ((ny >> 1) + 1);
  bool ok = true;
  trid_tile_sweep<double>(xs, nz, cp, bar, rpiv + pv, PS, a, c, var + t0 + lane, plane, err, ok);
  __syncwarp();
  if (lane == 0) trid_drain(bar, err);
}

// A low-wavenumber system of the mixed form whose right-hand side is the
// on-chip FP32 column xs (stride 32): FP64 pivots, arithmetic and forward
// values (in lq), solution stored to q.
struct LowSysSmem {
  const float *xs;
  float *q;
  long long plane;
  double *lq;
  long long LP;
  const double *rp;
  long long PS;
  const double *ca, *cc;
  __device__ __forceinline__ double rhs(int k) const { return double(xs[k * 32]); }
  __device__ __forceinline__ double piv(int k) const { return __ldg(rp + (long long)k * PS); }
  __device__ __forceinline__ double a(int k) const { return __ldg(ca + k); }
  __device__ __forceinline__ double c(int k) const { return __ldg(cc + k); }
  __device__ __forceinline__ void fwd_put(int k, double x) const { lq[k * LP] = x; }
  __device__ __forceinline__ double fwd_get(int k) const { return lq[k * LP]; }
  __device__ __forceinline__ void out(int k, double x) const {
    q[(long long)k * plane] = float(x);
  }
};

// Mixed form: the FP32 systems sweep on chip as above; the systems of the
// lowest wavenumbers (packed x and y indices below kLowModes) sweep in FP64
// with their forward values in `low`, reading their right-hand side from
// the same on-chip column.
__global__ void __launch_bounds__(32) k_trid_mixed_tile(
    int nx, int ny, int nz, const float *__restrict__ rpiv32, const float *__restrict__ a32,
    const float *__restrict__ c32, const double *__restrict__ rpiv,
    const double *__restrict__ a, const double *__restrict__ c, float *__restrict__ var,
    double *__restrict__ low, int *err) {
  extern __shared__ __align__(128) unsigned char trid_smem[];
  float *xs = reinterpret_cast<float *>(trid_smem);
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(
      trid_smem + ((size_t)nz * 32 * sizeof(float) + 15) / 16 * 16);
  const int lane = threadIdx.x;
  const long long plane = (long long)nx * ny;
  const long long t0 = (long long)blockIdx.x * 32;
  const int cp = (nz + kTridChunks - 1) / kTridChunks;
  trid_tile_load(xs, bar, var + t0, plane, nz, cp);
  int i, j;
  long long pv;
  trid_index((int)(t0 + lane), nx, ny, i, j, pv);
  const long long PS = (long long)((nx >> 1) + 1) * ((ny >> 1) + 1);
  bool ok = true;
  if (i < kLowModes && j < kLowModes) {
    // every chunk must have landed before the FP64 sweep reads the column
    for (int ch = 0; ch < kTridChunks && ok; ++ch) ok = trid_wait_chunk(bar, ch, err);
    if (ok) {
      constexpr long long LP = (long long)kLowModes * kLowModes;
      thomas_sweep<double, 8>(nz, LowSysSmem{xs + lane, var + t0 + lane, plane,
                                             low + j * kLowModes + i, LP, rpiv + pv, PS, a, c});
    }
  } else {
    trid_tile_sweep<float>(xs, nz, cp, bar, rpiv32 + pv, PS, a32, c32, var + t0 + lane, plane,
                           err, ok);
  }
  __syncwarp();
  if (lane == 0) trid_drain(bar, err);
}

// The same over the mixed-form channels of an ensemble: block b works on the
// 32 systems of block b - start[m] of channel m (start[m] <= b < start[m+1]);
// the shared memory holds the longest column of the launch.
struct TrtMember {
  int nx, ny, nz;
  const float *rpiv32, *a32, *c32;
  const double *rpiv, *a, *c;
  float *var;
  double *low;
  int *err;
};
struct TrtBatch {
  int n;
  int start[kBatchMax + 1];
  TrtMember m[kBatchMax];
};
static_assert(sizeof(TrtBatch) <= 32000, "kernel parameters are limited to 32764 bytes");
__global__ void __launch_bounds__(32) k_trid_mixed_tile_batch(const __grid_constant__ TrtBatch bt) {
  batch_grid_sync();
  const int q = batch_member(bt.start, bt.n, (int)blockIdx.x);
  const TrtMember &M = bt.m[q];
  const int nx = M.nx, ny = M.ny, nz = M.nz;
  float *var = M.var;
  extern __shared__ __align__(128) unsigned char trid_smem[];
  float *xs = reinterpret_cast<float *>(trid_smem);
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(
      trid_smem + ((size_t)nz * 32 * sizeof(float) + 15) / 16 * 16);
  const int lane = threadIdx.x;
  const long long plane = (long long)nx * ny;
  const long long t0 = (long long)((int)blockIdx.x - bt.start[q]) * 32;
  const int cp = (nz + kTridChunks - 1) / kTridChunks;
  trid_tile_load(xs, bar, var + t0, plane, nz, cp);
  int i, j;
  long long pv;
  trid_index((int)(t0 + lane), nx, ny, i, j, pv);
  const long long PS = (long long)((nx >> 1) + 1) * ((ny >> 1) + 1);
  bool ok = true;
  if (i < kLowModes && j < kLowModes) {
    for (int ch = 0; ch < kTridChunks && ok; ++ch) ok = trid_wait_chunk(bar, ch, M.err);
    if (ok) {
      constexpr long long LP = (long long)kLowModes * kLowModes;
      thomas_sweep<double, 8>(nz, LowSysSmem{xs + lane, var + t0 + lane, plane,
                                             M.low + j * kLowModes + i, LP, M.rpiv + pv, PS, M.a,
                                             M.c});
    }
  } else {
    trid_tile_sweep<float>(xs, nz, cp, bar, M.rpiv32 + pv, PS, M.a32, M.c32, var + t0 + lane,
                           plane, M.err, ok);
  }
  __syncwarp();
  if (lane == 0) trid_drain(bar, M.err);
}

template <class T>
FftDev<typename Cx<T>::V> dev_plan(const FftPlan &p) {
  FftDev<typename Cx<T>::V> d;
  d.n = p.n;
  d.npass = p.npass;
  d.radices = 0ull;
  for (int r = 0; r < p.npass; ++r) d.radices |= (unsigned long long)(p.radix[r] - 1) << (4 * r);
  if constexpr (std::is_same<T, double>::value)
    d.tw = p.tw;
  else
    d.tw = p.tw32;
  return d;
}

template <class T>
size_t fft_bytes(int n, int lines) {
  using V = typename Cx<T>::V;
  return 2ull * (size_t)lines * (size_t)line_stride<V>(n) * sizeof(V);
}

}  // namespace

size_t fft_smem_bytes(int n, int lines) { return fft_bytes<double>(n, lines); }

namespace {
// halo'd row length of a field: nx + 2, padded to 16 bytes in FP32
template <class T>
size_t x_pitch(int nx) {
  return sizeof(T) == 4 ? (size_t)((nx + 2 + 3) / 4) * 4 : (size_t)nx + 2;
}
template <class T>
size_t smem_x_fwd(int nx, int nl) {
  return fft_bytes<T>(nx, nl) + (size_t)2 * nl * x_pitch<T>(nx) * sizeof(T);
}
template <class T>
size_t smem_x_bwd(int nx, int nl) {
  return fft_bytes<T>(nx, nl) + (size_t)2 * nl * nx * sizeof(T);
}
template <class T>
size_t smem_y(int ny, int nl) {
  return fft_bytes<T>(ny, nl) + (size_t)ny * 2 * nl * sizeof(T);
}
// Largest number of line pairs per tile that divides `pairs`, is a multiple
// of `step` and keeps the kernel's shared memory under `cap` bytes.
template <class F>
int pick_lines(int pairs, size_t cap, F bytes, int step = 1) {
  int best = step;
  for (int d = step; d <= pairs && d <= 16; d += step)
    if (pairs % d == 0 && bytes(d) <= cap) best = d;
  return best;
}
template <class K>
int persistent_grid(K kernel, int threads, size_t smem, int sms, long long ntiles) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) !=
          cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  long long g = (long long)per_sm * sms;
  if (g > ntiles) g = ntiles;
  return (int)(g < 1 ? 1 : g);
}
}  // namespace

// Line lengths with compile-time plans (the grids of the supported channel
// cases); any other 2^a 3^b length runs the runtime plan (N = 0).
template <class F>
cudaError_t with_size(int n, F &&f) {
  switch (n) {
    case 32: return f(std::integral_constant<int, 32>{});
    case 48: return f(std::integral_constant<int, 48>{});
    case 64: return f(std::integral_constant<int, 64>{});
    case 96: return f(std::integral_constant<int, 96>{});
    case 128: return f(std::integral_constant<int, 128>{});
    case 192: return f(std::integral_constant<int, 192>{});
    case 256: return f(std::integral_constant<int, 256>{});
    case 384: return f(std::integral_constant<int, 384>{});
    case 512: return f(std::integral_constant<int, 512>{});
    case 768: return f(std::integral_constant<int, 768>{});
    default: return f(std::integral_constant<int, 0>{});
  }
}
constexpr int kPlanSizes[] = {0, 32, 48, 64, 96, 128, 192, 256, 384, 512, 768};

// The plan family of a transform of length N: 1 (radix 24) only where the
// length has that family, 0 otherwise.
template <int N, class F>
cudaError_t with_plan(int plan, F &&f) {
  if constexpr (N > 0 && plan_has24(N)) {
    if (plan == 1) return f(std::integral_constant<int, 1>{});
  }
  return f(std::integral_constant<int, 0>{});
}
// A warp-line plan (family 2) exists for length n and a line-pair axis of
// `pairs_axis` real lines (ny for the x transforms, nx for the y transforms).
bool fft_has_warp_plan(int n, int lines_axis) {
  // the larger line count (FP32 y transforms) must divide as well
  const int L = wp_lines(n, true);
  return L > 0 && lines_axis % (2 * L) == 0;
}
// A two-pass y plan (family 3) for line length ny over nx columns (whole
// blocks of 2 y2_lines columns) in the form whose elements have elem bytes.
bool fft_has_y2_plan(int ny, int nx, int elem) {
  const int L = elem == 4 ? y2_lines<float>() : y2_lines<double>();
  return y2_r1(ny) > 0 && nx % (2 * L) == 0;
}
// A two-pass x plan (family 3) for line length nx over ny rows (whole
// blocks of 2 x2_lines rows).
bool fft_has_x2_plan(int nx, int ny) {
  return x2_r1(nx) > 0 && ny % (2 * x2_lines(nx)) == 0;
}
bool fft_has_two_plans(int n) {
  bool two = false;
  with_size(n, [&](auto NC) -> cudaError_t {
    constexpr int N = decltype(NC)::value;
    two = N > 0 && plan_has24(N);
    return cudaSuccess;
  });
  return two;
}

// Raises the dynamic shared-memory limit of every FFT kernel (once per process).
cudaError_t fft_configure(size_t max_bytes) {
  for (int n : kPlanSizes) {
    const cudaError_t e = with_size(n, [&](auto NC) -> cudaError_t {
      constexpr int N = decltype(NC)::value;
      cudaError_t r;
// the dynamic limit is what the device allows beyond the kernel's static shared memory
#define PLC_SMEM(kern)                                                                    \
  {                                                                                       \
    cudaFuncAttributes fa;                                                                \
    r = cudaFuncGetAttributes(&fa, kern);                                                 \
    if (r != cudaSuccess) return r;                                                       \
    r = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,          \
                             (int)(max_bytes - fa.sharedSizeBytes));                      \
    if (r != cudaSuccess) return r;                                                       \
  }
      auto conf = [&](auto PC) -> cudaError_t {
        constexpr int PL = decltype(PC)::value;
        PLC_SMEM((k_fft_x_fwd<double, N, PL>));
        PLC_SMEM((k_fft_x_fwd_div<double, N, true, PL>));
        PLC_SMEM((k_fft_x_bwd<double, N, true, PL>));
        PLC_SMEM((k_fft_x_bwd<double, N, false, PL>));
        PLC_SMEM((k_fft_y<double, N, true, PL>));
        PLC_SMEM((k_fft_y<double, N, false, PL>));
        PLC_SMEM((k_fft_x_fwd<float, N, PL>));
        PLC_SMEM((k_fft_x_fwd_div<float, N, true, PL>));
        PLC_SMEM((k_fft_x_bwd<float, N, true, PL>));
        PLC_SMEM((k_fft_x_bwd<float, N, false, PL>));
        PLC_SMEM((k_fft_y<float, N, true, PL>));
        PLC_SMEM((k_fft_y<float, N, false, PL>));
        PLC_SMEM((k_fft_x_fwd_div_batch<N, PL>));
        PLC_SMEM((k_fft_x_bwd_batch<N, PL>));
        PLC_SMEM((k_fft_y_batch<N, true, PL>));
        PLC_SMEM((k_fft_y_batch<N, false, PL>));
        return cudaSuccess;
      };
      if constexpr (N > 0 && x2_r1(N) > 0) {
        PLC_SMEM((k_fft_x2_fwd<double, N, false>));
        PLC_SMEM((k_fft_x2_fwd<double, N, true>));
        PLC_SMEM((k_fft_x2_bwd<double, N, false>));
        PLC_SMEM((k_fft_x2_bwd<double, N, true>));
        PLC_SMEM((k_fft_x2_fwd<float, N, false>));
        PLC_SMEM((k_fft_x2_fwd<float, N, true>));
        PLC_SMEM((k_fft_x2_bwd<float, N, false>));
        PLC_SMEM((k_fft_x2_bwd<float, N, true>));
      }
      if constexpr (N > 0 && y2_r1(N) > 0) {
        PLC_SMEM((k_fft_y2<double, N, false>));
        PLC_SMEM((k_fft_y2<double, N, true>));
        PLC_SMEM((k_fft_y2<float, N, false>));
        PLC_SMEM((k_fft_y2<float, N, true>));
        PLC_SMEM((k_fft_y2_batch<N, false>));
        PLC_SMEM((k_fft_y2_batch<N, true>));
      }
      if constexpr (N > 0 && wp_base_lines(N) > 0) {
        PLC_SMEM((k_wfft_y<double, N, false>));
        PLC_SMEM((k_wfft_y<double, N, true>));
        PLC_SMEM((k_wfft_x_fwd<double, N, true>));
        PLC_SMEM((k_wfft_x_fwd<double, N, false>));
        PLC_SMEM((k_wfft_x_bwd<double, N, true>));
        PLC_SMEM((k_wfft_x_bwd<double, N, false>));
        PLC_SMEM((k_wfft_y<float, N, false>));
        PLC_SMEM((k_wfft_y<float, N, true>));
        PLC_SMEM((k_wfft_x_fwd<float, N, true>));
        PLC_SMEM((k_wfft_x_fwd<float, N, false>));
        PLC_SMEM((k_wfft_x_bwd<float, N, true>));
        PLC_SMEM((k_wfft_x_bwd<float, N, false>));
      }
      if constexpr (N == 0) {
        PLC_SMEM(k_trid_tile);
        PLC_SMEM(k_trid_mixed_tile);
        PLC_SMEM(k_trid_mixed_tile_batch);
      }
      r = conf(std::integral_constant<int, 0>{});
      if (r != cudaSuccess) return r;
      if constexpr (N > 0 && plan_has24(N)) {
        r = conf(std::integral_constant<int, 1>{});
        if (r != cudaSuccess) return r;
      }
#undef PLC_SMEM
      return cudaSuccess;
    });
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

namespace {
// Persistent grid sizes for the context's line counts; fails if a kernel's
// shared memory exceeds the device limit.
template <class T>
cudaError_t fft_grids_t(plc_ctx *c, size_t dev_max, int sms) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  const size_t need[4] = {smem_x_fwd<T>(nx, c->fft_lines_x), fft_bytes<T>(nx, c->fft_lines_xf),
                          smem_x_bwd<T>(nx, c->fft_lines_x), smem_y<T>(ny, c->fft_lines_y)};
  for (size_t b : need)
    if (b > dev_max) return cudaErrorInvalidValue;
  const long long tiles_x = (long long)(ny / (2 * c->fft_lines_x)) * nz;
  const long long tiles_y = (long long)(nx / (2 * c->fft_lines_y)) * nz;
  cudaError_t e = with_size(nx, [&](auto NC) -> cudaError_t {
    constexpr int N = decltype(NC)::value;
    return with_plan<N>(c->fft_plan_x, [&](auto PC) -> cudaError_t {
      constexpr int PL = decltype(PC)::value;
      c->grid_xf = persistent_grid(k_fft_x_fwd<T, N, PL>, 128, need[0], sms, tiles_x);
      c->grid_xb = persistent_grid(k_fft_x_bwd<T, N, true, PL>, 128, need[2], sms, tiles_x);
      return cudaSuccess;
    });
  });
  if (e != cudaSuccess) return e;
  return with_size(ny, [&](auto NC) -> cudaError_t {
    constexpr int N = decltype(NC)::value;
    return with_plan<N>(c->fft_plan_y, [&](auto PC) -> cudaError_t {
      constexpr int PL = decltype(PC)::value;
      c->grid_y = persistent_grid(k_fft_y<T, N, false, PL>, 256, need[3], sms, tiles_y);
      return cudaSuccess;
    });
  });
}

template <class T>
cudaError_t fft_setup_t(plc_ctx *c, size_t smem_cap_per_block, size_t dev_max, int sms) {
  const int nx = c->nx, ny = c->ny;
  // FP32 staging copies 16-byte chunks of 4 elements: tiles of the y
  // transform then span a multiple of 4 columns (an even number of pairs)
  const int ystep = sizeof(T) == 4 ? 2 : 1;
  c->fft_lines_x =
      pick_lines(ny / 2, smem_cap_per_block, [&](int d) { return smem_x_bwd<T>(nx, d); });
  c->fft_lines_xf = pick_lines(ny / 2, 64 * 1024, [&](int d) { return fft_bytes<T>(nx, d); });
  c->fft_lines_y = pick_lines(
      nx / 2, smem_cap_per_block, [&](int d) { return smem_y<T>(ny, d); }, ystep);
  return fft_grids_t<T>(c, dev_max, sms);
}
}  // namespace

// Tile sizes (line pairs per tile) and persistent grid sizes of the
// transforms, from the shared memory each needs and the occupancy it gets.
cudaError_t fft_setup(plc_ctx *c, size_t smem_cap_per_block, size_t dev_max) {
  const int sms = c->num_sms;  // the context's SM budget
  return c->mixed ? fft_setup_t<float>(c, smem_cap_per_block, dev_max, sms)
                  : fft_setup_t<double>(c, smem_cap_per_block, dev_max, sms);
}

namespace {
// Warp-line launch geometry: blocks of GPB line groups (G warps each) over
// the `groups` line groups of one plane, grid (groups / GPB, nz); shared
// memory GPB L line strides.
template <class T, int N, bool YDIR>
struct WpLaunch {
  dim3 grid, block;
  size_t smem;
  WpLaunch(int lines_axis, int nz) {
    using V = typename Cx<T>::V;
    constexpr int G = wp_group(N), L = wp_lines(N, YDIR && sizeof(T) == 4);
    const int groups = lines_axis / (2 * L);
    const int gpb = wp_groups_per_block(groups, G);
    grid = dim3(groups / gpb, nz);
    block = dim3(32 * G * gpb);
    smem = (size_t)gpb * L * line_stride<V>(N) * sizeof(V);
  }
};

template <class T>
cudaError_t fft_x_fwd_t(const plc_ctx *c, const T *p, const T *u, const T *v, const T *w, T *var,
                        cudaStream_t s) {
  // the forward transform's own family (the backward one's when not set);
  // the shared-memory families take the backward one's radix family
  const int pf = c->fft_plan_xf >= 0 ? c->fft_plan_xf : c->fft_plan_x;
  const int pfam = pf >= 2 ? (c->fft_plan_x >= 2 ? 0 : c->fft_plan_x) : pf;
  return with_size(c->nx, [&](auto NC) -> cudaError_t {
    constexpr int N = decltype(NC)::value;
    if constexpr (N > 0 && x2_r1(N) > 0) {
      if (pf == 3) {
        using V = typename Cx<T>::V;
        constexpr int L = x2_lines(N);
        const dim3 grid(c->ny / (2 * L), c->nz);
        const size_t smem = (size_t)L * x2_line_elems(N) * sizeof(V);
        const auto tw = dev_plan<T>(c->plan_x).tw;
        if (p)
          k_fft_x2_fwd<T, N, false><<<grid, L * x2_r1(N), smem, s>>>(
              c->geo(), tw, c->d_sc, p, nullptr, nullptr, nullptr, var);
        else
          k_fft_x2_fwd<T, N, true><<<grid, L * x2_r1(N), smem, s>>>(c->geo(), tw, c->d_sc,
                                                                    nullptr, u, v, w, var);
        return cudaGetLastError();
      }
    }
    if constexpr (N > 0 && wp_base_lines(N) > 0) {
      if (pf == 2) {
        const WpLaunch<T, N, false> lc(c->ny, c->nz);
        const auto tw = dev_plan<T>(c->plan_x).tw;
        if (p)
          k_wfft_x_fwd<T, N, false><<<lc.grid, lc.block, lc.smem, s>>>(
              c->geo(), tw, c->d_sc, p, nullptr, nullptr, nullptr, var);
        else
          k_wfft_x_fwd<T, N, true><<<lc.grid, lc.block, lc.smem, s>>>(c->geo(), tw, c->d_sc,
                                                                       nullptr, u, v, w, var);
        return cudaGetLastError();
      }
    }
    return with_plan<N>(pfam, [&](auto PC) -> cudaError_t {
      constexpr int PL = decltype(PC)::value;
      if (p) {
        const int nl = c->fft_lines_x;
        k_fft_x_fwd<T, N, PL><<<c->grid_xf, 128, smem_x_fwd<T>(c->nx, nl), s>>>(
            c->geo(), dev_plan<T>(c->plan_x), nl, p, var);
      } else {
        const int nl = c->fft_lines_xf;
        dim3 grid(c->ny / (2 * nl), c->nz);
        k_fft_x_fwd_div<T, N, true, PL><<<grid, 256, fft_bytes<T>(c->nx, nl), s>>>(
            c->geo(), dev_plan<T>(c->plan_x), nl, c->d_sc, nullptr, u, v, w, var);
      }
      return cudaGetLastError();
    });
  });
}

template <class T>
cudaError_t fft_x_bwd_t(const plc_ctx *c, const T *var, T *p, bool fuse_bc, cudaStream_t s) {
  const int nl = c->fft_lines_x;
  const size_t sm = smem_x_bwd<T>(c->nx, nl);
  const double nf = 1.0 / (c->nx * c->ny);  // mod_fft.cc:57
  return with_size(c->nx, [&](auto NC) -> cudaError_t {
    constexpr int N = decltype(NC)::value;
    if constexpr (N > 0 && x2_r1(N) > 0) {
      if (c->fft_plan_x == 3) {
        using V = typename Cx<T>::V;
        constexpr int L = x2_lines(N);
        const dim3 grid(c->ny / (2 * L), c->nz);
        const size_t smem = (size_t)L * x2_line_elems(N) * sizeof(V);
        const auto tw = dev_plan<T>(c->plan_x).tw;
        if (fuse_bc)
          k_fft_x2_bwd<T, N, true><<<grid, L * x2_r1(N), smem, s>>>(c->geo(), tw, nf, var, p,
                                                                   c->order[SK_XB]);
        else
          k_fft_x2_bwd<T, N, false><<<grid, L * x2_r1(N), smem, s>>>(c->geo(), tw, nf, var, p,
                                                                    c->order[SK_XB]);
        return cudaGetLastError();
      }
    }
    if constexpr (N > 0 && wp_base_lines(N) > 0) {
      if (c->fft_plan_x == 2) {
        const WpLaunch<T, N, false> lc(c->ny, c->nz);
        const auto tw = dev_plan<T>(c->plan_x).tw;
        if (fuse_bc)
          k_wfft_x_bwd<T, N, true><<<lc.grid, lc.block, lc.smem, s>>>(c->geo(), tw, nf, var, p,
                                                                       c->order[SK_XB]);
        else
          k_wfft_x_bwd<T, N, false><<<lc.grid, lc.block, lc.smem, s>>>(c->geo(), tw, nf, var, p,
                                                                        c->order[SK_XB]);
        return cudaGetLastError();
      }
    }
    return with_plan<N>(c->fft_plan_x, [&](auto PC) -> cudaError_t {
      constexpr int PL = decltype(PC)::value;
      if (fuse_bc)
        k_fft_x_bwd<T, N, true, PL><<<c->grid_xb, 128, sm, s>>>(
            c->geo(), dev_plan<T>(c->plan_x), nl, nf, var, p, c->order[SK_XB]);
      else
        k_fft_x_bwd<T, N, false, PL><<<c->grid_xb, 128, sm, s>>>(
            c->geo(), dev_plan<T>(c->plan_x), nl, nf, var, p, c->order[SK_XB]);
      return cudaGetLastError();
    });
  });
}

template <class T>
cudaError_t fft_y_t(const plc_ctx *c, T *var, bool inverse, cudaStream_t s) {
  const int nl = c->fft_lines_y;
  const size_t sm = smem_y<T>(c->ny, nl);
  return with_size(c->ny, [&](auto NC) -> cudaError_t {
    constexpr int N = decltype(NC)::value;
    if constexpr (N > 0 && y2_r1(N) > 0) {
      if (c->fft_plan_y == 3) {
        using V = typename Cx<T>::V;
        constexpr int L = y2_lines<T>(), threads = L * y2_r1(N);
        const unsigned grid = (unsigned)(c->nx / (2 * L) * c->nz);
        const size_t smem = (size_t)L * N * sizeof(V);
        const auto tw = dev_plan<T>(c->plan_y).tw;
        if (inverse)
          k_fft_y2<T, N, true><<<grid, threads, smem, s>>>(c->nx, c->ny, c->nz, tw, var,
                                                           c->order[SK_YB]);
        else
          k_fft_y2<T, N, false><<<grid, threads, smem, s>>>(c->nx, c->ny, c->nz, tw, var,
                                                            c->order[SK_YF]);
        return cudaGetLastError();
      }
    }
    if constexpr (N > 0 && wp_base_lines(N) > 0) {
      if (c->fft_plan_y == 2) {
        const WpLaunch<T, N, true> lc(c->nx, c->nz);
        const auto tw = dev_plan<T>(c->plan_y).tw;
        if (inverse)
          k_wfft_y<T, N, true><<<lc.grid, lc.block, lc.smem, s>>>(c->nx, c->ny, c->nz, tw, var,
                                                                   c->order[SK_YB]);
        else
          k_wfft_y<T, N, false><<<lc.grid, lc.block, lc.smem, s>>>(c->nx, c->ny, c->nz, tw, var,
                                                                    c->order[SK_YF]);
        return cudaGetLastError();
      }
    }
    return with_plan<N>(c->fft_plan_y, [&](auto PC) -> cudaError_t {
      constexpr int PL = decltype(PC)::value;
      if (inverse)
        k_fft_y<T, N, true, PL><<<c->grid_y, 256, sm, s>>>(c->nx, c->ny, c->nz,
                                                            dev_plan<T>(c->plan_y), nl, var,
                                                            c->order[SK_YB]);
      else
        k_fft_y<T, N, false, PL><<<c->grid_y, 256, sm, s>>>(c->nx, c->ny, c->nz,
                                                             dev_plan<T>(c->plan_y), nl, var,
                                                             c->order[SK_YF]);
      return cudaGetLastError();
    });
  });
}

}  // namespace

cudaError_t launch_fft_x_fwd(const plc_ctx *c, const double *p, const double *u, const double *v,
                             const double *w, double *var, cudaStream_t s) {
  return fft_x_fwd_t<double>(c, p, u, v, w, var, s);
}
cudaError_t launch_fft_x_fwd(const plc_ctx *c, const float *u, const float *v, const float *w,
                             float *var, cudaStream_t s) {
  return fft_x_fwd_t<float>(c, nullptr, u, v, w, var, s);
}
cudaError_t launch_fft_x_bwd(const plc_ctx *c, const double *var, double *p, bool fuse_bc,
                             cudaStream_t s) {
  return fft_x_bwd_t<double>(c, var, p, fuse_bc, s);
}
cudaError_t launch_fft_x_bwd(const plc_ctx *c, const float *var, float *p, bool fuse_bc,
                             cudaStream_t s) {
  return fft_x_bwd_t<float>(c, var, p, fuse_bc, s);
}
cudaError_t launch_fft_y(const plc_ctx *c, double *var, bool inverse, cudaStream_t s) {
  return fft_y_t<double>(c, var, inverse, s);
}
cudaError_t launch_fft_y(const plc_ctx *c, float *var, bool inverse, cudaStream_t s) {
  return fft_y_t<float>(c, var, inverse, s);
}
// ---------------------------------------------------------------------------
// Autotuner of the transforms' tile sizes.  Each transform processes its
// lines independently, so the number of line pairs per tile changes only the
// speed, never the result.  For each transform the feasible tile sizes
// (divisors of the line-pair count, up to 16, within the device's shared
// memory) are timed on the context's own buffers and the fastest is kept.
// Call it while the fields hold no data to keep: it overwrites the spectral
// array and the pressure with transforms of the current fields.
// ---------------------------------------------------------------------------
namespace {
template <class T>
cudaError_t fft_autotune_t(plc_ctx *c, T *const *f, size_t dev_max, int sms) {
  const int nx = c->nx, ny = c->ny;
  cudaStream_t s = c->stream;
  cudaEvent_t e0, e1;
  cudaError_t e = cudaEventCreate(&e0);
  if (e != cudaSuccess) return e;
  if ((e = cudaEventCreate(&e1)) != cudaSuccess) {
    cudaEventDestroy(e0);
    return e;
  }
  auto time_of = [&](auto launch) -> float {
    // one untimed launch, then the best of three
    if (launch() != cudaSuccess) return -1.f;
    float best = -1.f;
    for (int r = 0; r < 3; ++r) {
      if (cudaEventRecord(e0, s) != cudaSuccess || launch() != cudaSuccess ||
          cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess)
        return -1.f;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (best < 0.f || ms < best) best = ms;
    }
    return best;
  };
  // tunes one line count *field over the divisors of `pairs` (multiples of
  // `step`) and, when `plan` is given and the length has two plan families
  // (`two`), the family *plan with it; `fits` says whether a value fits the
  // device
  auto tune = [&](int *field, int *plan, bool two, bool warp, bool f3, int pairs, int step,
                  auto fits, auto launch) {
    int best_d = *field, best_p = plan ? *plan : 0;
    float best_t = -1.f;
    const bool free_plan = plan && !c->fft_plans_pinned;
    const int p0 = free_plan ? 0 : (plan ? *plan : 0);
    const int p1 = free_plan ? (f3 ? 3 : (warp ? 2 : (two ? 1 : 0))) : p0;
    for (int pl = p0; pl <= p1; ++pl) {
      if ((pl == 1 && !two) || (pl == 2 && !warp) || (pl == 3 && !f3)) continue;
      if (plan) *plan = pl;
      if (pl >= 2) {
        // the warp-line and two-pass kernels have no tile size of their own
        const float t = time_of(launch);
        if (t >= 0.f && (best_t < 0.f || t < best_t)) {
          best_t = t;
          best_p = pl;
        }
        continue;
      }
      for (int d = step; d <= pairs && d <= 16; d += step) {
        if (pairs % d || !fits(d)) continue;
        *field = d;
        if (fft_grids_t<T>(c, dev_max, sms) != cudaSuccess) continue;
        const float t = time_of(launch);
        if (t >= 0.f && (best_t < 0.f || t < best_t)) {
          best_t = t;
          best_d = d;
          best_p = pl;
        }
      }
    }
    *field = best_d;
    if (plan) *plan = best_p;
    cudaGetLastError();  // a candidate that failed to launch leaves no error behind
  };
  T *u = f[PLC_U], *v = f[PLC_V], *w = f[PLC_W], *p = f[PLC_P], *spec = f[PLC_SPEC];
  // y: tile and plan family timed on a forward and an inverse transform
  tune(&c->fft_lines_y, &c->fft_plan_y, fft_has_two_plans(ny), fft_has_warp_plan(ny, nx),
       fft_has_y2_plan(ny, nx, sizeof(T)), nx / 2, sizeof(T) == 4 ? 2 : 1,
       [&](int d) { return smem_y<T>(ny, d) <= dev_max; },
       [&]() -> cudaError_t {
         cudaError_t r = launch_fft_y(c, spec, false, s);
         return r == cudaSuccess ? launch_fft_y(c, spec, true, s) : r;
       });
  // x: the plan family (shared by both x transforms) with the backward tile,
  // then the forward tile under that family
  tune(&c->fft_lines_x, &c->fft_plan_x, fft_has_two_plans(nx), fft_has_warp_plan(nx, ny),
       fft_has_x2_plan(nx, ny), ny / 2, 1,
       [&](int d) { return smem_x_bwd<T>(nx, d) <= dev_max && smem_x_fwd<T>(nx, d) <= dev_max; },
       [&]() -> cudaError_t { return launch_fft_x_bwd(c, spec, p, true, s); });
  tune(&c->fft_lines_xf, &c->fft_plan_xf, fft_has_two_plans(nx), fft_has_warp_plan(nx, ny),
       fft_has_x2_plan(nx, ny), ny / 2, 1,
       [&](int d) { return fft_bytes<T>(nx, d) <= dev_max; },
       [&]() -> cudaError_t {
         if constexpr (sizeof(T) == 8)
           return launch_fft_x_fwd(c, nullptr, u, v, w, spec, s);
         else
           return launch_fft_x_fwd(c, u, v, w, spec, s);
       });
  // the Thomas sweep: on chip or streaming, timed on the spectral array (the
  // choice changes speed, never results)
  if (c->nx % 32 == 0 && !c->trid_pinned) {
    float t_tile = -1.f, t_stream = -1.f;
    c->trid_tile = true;
    t_tile = time_of([&]() -> cudaError_t { return launch_trid(c, spec, s); });
    c->trid_tile = false;
    t_stream = time_of([&]() -> cudaError_t { return launch_trid(c, spec, s); });
    c->trid_tile = t_tile >= 0.f && (t_stream < 0.f || t_tile <= t_stream);
    cudaGetLastError();
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return fft_grids_t<T>(c, dev_max, sms);
}
}  // namespace

cudaError_t fft_autotune(plc_ctx *c) {
  const int sms = c->num_sms;
  int dev_max = 0;
  cudaError_t e = cudaDeviceGetAttribute(&dev_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
  if (e != cudaSuccess) return e;
  e = c->mixed ? fft_autotune_t<float>(c, c->f_field, (size_t)dev_max, sms)
               : fft_autotune_t<double>(c, c->d_field, (size_t)dev_max, sms);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  return e;
}

// Applies line counts chosen earlier (a re-initialised solver keeps the
// context's tuning).
cudaError_t fft_set_lines(plc_ctx *c, int lines_xf, int lines_x, int lines_y) {
  const int sms = c->num_sms;
  int dev_max = 0;
  cudaError_t e = cudaDeviceGetAttribute(&dev_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
  if (e != cudaSuccess) return e;
  c->fft_lines_xf = lines_xf;
  c->fft_lines_x = lines_x;
  c->fft_lines_y = lines_y;
  return c->mixed ? fft_grids_t<float>(c, (size_t)dev_max, sms)
                  : fft_grids_t<double>(c, (size_t)dev_max, sms);
}

// The on-chip sweep needs whole 32-system rows (nx a multiple of 32) and its
// columns within the device's shared memory; else the streaming sweep runs.
static bool trid_tile_ok(const plc_ctx *c, size_t elem) {
  return c->trid_tile && c->nx % 32 == 0 && trid_tile_smem(c->nz, elem) <= c->trid_smem_max;
}
cudaError_t launch_trid(const plc_ctx *c, double *var, cudaStream_t s) {
  const long long plane = (long long)c->nx * c->ny;
  if (trid_tile_ok(c, sizeof(double))) {
    k_trid_tile<<<(unsigned)(plane / 32), 32, trid_tile_smem(c->nz, sizeof(double)), s>>>(
        c->nx, c->ny, c->nz, c->d_rpiv, c->d_ac, c->d_ac + c->nz, var, c->d_err);
    return cudaGetLastError();
  }
  const int bs = 128;
  k_trid<<<(unsigned)((plane + bs - 1) / bs), bs, 0, s>>>(c->nx, c->ny, c->nz, c->d_rpiv,
                                                          c->d_ac, c->d_ac + c->nz, var);
  return cudaGetLastError();
}
cudaError_t launch_trid(const plc_ctx *c, float *var, cudaStream_t s) {
  const long long plane = (long long)c->nx * c->ny;
  if (trid_tile_ok(c, sizeof(float))) {
    k_trid_mixed_tile<<<(unsigned)(plane / 32), 32, trid_tile_smem(c->nz, sizeof(float)), s>>>(
        c->nx, c->ny, c->nz, c->d_rpiv32, c->d_ac32, c->d_ac32 + c->nz, c->d_rpiv, c->d_ac,
        c->d_ac + c->nz, var, c->d_low, c->d_err);
    return cudaGetLastError();
  }
  const int bs = 128;
  k_trid_mixed<<<(unsigned)((plane + bs - 1) / bs), bs, 0, s>>>(
      c->nx, c->ny, c->nz, c->d_rpiv32, c->d_ac32, c->d_ac32 + c->nz, c->d_rpiv, c->d_ac,
      c->d_ac + c->nz, var, c->d_low);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Launchers of the batched stages (mixed-form channels of an ensemble).
// ---------------------------------------------------------------------------
namespace {
// Channels of one batched transform launch: those whose line length has the
// same compiled plan (every length without one shares the runtime plan,
// N = 0), with the family and the tile of the batch plan, else of the
// group's largest channel and the largest tile all its channels admit (the
// warp-line family runs as family 0 in a batch; tiles only change the speed).
struct BatchGroup {
  int N = 0, PL = 0, nl = 1;
  size_t smem = 0;
  std::vector<plc_ctx *> ms;
};

int compiled_len(int n) {
  int key = 0;
  with_size(n, [&](auto NC) -> cudaError_t {
    key = decltype(NC)::value;
    return cudaSuccess;
  });
  return key;
}

// line pairs of a channel's tiles (the lines of the other axis) and the step
// of the tile sizes (FP32 y tiles span a multiple of 4 columns)
int batch_pairs(const plc_ctx *c, int dir) { return (dir == BATCH_Y ? c->nx : c->ny) / 2; }
int batch_step(int dir) { return dir == BATCH_Y ? 2 : 1; }
size_t batch_bytes(const plc_ctx *c, int dir, int d) {
  return dir == BATCH_Y ? smem_y<float>(c->ny, d)
                        : (dir == BATCH_XF ? fft_bytes<float>(c->nx, d) : smem_x_bwd<float>(c->nx, d));
}
// whether every channel of the group admits tiles of d line pairs
bool batch_tile_ok(const BatchGroup &g, int dir, int d) {
  if (d < batch_step(dir) || d % batch_step(dir)) return false;
  for (const plc_ctx *c : g.ms)
    if (batch_pairs(c, dir) % d || batch_bytes(c, dir, d) > c->trid_smem_max) return false;
  return true;
}
bool batch_family_ok(const BatchGroup &g, int dir, int pl) {
  if (pl == 0) return true;
  if (pl == 1) return g.N > 0 && plan_has24(g.N);
  if (pl != 3 || dir != BATCH_Y || g.N <= 0 || y2_r1(g.N) == 0) return false;
  for (const plc_ctx *c : g.ms)  // the two-pass y kernels take whole blocks of columns
    if (c->nx % (2 * y2_lines<float>())) return false;
  return true;
}
void batch_set_tile(BatchGroup &g, int dir, int nl) {
  g.nl = nl;
  g.smem = 0;
  for (const plc_ctx *c : g.ms) g.smem = std::max(g.smem, batch_bytes(c, dir, nl));
}

std::vector<BatchGroup> batch_groups(plc_ctx *const *cs, int n, int dir, const BatchPlan *bp) {
  std::vector<BatchGroup> out;
  for (int m = 0; m < n; ++m) {
    plc_ctx *c = cs[m];
    const int key = compiled_len(dir == BATCH_Y ? c->ny : c->nx);
    BatchGroup *g = nullptr;
    for (BatchGroup &x : out)
      if (x.N == key) g = &x;
    if (!g) {
      out.emplace_back();
      g = &out.back();
      g->N = key;
    }
    g->ms.push_back(c);
  }
  for (BatchGroup &g : out) {
    const plc_ctx *lead = g.ms[0];
    for (const plc_ctx *c : g.ms)
      if ((double)c->nx * c->ny * c->nz > (double)lead->nx * lead->ny * lead->nz) lead = c;
    int pl = dir == BATCH_Y ? lead->fft_plan_y
                            : (dir == BATCH_XF && lead->fft_plan_xf >= 0 ? lead->fft_plan_xf
                                                                         : lead->fft_plan_x);
    if (!batch_family_ok(g, dir, pl)) pl = 0;
    g.PL = pl;
    // default tile: the largest admitted by all the channels, up to 16 pairs
    // and 64 KB of shared memory
    int nl = 0;
    for (int d = 16; d >= batch_step(dir) && nl == 0; --d) {
      bool ok = batch_tile_ok(g, dir, d);
      for (const plc_ctx *c : g.ms) ok = ok && batch_bytes(c, dir, d) <= 64 * 1024;
      if (ok) nl = d;
    }
    if (nl == 0) nl = batch_step(dir);
    if (bp)
      for (const BatchPlan::Group &q : bp->dir[dir])
        if (q.len_key == g.N) {
          if (batch_family_ok(g, dir, q.pl)) g.PL = q.pl;
          if (batch_tile_ok(g, dir, q.nl)) nl = q.nl;
        }
    batch_set_tile(g, dir, nl);
  }
  return out;
}

// resident blocks of a kernel on the whole device
template <class K>
long long device_blocks(K kernel, int threads, size_t smem, int sms) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  return (long long)per_sm * sms;
}

// the persistent blocks of each channel: its tiles spread over its share of
// the launch's resident blocks (tiles per block alike for all the channels)
template <class B>
int share_blocks(B &b, const long long *tiles, long long resident) {
  long long tot = 0;
  for (int q = 0; q < b.n; ++q) tot += tiles[q];
  const long long per = std::max(1ll, (tot + resident - 1) / resident);
  int start = 0;
  for (int q = 0; q < b.n; ++q) {
    b.start[q] = start;
    b.m[q].vblocks = (int)std::max(1ll, (tiles[q] + per - 1) / per);
    start += b.m[q].vblocks;
  }
  b.start[b.n] = start;
  return start;
}

cudaError_t launch_group_xf(const BatchGroup &G, cudaStream_t s, bool pdl = false) {
  for (size_t q0 = 0; q0 < G.ms.size(); q0 += kBatchMax) {
    XfBatch b;
    std::memset(&b, 0, sizeof b);
    b.n = (int)std::min<size_t>(kBatchMax, G.ms.size() - q0);
    int tot = 0;
    for (int q = 0; q < b.n; ++q) {
      const plc_ctx *c = G.ms[q0 + q];
      XfMember &a = b.m[q];
      a.g = c->geo();
      a.P = dev_plan<float>(c->plan_x);
      a.nl = G.nl;
      a.gx = c->ny / (2 * G.nl);
      a.gy = c->nz;
      a.sc = c->d_sc;
      a.u = c->f_field[PLC_U];
      a.v = c->f_field[PLC_V];
      a.w = c->f_field[PLC_W];
      a.var = c->f_field[PLC_SPEC];
      b.start[q] = tot;
      tot += a.gx * a.gy;
    }
    b.start[b.n] = tot;
    const cudaError_t e = with_size(G.N, [&](auto NC) -> cudaError_t {
      constexpr int N = decltype(NC)::value;
      return with_plan<N>(G.PL, [&](auto PC) -> cudaError_t {
        constexpr int PL = decltype(PC)::value;
        return launch_batched(k_fft_x_fwd_div_batch<N, PL>, (unsigned)tot, dim3(256), G.smem, s, b,
                              pdl);
      });
    });
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_group_y(const BatchGroup &G, bool inverse, cudaStream_t s, bool pdl = false) {
  if (G.PL == 3) {
    return with_size(G.N, [&](auto NC) -> cudaError_t {
      constexpr int N = decltype(NC)::value;
      if constexpr (N > 0 && y2_r1(N) > 0) {
        constexpr int L = y2_lines<float>(), threads = L * y2_r1(N);
        const size_t smem = (size_t)L * N * sizeof(float2);
        for (size_t q0 = 0; q0 < G.ms.size(); q0 += kBatchMax) {
          Y2Batch b;
          std::memset(&b, 0, sizeof b);
          b.n = (int)std::min<size_t>(kBatchMax, G.ms.size() - q0);
          int tot = 0;
          for (int q = 0; q < b.n; ++q) {
            const plc_ctx *c = G.ms[q0 + q];
            b.m[q] = Y2Member{c->nx, c->ny, c->nz, c->order[inverse ? SK_YB : SK_YF],
                              dev_plan<float>(c->plan_y).tw, c->f_field[PLC_SPEC]};
            b.start[q] = tot;
            tot += c->nx / (2 * L) * c->nz;
          }
          b.start[b.n] = tot;
          const cudaError_t e =
              inverse ? launch_batched(k_fft_y2_batch<N, true>, (unsigned)tot, dim3(threads), smem,
                                       s, b, pdl)
                      : launch_batched(k_fft_y2_batch<N, false>, (unsigned)tot, dim3(threads), smem,
                                       s, b, pdl);
          if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
      } else {
        return cudaErrorInvalidValue;
      }
    });
  }
  for (size_t q0 = 0; q0 < G.ms.size(); q0 += kBatchMax) {
    YBatch b;
    std::memset(&b, 0, sizeof b);
    b.n = (int)std::min<size_t>(kBatchMax, G.ms.size() - q0);
    long long tiles[kBatchMax];
    for (int q = 0; q < b.n; ++q) {
      const plc_ctx *c = G.ms[q0 + q];
      YMember &a = b.m[q];
      a.nx = c->nx;
      a.ny = c->ny;
      a.nz = c->nz;
      a.nl = G.nl;
      a.rev = c->order[inverse ? SK_YB : SK_YF];
      a.P = dev_plan<float>(c->plan_y);
      a.var = c->f_field[PLC_SPEC];
      tiles[q] = (long long)(c->nx / (2 * G.nl)) * c->nz;
    }
    const int sms = G.ms[0]->device_sms;
    const cudaError_t e = with_size(G.N, [&](auto NC) -> cudaError_t {
      constexpr int N = decltype(NC)::value;
      return with_plan<N>(G.PL, [&](auto PC) -> cudaError_t {
        constexpr int PL = decltype(PC)::value;
        if (inverse) {
          const int tot =
              share_blocks(b, tiles, device_blocks(k_fft_y_batch<N, true, PL>, 256, G.smem, sms));
          return launch_batched(k_fft_y_batch<N, true, PL>, (unsigned)tot, dim3(256), G.smem, s, b,
                                pdl);
        } else {
          const int tot =
              share_blocks(b, tiles, device_blocks(k_fft_y_batch<N, false, PL>, 256, G.smem, sms));
          return launch_batched(k_fft_y_batch<N, false, PL>, (unsigned)tot, dim3(256), G.smem, s,
                                b, pdl);
        }
      });
    });
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_group_xb(const BatchGroup &G, cudaStream_t s, bool pdl = false) {
  for (size_t q0 = 0; q0 < G.ms.size(); q0 += kBatchMax) {
    XbBatch b;
    std::memset(&b, 0, sizeof b);
    b.n = (int)std::min<size_t>(kBatchMax, G.ms.size() - q0);
    long long tiles[kBatchMax];
    for (int q = 0; q < b.n; ++q) {
      const plc_ctx *c = G.ms[q0 + q];
      XbMember &a = b.m[q];
      a.g = c->geo();
      a.P = dev_plan<float>(c->plan_x);
      a.nl = G.nl;
      a.rev = c->order[SK_XB];
      a.nf = 1.0 / (c->nx * c->ny);  // mod_fft.cc:57
      a.var = c->f_field[PLC_SPEC];
      a.p = c->f_field[PLC_P];
      tiles[q] = (long long)(c->ny / (2 * G.nl)) * c->nz;
    }
    const int sms = G.ms[0]->device_sms;
    const cudaError_t e = with_size(G.N, [&](auto NC) -> cudaError_t {
      constexpr int N = decltype(NC)::value;
      return with_plan<N>(G.PL, [&](auto PC) -> cudaError_t {
        constexpr int PL = decltype(PC)::value;
        const int tot =
            share_blocks(b, tiles, device_blocks(k_fft_x_bwd_batch<N, PL>, 128, G.smem, sms));
        return launch_batched(k_fft_x_bwd_batch<N, PL>, (unsigned)tot, dim3(128), G.smem, s, b, pdl);
      });
    });
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}
}  // namespace

int fft_batch_groups(plc_ctx *const *cs, int n, bool ydir) {
  return (int)batch_groups(cs, n, ydir ? BATCH_Y : BATCH_XF, nullptr).size();
}

cudaError_t launch_fft_x_fwd_batch(plc_ctx *const *cs, int n, const BatchPlan *bp,
                                   const cudaStream_t *ss, int ns) {
  const std::vector<BatchGroup> gs = batch_groups(cs, n, BATCH_XF, bp);
  for (size_t gi = 0; gi < gs.size(); ++gi)
    if (cudaError_t e = launch_group_xf(gs[gi], ss[gi % ns], bp && bp->pdl)) return e;
  return cudaSuccess;
}

cudaError_t launch_fft_y_batch(plc_ctx *const *cs, int n, bool inverse, const BatchPlan *bp,
                               const cudaStream_t *ss, int ns) {
  const std::vector<BatchGroup> gs = batch_groups(cs, n, BATCH_Y, bp);
  for (size_t gi = 0; gi < gs.size(); ++gi)
    if (cudaError_t e = launch_group_y(gs[gi], inverse, ss[gi % ns], bp && bp->pdl)) return e;
  return cudaSuccess;
}

cudaError_t launch_fft_x_bwd_batch(plc_ctx *const *cs, int n, const BatchPlan *bp,
                                   const cudaStream_t *ss, int ns) {
  const std::vector<BatchGroup> gs = batch_groups(cs, n, BATCH_XB, bp);
  for (size_t gi = 0; gi < gs.size(); ++gi)
    if (cudaError_t e = launch_group_xb(gs[gi], ss[gi % ns], bp && bp->pdl)) return e;
  return cudaSuccess;
}

// The batch autotuner: for every group of every batched transform, the
// feasible families (only the channels' own where they are pinned) and
// tiles, one untimed launch and the best of three timed ones each; then the
// RK stages' z chunk (unless a channel pins its own) and resident blocks per
// SM, both stages timed.
cudaError_t batch_autotune(plc_ctx *const *cs, int n, cudaStream_t s, BatchPlan *bp) {
  cudaEvent_t e0, e1;
  cudaError_t e = cudaEventCreate(&e0);
  if (e != cudaSuccess) return e;
  if ((e = cudaEventCreate(&e1)) != cudaSuccess) {
    cudaEventDestroy(e0);
    return e;
  }
  auto time_of = [&](auto launch) -> float {
    if (launch() != cudaSuccess) return -1.f;
    float best = -1.f;
    for (int r = 0; r < 3; ++r) {
      if (cudaEventRecord(e0, s) != cudaSuccess || launch() != cudaSuccess ||
          cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess)
        return -1.f;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (best < 0.f || ms < best) best = ms;
    }
    return best;
  };
  bool fam_pinned = false, rk_pinned = false;
  for (int m = 0; m < n; ++m) {
    fam_pinned = fam_pinned || cs[m]->fft_plans_pinned;
    rk_pinned = rk_pinned || cs[m]->rk_pinned;
  }
  *bp = BatchPlan();
  for (int dir = 0; dir < 3; ++dir) {
    std::vector<BatchGroup> gs = batch_groups(cs, n, dir, nullptr);
    for (BatchGroup &G : gs) {
      BatchPlan::Group best{G.N, G.PL, G.nl};
      float best_t = -1.f;
      for (int pl = 0; pl <= 3; ++pl) {
        if (!batch_family_ok(G, dir, pl) || (fam_pinned && pl != G.PL)) continue;
        G.PL = pl;
        for (int d = batch_step(dir); d <= 16; d += batch_step(dir)) {
          if (!batch_tile_ok(G, dir, d) || (pl == 3 && d != G.nl)) continue;  // no tile in family 3
          batch_set_tile(G, dir, d);
          const float t = time_of([&]() -> cudaError_t {
            if (dir == BATCH_XF) return launch_group_xf(G, s);
            if (dir == BATCH_XB) return launch_group_xb(G, s);
            const cudaError_t r = launch_group_y(G, false, s);
            return r == cudaSuccess ? launch_group_y(G, true, s) : r;
          });
          if (t >= 0.f && (best_t < 0.f || t < best_t)) {
            best_t = t;
            best = BatchPlan::Group{G.N, pl, d};
          }
        }
      }
      bp->dir[dir].push_back(best);
    }
  }
  // the Thomas sweep: streamed, or with the columns on chip (as the channels
  // have it where PLC_TRID pins it)
  bp->trid_tile = false;
  bool trid_pinned = false, trid_tiles = true;
  for (int m = 0; m < n; ++m) {
    trid_pinned = trid_pinned || cs[m]->trid_pinned;
    trid_tiles = trid_tiles && cs[m]->trid_tile;
  }
  if (trid_pinned) {
    bp->trid_tile = trid_tiles && trid_tile_batch_ok(cs, n);
  } else if (trid_tile_batch_ok(cs, n)) {
    const float ts = time_of([&]() { return launch_trid_batch(cs, n, false, s); });
    const float tt = time_of([&]() { return launch_trid_batch(cs, n, true, s); });
    bp->trid_tile = tt >= 0.f && (ts < 0.f || tt < ts);
  }
  {
    float best_t = -1.f;
    for (int minb = 3; minb <= 4; ++minb)
      for (int kc : kRkChunks) {
        if (rk_pinned && kc != kRkChunks[0]) continue;  // the channels' own chunks
        const int k = rk_pinned ? 0 : kc;
        const float t = time_of([&]() -> cudaError_t {
          const cudaError_t r = launch_rk_batch(cs, n, 1, k, minb, s);
          return r == cudaSuccess ? launch_rk_batch(cs, n, 2, k, minb, s) : r;
        });
        if (t >= 0.f && (best_t < 0.f || t < best_t)) {
          best_t = t;
          bp->rk_kchunk = k;
          bp->rk_minb = minb;
        }
      }
  }
  cudaGetLastError();  // a candidate that failed to launch leaves no error behind
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return cudaSuccess;
}

// whether every channel admits the on-chip sweep (whole blocks of 32 systems,
// its column in shared memory)
bool trid_tile_batch_ok(plc_ctx *const *cs, int n) {
  for (int m = 0; m < n; ++m)
    if (cs[m]->nx % 32 || trid_tile_smem(cs[m]->nz, sizeof(float)) > cs[m]->trid_smem_max)
      return false;
  return n > 0;
}

cudaError_t launch_trid_batch(plc_ctx *const *cs, int n, bool tile, cudaStream_t s, bool pdl) {
  if (tile && trid_tile_batch_ok(cs, n)) {
    for (int q0 = 0; q0 < n; q0 += kBatchMax) {
      TrtBatch b;
      std::memset(&b, 0, sizeof b);
      b.n = std::min(kBatchMax, n - q0);
      int tot = 0, nzmax = 0;
      for (int q = 0; q < b.n; ++q) {
        const plc_ctx *c = cs[q0 + q];
        b.m[q] = TrtMember{c->nx,     c->ny,     c->nz,           c->d_rpiv32, c->d_ac32,
                           c->d_ac32 + c->nz, c->d_rpiv, c->d_ac, c->d_ac + c->nz,
                           c->f_field[PLC_SPEC], c->d_low, c->d_err};
        b.start[q] = tot;
        tot += (int)((long long)c->nx * c->ny / 32);
        nzmax = std::max(nzmax, c->nz);
      }
      b.start[b.n] = tot;
      const cudaError_t e = launch_batched(k_trid_mixed_tile_batch, (unsigned)tot, dim3(32),
                                           trid_tile_smem(nzmax, sizeof(float)), s, b, pdl);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  for (int q0 = 0; q0 < n; q0 += kBatchMax) {
    TrBatch b;
    std::memset(&b, 0, sizeof b);
    b.n = std::min(kBatchMax, n - q0);
    int tot = 0;
    for (int q = 0; q < b.n; ++q) {
      const plc_ctx *c = cs[q0 + q];
      b.m[q] = TrMember{c->nx,     c->ny,         c->nz,  c->d_rpiv32, c->d_ac32,
                        c->d_ac32 + c->nz, c->d_rpiv, c->d_ac, c->d_ac + c->nz,
                        c->f_field[PLC_SPEC], c->d_low};
      b.start[q] = tot;
      tot += (int)(((long long)c->nx * c->ny + 127) / 128);
    }
    b.start[b.n] = tot;
    const cudaError_t e = launch_batched(k_trid_mixed_batch, (unsigned)tot, dim3(128), 0, s, b, pdl);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace plc
