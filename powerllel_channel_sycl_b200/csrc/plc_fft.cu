// Batched real FFTs and the wall-normal tridiagonal solve of the Poisson
// projection (FP64).
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
//  * The complex FFT is a mixed-radix (8, 4, 2, 3) Stockham transform between
//    two shared-memory buffers, one butterfly per thread and pass; element e
//    of a line lives at e + e/8 to spread the strided accesses over banks.
//  * Both transforms are unscaled; the backward x transform multiplies by
//    1/(nx*ny) (mod_fft.cc:57,116-117) and, in the fused step, also writes
//    the pressure halos (updateBoundP, mod_updateBound.cc:287-330).
//
// The tridiagonal solve (ssolve_trid, mod_poisson_solver.cc:317-357) is a
// Thomas sweep per (kx,ky) system, one thread per system, coalesced over kx,
// with the pre-factored reciprocal pivots read from a table indexed by the
// distinct wavenumber pair.

#include <cuda_runtime.h>

#include "plc_device.cuh"
#include "plc_internal.h"

namespace plc {

namespace {

struct FftDev {
  int n, npass;
  int radix[16];
  const double2 *tw;
};

__device__ __forceinline__ int padi(int e) { return e + (e >> 3); }

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ double2 rot90(double2 a) {
  return INV ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

template <int R, bool INV>
struct Dft;

template <bool INV>
struct Dft<2, INV> {
  __device__ __forceinline__ static void run(double2 (&v)[2]) {
    const double2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <bool INV>
struct Dft<4, INV> {
  __device__ __forceinline__ static void run(double2 (&v)[4]) {
    const double2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    const double2 t2 = cadd(v[1], v[3]), t3 = rot90<INV>(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  }
};

template <bool INV>
struct Dft<8, INV> {
  __device__ __forceinline__ static void run(double2 (&v)[8]) {
    const double s = 0.70710678118654752440;  // 1/sqrt(2)
    double2 e[4] = {v[0], v[2], v[4], v[6]};
    double2 o[4] = {v[1], v[3], v[5], v[7]};
    Dft<4, INV>::run(e);
    Dft<4, INV>::run(o);
    // o[m] *= W8^m, W8 = exp(-+ i pi/4)
    double2 x = o[1];
    o[1] = INV ? make_double2(s * (x.x - x.y), s * (x.x + x.y))
               : make_double2(s * (x.x + x.y), s * (x.y - x.x));
    o[2] = rot90<INV>(o[2]);
    x = o[3];
    o[3] = INV ? make_double2(-s * (x.x + x.y), s * (x.x - x.y))
               : make_double2(s * (x.y - x.x), -s * (x.x + x.y));
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      v[m] = cadd(e[m], o[m]);
      v[m + 4] = csub(e[m], o[m]);
    }
  }
};

template <bool INV>
struct Dft<3, INV> {
  __device__ __forceinline__ static void run(double2 (&v)[3]) {
    const double h = 0.86602540378443864676;  // sqrt(3)/2
    const double2 t1 = cadd(v[1], v[2]);
    const double2 t2 = make_double2(v[0].x - 0.5 * t1.x, v[0].y - 0.5 * t1.y);
    const double2 d = csub(v[1], v[2]);
    const double2 t3 = INV ? make_double2(-h * d.y, h * d.x) : make_double2(h * d.y, -h * d.x);
    v[0] = cadd(v[0], t1);
    v[1] = cadd(t2, t3);
    v[2] = csub(t2, t3);
  }
};

// One Stockham pass of radix R over nl lines of length n (line stride LS).
template <int R, bool INV>
__device__ __forceinline__ void fft_pass(const double2 *__restrict__ src, double2 *__restrict__ dst,
                                         int nl, int n, int LS, int Ns,
                                         const double2 *__restrict__ tw) {
  const int nb = n / R;
  const int tot = nl * nb;
  const int tws = n / (Ns * R);
  for (int b = threadIdx.x; b < tot; b += blockDim.x) {
    const int l = b / nb;
    const int j = b - l * nb;
    const double2 *s = src + l * LS;
    double2 *d = dst + l * LS;
    const int jm = j % Ns;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = s[padi(j + r * nb)];
    if (jm != 0) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        const double2 w = __ldg(tw + r * jm * tws);
        v[r] = INV ? cmulc(v[r], w) : cmul(v[r], w);
      }
    }
    Dft<R, INV>::run(v);
    const int idxD = (j / Ns) * Ns * R + jm;
#pragma unroll
    for (int r = 0; r < R; ++r) d[padi(idxD + r * Ns)] = v[r];
  }
}

// Complex FFT of nl lines held in A; returns the buffer holding the result.
template <bool INV>
__device__ double2 *fft_run(double2 *A, double2 *B, int nl, int LS, const FftDev &P) {
  int Ns = 1;
  for (int p = 0; p < P.npass; ++p) {
    const int R = P.radix[p];
    switch (R) {
      case 8: fft_pass<8, INV>(A, B, nl, P.n, LS, Ns, P.tw); break;
      case 4: fft_pass<4, INV>(A, B, nl, P.n, LS, Ns, P.tw); break;
      case 2: fft_pass<2, INV>(A, B, nl, P.n, LS, Ns, P.tw); break;
      default: fft_pass<3, INV>(A, B, nl, P.n, LS, Ns, P.tw); break;
    }
    __syncthreads();
    double2 *t = A;
    A = B;
    B = t;
    Ns *= R;
  }
  return A;
}

__host__ __device__ __forceinline__ int line_stride(int n) { return n + (n >> 3) + 1; }

// Packed output q of the two real lines encoded in Z (line of length n):
// A for the real part sequence, B for the imaginary part sequence.
__device__ __forceinline__ void unpack_pair(const double2 *Z, int n, int q, double &a, double &b) {
  const int m = (q == 0) ? 0 : ((q == 1) ? (n >> 1) : (q >> 1));
  const int part = (q < 2) ? 0 : (q & 1);
  const double2 zm = Z[padi(m)];
  const double2 zc = Z[padi(m == 0 ? 0 : n - m)];
  if (part == 0) {
    a = (zm.x + zc.x) * 0.5;
    b = (zm.y + zc.y) * 0.5;
  } else {
    a = (zm.y - zc.y) * 0.5;
    b = (zc.x - zm.x) * 0.5;
  }
}

// Builds Z_m and Z_{n-m} (0 <= m <= n/2) of the pair whose packed spectra are
// ra[] (real sequence a) and rb[] (real sequence b), read with stride `st`.
__device__ __forceinline__ void pack_pair(double2 *Z, int n, int m, const double *ra,
                                          const double *rb, int st) {
  double reA, imA, reB, imB;
  if (m == 0) {
    reA = ra[0];
    reB = rb[0];
    imA = imB = 0.0;
  } else if (m == (n >> 1)) {
    reA = ra[st];
    reB = rb[st];
    imA = imB = 0.0;
  } else {
    reA = ra[(2 * m) * st];
    imA = ra[(2 * m + 1) * st];
    reB = rb[(2 * m) * st];
    imB = rb[(2 * m + 1) * st];
  }
  Z[padi(m)] = make_double2(reA - imB, imA + reB);
  if (m != 0 && m != (n >> 1)) Z[padi(n - m)] = make_double2(reA + imB, reB - imA);
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

// Forward x transform: rows (j0+2l, j0+2l+1) of plane k -> packed spectra.
// FUSED: the rows are div(u)/dt evaluated on the fly (calcRHS).
template <bool FUSED>
__global__ void __launch_bounds__(256) k_fft_x_fwd(Geo g, FftDev P, int nl,
                                                   const StepConst *__restrict__ sc,
                                                   const double *__restrict__ p,
                                                   const double *__restrict__ u,
                                                   const double *__restrict__ v,
                                                   const double *__restrict__ w,
                                                   double *__restrict__ var) {
  extern __shared__ double2 smem[];
  const int n = g.nx, LS = line_stride(n);
  double2 *A = smem, *B = smem + nl * LS;
  const int j0 = blockIdx.x * 2 * nl;  // 0-based row in the plane
  const int k = blockIdx.y;            // 0-based plane
  double dti = 0, dtidxi = 0, dtidyi = 0, dzfi = 0;
  if (FUSED) {
    dti = sc->dti;
    dtidxi = sc->dtidxi;
    dtidyi = sc->dtidyi;
    dzfi = __ldg(g.dzf_inv + k + 1);
  }
  for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
    const int l = e / n, t = e - l * n;
    const long long ca = g.at(t + 1, j0 + 2 * l + 1, k + 1);
    const long long cb = ca + g.X;
    double a, b;
    if (FUSED) {
      a = div_dt(u, v, w, ca, g.X, g.XY, dtidxi, dtidyi, dti, dzfi);
      b = div_dt(u, v, w, cb, g.X, g.XY, dtidxi, dtidyi, dti, dzfi);
    } else {
      a = p[ca];
      b = p[cb];
    }
    A[l * LS + padi(t)] = make_double2(a, b);
  }
  __syncthreads();
  const double2 *Z = fft_run<false>(A, B, nl, LS, P);
  for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
    const int l = e / n, q = e - l * n;
    double a, b;
    unpack_pair(Z + l * LS, n, q, a, b);
    const long long row = (long long)k * g.ny + j0 + 2 * l;
    var[row * n + q] = a;
    var[(row + 1) * n + q] = b;
  }
}

// Backward x transform: packed spectra -> p interior scaled by nf; with
// FUSE_BC the pressure halos are written as well (updateBoundP).
template <bool FUSE_BC>
__global__ void __launch_bounds__(256) k_fft_x_bwd(Geo g, FftDev P, int nl, double nf,
                                                   const double *__restrict__ var, double *p) {
  extern __shared__ double2 smem[];
  const int n = g.nx, LS = line_stride(n);
  double2 *A = smem, *B = smem + nl * LS;
  double *raw = reinterpret_cast<double *>(B);  // 2*nl rows of n doubles
  const int j0 = blockIdx.x * 2 * nl;
  const int k = blockIdx.y;
  const double *src = var + ((long long)k * g.ny + j0) * n;
  for (int e = threadIdx.x; e < 2 * nl * n; e += blockDim.x) raw[e] = src[e];
  __syncthreads();
  const int half = n >> 1;
  for (int e = threadIdx.x; e < nl * (half + 1); e += blockDim.x) {
    const int l = e / (half + 1), m = e - l * (half + 1);
    pack_pair(A + l * LS, n, m, raw + (2 * l) * n, raw + (2 * l + 1) * n, 1);
  }
  __syncthreads();
  const double2 *Z = fft_run<true>(A, B, nl, LS, P);
  for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
    const int l = e / n, t = e - l * n;
    const double2 z = Z[l * LS + padi(t)];
    const double a = nf * z.x, b = nf * z.y;
    const int i = t + 1, ja = j0 + 2 * l + 1, kk = k + 1;
    if (FUSE_BC) {
      store_with_halo(p, g, i, ja, kk, a, BC_ZEROGRAD, 0.0);
      store_with_halo(p, g, i, ja + 1, kk, b, BC_ZEROGRAD, 0.0);
    } else {
      const long long ca = g.at(i, ja, kk);
      p[ca] = a;
      p[ca + g.X] = b;
    }
  }
}

// y transform in place on the spectral array: columns i0..i0+2nl-1 of plane k.
template <bool INV>
__global__ void __launch_bounds__(256) k_fft_y(int nx, int ny, FftDev P, int nl,
                                               double *__restrict__ var) {
  extern __shared__ double2 smem[];
  const int n = ny, LS = line_stride(n), TX = 2 * nl;
  double2 *A = smem, *B = smem + nl * LS;
  const int i0 = blockIdx.x * TX;
  double *plane = var + (long long)blockIdx.y * nx * ny + i0;
  if (!INV) {
    for (int e = threadIdx.x; e < n * TX; e += blockDim.x) {
      const int t = e / TX, c = e - t * TX;
      reinterpret_cast<double *>(A + (c >> 1) * LS + padi(t))[c & 1] = plane[(long long)t * nx + c];
    }
    __syncthreads();
    const double2 *Z = fft_run<false>(A, B, nl, LS, P);
    for (int e = threadIdx.x; e < n * TX; e += blockDim.x) {
      const int q = e / TX, c = e - q * TX;
      double a, b;
      unpack_pair(Z + (c >> 1) * LS, n, q, a, b);
      plane[(long long)q * nx + c] = (c & 1) ? b : a;
    }
  } else {
    double *raw = reinterpret_cast<double *>(B);  // n rows of TX doubles
    for (int e = threadIdx.x; e < n * TX; e += blockDim.x) {
      const int t = e / TX, c = e - t * TX;
      raw[e] = plane[(long long)t * nx + c];
    }
    __syncthreads();
    const int half = n >> 1;
    for (int e = threadIdx.x; e < nl * (half + 1); e += blockDim.x) {
      const int l = e / (half + 1), m = e - l * (half + 1);
      pack_pair(A + l * LS, n, m, raw + 2 * l, raw + 2 * l + 1, TX);
    }
    __syncthreads();
    const double2 *Z = fft_run<true>(A, B, nl, LS, P);
    for (int e = threadIdx.x; e < n * TX; e += blockDim.x) {
      const int t = e / TX, c = e - t * TX;
      const double2 z = Z[(c >> 1) * LS + padi(t)];
      plane[(long long)t * nx + c] = (c & 1) ? z.y : z.x;
    }
  }
}

// Thomas sweep per (i,j) system with the reciprocal pivot table
// rpiv[(k*(ny/2+1) + my)*(nx/2+1) + mx]; the reference's divisions by b
// become multiplications by 1/b (mod_poisson_solver.cc:334-354).
__global__ void __launch_bounds__(128) k_trid(int nx, int ny, int nz,
                                              const double *__restrict__ rpiv,
                                              const double *__restrict__ a,
                                              const double *__restrict__ c,
                                              double *__restrict__ var) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const long long plane = (long long)nx * ny;
  if (t >= plane) return;
  const int i = t % nx, j = t / nx;
  const int mx = (i == 0) ? 0 : ((i == 1) ? (nx >> 1) : (i >> 1));
  const int my = (j == 0) ? 0 : ((j == 1) ? (ny >> 1) : (j >> 1));
  const int MX = (nx >> 1) + 1;
  const long long PS = (long long)MX * ((ny >> 1) + 1);
  const double *rp = rpiv + (long long)my * MX + mx;
  double *q = var + t;
  double prev = q[0];
#pragma unroll 4
  for (int k = 1; k < nz; ++k) {
    double cur = q[k * plane];
    cur -= (__ldg(a + k) * __ldg(rp + (k - 1) * PS)) * prev;
    q[k * plane] = cur;
    prev = cur;
  }
  prev *= __ldg(rp + (nz - 1) * PS);
  q[(nz - 1) * plane] = prev;
#pragma unroll 4
  for (int k = nz - 2; k >= 0; --k) {
    const double cur = (q[k * plane] - __ldg(c + k) * prev) * __ldg(rp + k * PS);
    q[k * plane] = cur;
    prev = cur;
  }
}

FftDev dev_plan(const FftPlan &p) {
  FftDev d;
  d.n = p.n;
  d.npass = p.npass;
  for (int r = 0; r < 16; ++r) d.radix[r] = p.radix[r];
  d.tw = p.tw;
  return d;
}

}  // namespace

size_t fft_smem_bytes(int n, int lines) {
  return 2ull * (size_t)lines * (size_t)line_stride(n) * sizeof(double2);
}

// Raises the dynamic shared-memory limit of every FFT kernel (once per process).
cudaError_t fft_configure(size_t max_bytes) {
  cudaError_t e;
#define PLC_SMEM(kern)                                                                    \
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_bytes); \
  if (e != cudaSuccess) return e;
  PLC_SMEM(k_fft_x_fwd<true>);
  PLC_SMEM(k_fft_x_fwd<false>);
  PLC_SMEM(k_fft_x_bwd<true>);
  PLC_SMEM(k_fft_x_bwd<false>);
  PLC_SMEM(k_fft_y<true>);
  PLC_SMEM(k_fft_y<false>);
#undef PLC_SMEM
  return cudaSuccess;
}

cudaError_t launch_fft_x_fwd(const plc_ctx *c, const double *p, const double *u, const double *v,
                             const double *w, double *var, cudaStream_t s) {
  const int nl = c->fft_lines_x;
  dim3 grid(c->ny / (2 * nl), c->nz);
  const size_t sm = fft_smem_bytes(c->nx, nl);
  if (p)
    k_fft_x_fwd<false><<<grid, 256, sm, s>>>(c->geo(), dev_plan(c->plan_x), nl, c->d_sc, p,
                                              nullptr, nullptr, nullptr, var);
  else
    k_fft_x_fwd<true><<<grid, 256, sm, s>>>(c->geo(), dev_plan(c->plan_x), nl, c->d_sc, nullptr,
                                             u, v, w, var);
  return cudaGetLastError();
}

cudaError_t launch_fft_x_bwd(const plc_ctx *c, const double *var, double *p, bool fuse_bc,
                             cudaStream_t s) {
  const int nl = c->fft_lines_x;
  dim3 grid(c->ny / (2 * nl), c->nz);
  const size_t sm = fft_smem_bytes(c->nx, nl);
  const double nf = 1.0 / (c->nx * c->ny);  // mod_fft.cc:57
  if (fuse_bc)
    k_fft_x_bwd<true><<<grid, 256, sm, s>>>(c->geo(), dev_plan(c->plan_x), nl, nf, var, p);
  else
    k_fft_x_bwd<false><<<grid, 256, sm, s>>>(c->geo(), dev_plan(c->plan_x), nl, nf, var, p);
  return cudaGetLastError();
}

cudaError_t launch_fft_y(const plc_ctx *c, double *var, bool inverse, cudaStream_t s) {
  const int nl = c->fft_lines_y;
  dim3 grid(c->nx / (2 * nl), c->nz);
  const size_t sm = fft_smem_bytes(c->ny, nl);
  if (inverse)
    k_fft_y<true><<<grid, 256, sm, s>>>(c->nx, c->ny, dev_plan(c->plan_y), nl, var);
  else
    k_fft_y<false><<<grid, 256, sm, s>>>(c->nx, c->ny, dev_plan(c->plan_y), nl, var);
  return cudaGetLastError();
}

cudaError_t launch_trid(const plc_ctx *c, double *var, cudaStream_t s) {
  const long long plane = (long long)c->nx * c->ny;
  const int bs = 128;
  k_trid<<<(unsigned)((plane + bs - 1) / bs), bs, 0, s>>>(c->nx, c->ny, c->nz, c->d_rpiv,
                                                          c->d_ac, c->d_ac + c->nz, var);
  return cudaGetLastError();
}

}  // namespace plc
