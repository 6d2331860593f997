// Device helpers shared by the kernels of libplc.so.
#pragma once

#include <cuda_runtime.h>

#include "plc_internal.h"

namespace plc {

// kinds of wall rule used by the fused halo writes
enum BcKind { BC_CENTRED = 0, BC_FACE = 1, BC_ZEROGRAD = 2 };

// Write value `val` of interior point (i,j,k) of field q together with its
// periodic images and, on the first/last interior plane, the wall ghosts.
// T is the storage type of the field (double, or float in the mixed form);
// the ghost rule is evaluated in T.
template <class T>
static __device__ __forceinline__ void store_with_halo(T *q, const Geo &g, int i, int j, int k,
                                                       T val, int kind, T bc) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int ib = (i == nx) ? 0 : ((i == 1) ? nx + 1 : -1);
  const int jb = (j == ny) ? 0 : ((j == 1) ? ny + 1 : -1);
  T v = val;
  if (kind == BC_FACE && k == nz) v = bc;  // w(nz) = bcvalue
  T gv;
  if (kind == BC_CENTRED)
    gv = T(2) * bc - v;
  else if (kind == BC_FACE)
    gv = bc;
  else
    gv = v;
  auto put = [&](int kk, T x) {
    q[g.at(i, j, kk)] = x;
    if (ib >= 0) q[g.at(ib, j, kk)] = x;
    if (jb >= 0) {
      q[g.at(i, jb, kk)] = x;
      if (ib >= 0) q[g.at(ib, jb, kk)] = x;
    }
  };
  put(k, v);
  if (k == 1) put(0, gv);
  if (k == nz) put(nz + 1, gv);
}

// The halo images of one interior column (i, j): the offsets from a point of
// the column to its periodic x image, its y image and its xy corner image
// (0 where the column has none).  Computed once per column, so that a kernel
// writing many planes of the column pays for the image rules once.  The
// offsets are within one plane (at most ny*pitch elements), so 32 bits hold
// them.
// Division by a divisor that is fixed for a kernel's lifetime, by one
// multiply-high, an add and a shift: q = (umulhi(e, mul) + e) >> shr with
// shr = ceil(log2 d) and mul = floor(2^32 (2^shr - d) / d) + 1 (the
// round-up multiplier method of Granlund and Montgomery, "Division by
// invariant integers using multiplication", 1994).  Exact for 1 <= d < 2^31
// and 0 <= e < 2^31.  A runtime integer division costs about twenty
// instructions; the index loops of the transforms divide once per element.
struct FastDiv {
  unsigned mul, shr;
  __host__ __device__ explicit FastDiv(unsigned d) {
    shr = 0;
    while ((1u << shr) < d) ++shr;
    mul = (unsigned)(((1ull << 32) * ((1ull << shr) - d)) / d + 1);
  }
  __device__ __forceinline__ int div(int e) const {
    return (int)((__umulhi((unsigned)e, mul) + (unsigned)e) >> shr);
  }
};

struct HaloCol {
  int dx, dy;
};
static __device__ __forceinline__ HaloCol halo_col(const Geo &g, int i, int j) {
  HaloCol h;
  h.dx = (i == g.nx) ? -g.nx : ((i == 1) ? g.nx : 0);
  h.dy = (j == g.ny) ? -g.ny * g.X : ((j == 1) ? g.ny * g.X : 0);
  return h;
}
template <class T>
static __device__ __forceinline__ void store_col(T *q, long long c, const HaloCol &h, T x) {
  q[c] = x;
  if (h.dx) q[c + h.dx] = x;
  if (h.dy) {
    q[c + h.dy] = x;
    if (h.dx) q[c + (h.dx + h.dy)] = x;
  }
}
// The image and ghost writes of store_point: rare (boundary columns and the
// wall planes), so kept out of line, off the kernels' common path.
template <class T>
static __device__ __noinline__ void store_images(T *q, const Geo &g, HaloCol h, long long c,
                                                 int k, T v, int kind, T bc) {
  if (h.dx) q[c + h.dx] = v;
  if (h.dy) {
    q[c + h.dy] = v;
    if (h.dx) q[c + (h.dx + h.dy)] = v;
  }
  if (k == 1 || k == g.nz) {
    T gv;
    if (kind == BC_CENTRED)
      gv = T(2) * bc - v;
    else if (kind == BC_FACE)
      gv = bc;
    else
      gv = v;
    if (k == 1) store_col(q, c - g.XY, h, gv);
    if (k == g.nz) store_col(q, c + g.XY, h, gv);
  }
}

// The same writes as store_with_halo for the point at halo'd index c of
// column h, plane k.
template <class T>
static __device__ __forceinline__ void store_point(T *q, const Geo &g, const HaloCol &h,
                                                   long long c, int k, T val, int kind, T bc) {
  T v = val;
  if (kind == BC_FACE && k == g.nz) v = bc;  // w(nz) = bcvalue
  q[c] = v;
  if ((h.dx | h.dy) != 0 || k == 1 || k == g.nz) store_images(q, g, h, c, k, v, kind, bc);
}

// The same writes inline: for kernels where boundary columns are common (the
// small channels of an ensemble), whose warps take this path together -- the
// image stores are predicated per lane, the ghost writes uniform per plane.
template <class T>
static __device__ __forceinline__ void store_point_inline(T *q, const Geo &g, const HaloCol &h,
                                                          long long c, int k, T val, int kind,
                                                          T bc) {
  T v = val;
  if (kind == BC_FACE && k == g.nz) v = bc;  // w(nz) = bcvalue
  store_col(q, c, h, v);
  if (k == 1 || k == g.nz) {
    T gv;
    if (kind == BC_CENTRED)
      gv = T(2) * bc - v;
    else if (kind == BC_FACE)
      gv = bc;
    else
      gv = v;
    store_col(q, k == 1 ? c - g.XY : c + g.XY, h, gv);
  }
}

// Block coordinates of a kernel body that runs as one block of a batched
// launch over several channels of an ensemble: the block's place in its
// channel's share of the grid.
struct VBlk {
  int x_, y_, z_, gx_, gy_, gz_;
  __device__ __forceinline__ int x() const { return x_; }
  __device__ __forceinline__ int y() const { return y_; }
  __device__ __forceinline__ int z() const { return z_; }
  __device__ __forceinline__ int gx() const { return gx_; }
  __device__ __forceinline__ int gy() const { return gy_; }
  __device__ __forceinline__ int gz() const { return gz_; }
  // block b (linear, x fastest) of a grid gx x gy x gz
  static __device__ __forceinline__ VBlk of(int b, int gx, int gy, int gz) {
    const int t = b / gx;
    return VBlk{b - t * gx, t % gy, t / gy, gx, gy, gz};
  }
};

// The channel of block b in a batched launch: start[m] <= b < start[m + 1]
// (start in the launch's parameters, n channels).
static __device__ __forceinline__ int batch_member(const int *start, int n, int b) {
  int m = 0;
  while (m + 1 < n && b >= start[m + 1]) ++m;
  return m;
}

// First statement of a batched kernel, which may be launched with
// programmatic stream serialisation (its blocks then become resident while
// the kernels it depends on drain): wait until those kernels have completed
// and their writes are visible, then allow the next kernel's launch to
// begin.  Both instructions are no-ops in a plain launch.  Every block runs
// it before anything else, so that this grid's completion implies its
// predecessors' completion for the kernels that in turn wait on it.
static __device__ __forceinline__ void batch_grid_sync() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

}  // namespace plc
