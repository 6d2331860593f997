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

}  // namespace plc
