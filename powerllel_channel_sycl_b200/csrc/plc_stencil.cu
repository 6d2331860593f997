// Stencil, boundary, forcing and reduction kernels of the FP64 time step.
//
// Fields use the reference's halo'd layout (one ghost cell per side, x
// fastest).  Kernels that end a stage of the fused step ("fused BC") also
// write the halo images of every interior value they produce, so the
// separate boundary update of the reference (mod_updateBound.cc) costs no
// extra pass over the field:
//   x and y periodic images:  (0,j)=(nx,j), (nx+1,j)=(1,j), same in y and for
//                             the corners (the y self-exchange of
//                             mod_type.hh:219-289 followed by the x copy of
//                             mod_updateBound.cc:32-73);
//   z walls, centred u and v: q(0) = 2*bc - q(1), q(nz+1) = 2*bc - q(nz),
//                             bc = -u_crf for u and 0 for v (:75-144);
//   z walls, face w:          w(0) = w(nz) = w(nz+1) = 0;
//   pressure:                 p(0) = p(1), p(nz+1) = p(nz) (:146-180).

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <type_traits>

#include "plc_device.cuh"
#include "plc_internal.h"

namespace plc {

namespace {

constexpr int BX = 32, BY = 8;

struct Rhs3 {
  double u, v, w;
};

// Operand access straight from global memory (read-only path).
struct GlobalAcc {
  const double *__restrict__ qu;
  const double *__restrict__ qv;
  const double *__restrict__ qw;
  long long c, X, XY;
  __device__ __forceinline__ double U(int di, int dj, int dk) const {
    return __ldg(qu + c + di + dj * X + dk * XY);
  }
  __device__ __forceinline__ double V(int di, int dj, int dk) const {
    return __ldg(qv + c + di + dj * X + dk * XY);
  }
  __device__ __forceinline__ double W(int di, int dj, int dk) const {
    return __ldg(qw + c + di + dj * X + dk * XY);
  }
};

// Wall-normal metric factors of plane k used by the momentum right-hand
// side: dzf(k-1..k+1), 1/dzf(k..k+1), 1/dzc(k-1..k).
struct alignas(16) ZMetric {
  double dzf_m, dzf_0, dzf_p, dzfi_0, dzfi_p, dzci_m, dzci_0, pad;
};
__device__ __forceinline__ ZMetric zmetric(const Geo &g, int k) {
  return ZMetric{__ldg(g.dzf + k - 1),     __ldg(g.dzf + k),         __ldg(g.dzf + k + 1),
                 __ldg(g.dzf_inv + k),     __ldg(g.dzf_inv + k + 1), __ldg(g.dzc_inv + k - 1),
                 __ldg(g.dzc_inv + k),     0.0};
}

// (visc - conv) of the three momentum components at (i,j,k),
// mod_calcVel.cc:61-125 (the same expression for RK1 and RK2).  Acc gives the
// operand values at offsets (di,dj,dk) from the point.  CRF = false drops the
// convecting-frame terms conv + 0.5*u_crf*(qe - qw)/dx, which add an exact
// zero when u_crf = 0.
template <bool CRF = true, class Acc>
__device__ __forceinline__ Rhs3 momentum_rhs(const Geo &g, double u_crf, const Acc &a,
                                             const ZMetric &z) {
  const double _dx_inv = g.dx_inv, _dy_inv = g.dy_inv, _re_inv = g.re_inv;
#define U(di, dj, dk) a.U(di, dj, dk)
#define V(di, dj, dk) a.V(di, dj, dk)
#define W(di, dj, dk) a.W(di, dj, dk)
  const double dzf_m = z.dzf_m, dzf_0 = z.dzf_0, dzf_p = z.dzf_p;
  const double dzfi_0 = z.dzfi_0, dzfi_p = z.dzfi_p;
  const double dzci_m = z.dzci_m, dzci_0 = z.dzci_0;
  double uw, ue, us, un, ub, ut;
  double ww, we, ws, wn, wb, wt;
  double vw, ve, vs, vn, vb, vt;
  double dqw, dqe, dqs, dqn, dqb, dqt;
  double conv, visc;
  Rhs3 r;
  const double u000 = U(0, 0, 0), v000 = V(0, 0, 0), w000 = W(0, 0, 0);
  // u component
  {
    const double up00 = U(1, 0, 0), um00 = U(-1, 0, 0), u0p0 = U(0, 1, 0),
                 u0m0 = U(0, -1, 0), u00p = U(0, 0, 1), u00m = U(0, 0, -1);
    ue = (u000 + up00);
    uw = (um00 + u000);
    un = (u000 + u0p0);
    us = (u0m0 + u000);
    ut = (u000 * dzf_p + u00p * dzf_0) * dzci_0;
    ub = (u000 * dzf_m + u00m * dzf_0) * dzci_m;
    vn = (v000 + V(1, 0, 0));
    vs = (V(0, -1, 0) + V(1, -1, 0));
    wt = (w000 + W(1, 0, 0));
    wb = (W(0, 0, -1) + W(1, 0, -1));
    dqe = (up00 - u000) * _dx_inv;
    dqw = (u000 - um00) * _dx_inv;
    dqn = (u0p0 - u000) * _dy_inv;
    dqs = (u000 - u0m0) * _dy_inv;
    dqt = (u00p - u000) * dzci_0;
    dqb = (u000 - u00m) * dzci_m;
    conv = 0.25 * ((ue * ue - uw * uw) * _dx_inv + (un * vn - us * vs) * _dy_inv +
                   (ut * wt - ub * wb) * dzfi_0);
    if (CRF) conv = conv + 0.5 * u_crf * (ue - uw) * _dx_inv;
    visc = ((dqe - dqw) * _dx_inv + (dqn - dqs) * _dy_inv + (dqt - dqb) * dzfi_0) * _re_inv;
    r.u = visc - conv;
  }
  // v component
  {
    const double vp00 = V(1, 0, 0), vm00 = V(-1, 0, 0), v0p0 = V(0, 1, 0),
                 v0m0 = V(0, -1, 0), v00p = V(0, 0, 1), v00m = V(0, 0, -1);
    ve = (v000 + vp00);
    vw = (vm00 + v000);
    vn = (v000 + v0p0);
    vs = (v0m0 + v000);
    vt = (v000 * dzf_p + v00p * dzf_0) * dzci_0;
    vb = (v000 * dzf_m + v00m * dzf_0) * dzci_m;
    ue = (u000 + U(0, 1, 0));
    uw = (U(-1, 0, 0) + U(-1, 1, 0));
    wt = (w000 + W(0, 1, 0));
    wb = (W(0, 0, -1) + W(0, 1, -1));
    dqe = (vp00 - v000) * _dx_inv;
    dqw = (v000 - vm00) * _dx_inv;
    dqn = (v0p0 - v000) * _dy_inv;
    dqs = (v000 - v0m0) * _dy_inv;
    dqt = (v00p - v000) * dzci_0;
    dqb = (v000 - v00m) * dzci_m;
    conv = 0.25 * ((ue * ve - uw * vw) * _dx_inv + (vn * vn - vs * vs) * _dy_inv +
                   (wt * vt - wb * vb) * dzfi_0);
    if (CRF) conv = conv + 0.5 * u_crf * (ve - vw) * _dx_inv;
    visc = ((dqe - dqw) * _dx_inv + (dqn - dqs) * _dy_inv + (dqt - dqb) * dzfi_0) * _re_inv;
    r.v = visc - conv;
  }
  // w component
  {
    const double wp00 = W(1, 0, 0), wm00 = W(-1, 0, 0), w0p0 = W(0, 1, 0),
                 w0m0 = W(0, -1, 0), w00p = W(0, 0, 1), w00m = W(0, 0, -1);
    we = (w000 + wp00);
    ww = (wm00 + w000);
    wn = (w000 + w0p0);
    ws = (w0m0 + w000);
    wt = (w000 + w00p);
    wb = (w000 + w00m);
    ue = (u000 * dzf_p + U(0, 0, 1) * dzf_0) * dzci_0;
    uw = (U(-1, 0, 0) * dzf_p + U(-1, 0, 1) * dzf_0) * dzci_0;
    vn = (v000 * dzf_p + V(0, 0, 1) * dzf_0) * dzci_0;
    vs = (V(0, -1, 0) * dzf_p + V(0, -1, 1) * dzf_0) * dzci_0;
    dqe = (wp00 - w000) * _dx_inv;
    dqw = (w000 - wm00) * _dx_inv;
    dqn = (w0p0 - w000) * _dy_inv;
    dqs = (w000 - w0m0) * _dy_inv;
    dqt = (w00p - w000) * dzfi_p;
    dqb = (w000 - w00m) * dzfi_0;
    conv = 0.25 * ((ue * we - uw * ww) * _dx_inv + (vn * wn - vs * ws) * _dy_inv +
                   (wt * wt - wb * wb) * dzci_0);
    if (CRF) conv = conv + 0.5 * u_crf * (we - ww) * _dx_inv;
    visc = ((dqe - dqw) * _dx_inv + (dqn - dqs) * _dy_inv + (dqt - dqb) * dzci_0) * _re_inv;
    r.w = visc - conv;
  }
#undef U
#undef V
#undef W
  return r;
}

// The z-face terms of the three components at one point, carried from plane
// k (top face) to plane k+1 (bottom face).  With the reference's expressions
// evaluated without contraction they are bit for bit the same numbers:
//   ub(k+1) = (u(k+1)*dzf(k) + u(k)*dzf(k+1))*dzc_inv(k)   (mod_calcVel.cc:66)
//   ut(k)   = (u(k)*dzf(k+1) + u(k+1)*dzf(k))*dzc_inv(k)   (mod_calcVel.cc:65)
// are the same two rounded products added in the other order (addition is
// commutative), wb(k+1) and wt(k) the same sum, and
//   dqb(k+1) = (u(k+1) - u(k))*dzc_inv(k) = dqt(k)          (mod_calcVel.cc:75-76)
// likewise for v and for w (wt = w(k) + w(k+1), dqt with dzf_inv(k+1)).
// Tu = ut*wt, Tv = wt*vt, Tw = wt*wt are the products of the conv terms;
// Du, Dv, Dw the dqt of the visc terms.
struct ZFace64 {
  double Tu, Tv, Tw, Du, Dv, Dw;
};

// momentum_rhs with the bottom-face terms taken from the plane below (bot;
// with FIRST evaluated from plane k-1 as momentum_rhs does) and the top-face
// terms returned in top: the same operations on the same operands, so the
// result is bit-identical to momentum_rhs.
template <bool CRF, bool FIRST, class Acc>
__device__ __forceinline__ Rhs3 momentum_rhs_c(const Geo &g, double u_crf, const Acc &a,
                                               const ZMetric &z, const ZFace64 &bot_in,
                                               ZFace64 &top) {
  const double _dx_inv = g.dx_inv, _dy_inv = g.dy_inv, _re_inv = g.re_inv;
#define U(di, dj, dk) a.U(di, dj, dk)
#define V(di, dj, dk) a.V(di, dj, dk)
#define W(di, dj, dk) a.W(di, dj, dk)
  const double dzf_m = z.dzf_m, dzf_0 = z.dzf_0, dzf_p = z.dzf_p;
  const double dzfi_0 = z.dzfi_0, dzfi_p = z.dzfi_p;
  const double dzci_m = z.dzci_m, dzci_0 = z.dzci_0;
  double uw, ue, us, un, ut;
  double ww, we, ws, wn, wt;
  double vw, ve, vs, vn, vt;
  double dqw, dqe, dqs, dqn;
  double conv, visc;
  Rhs3 r;
  const double u000 = U(0, 0, 0), v000 = V(0, 0, 0), w000 = W(0, 0, 0);
  ZFace64 bot = bot_in;
  if (FIRST) {
    const double u00m = U(0, 0, -1), v00m = V(0, 0, -1), w00m = W(0, 0, -1);
    const double ub = (u000 * dzf_m + u00m * dzf_0) * dzci_m;
    const double wbu = (W(0, 0, -1) + W(1, 0, -1));
    const double vb = (v000 * dzf_m + v00m * dzf_0) * dzci_m;
    const double wbv = (W(0, 0, -1) + W(0, 1, -1));
    const double wbw = (w000 + w00m);
    bot.Tu = ub * wbu;
    bot.Tv = wbv * vb;
    bot.Tw = wbw * wbw;
    bot.Du = (u000 - u00m) * dzci_m;
    bot.Dv = (v000 - v00m) * dzci_m;
    bot.Dw = (w000 - w00m) * dzfi_0;
  }
  // u component
  {
    const double up00 = U(1, 0, 0), um00 = U(-1, 0, 0), u0p0 = U(0, 1, 0),
                 u0m0 = U(0, -1, 0), u00p = U(0, 0, 1);
    ue = (u000 + up00);
    uw = (um00 + u000);
    un = (u000 + u0p0);
    us = (u0m0 + u000);
    ut = (u000 * dzf_p + u00p * dzf_0) * dzci_0;
    vn = (v000 + V(1, 0, 0));
    vs = (V(0, -1, 0) + V(1, -1, 0));
    wt = (w000 + W(1, 0, 0));
    dqe = (up00 - u000) * _dx_inv;
    dqw = (u000 - um00) * _dx_inv;
    dqn = (u0p0 - u000) * _dy_inv;
    dqs = (u000 - u0m0) * _dy_inv;
    top.Du = (u00p - u000) * dzci_0;
    top.Tu = ut * wt;
    conv = 0.25 * ((ue * ue - uw * uw) * _dx_inv + (un * vn - us * vs) * _dy_inv +
                   (top.Tu - bot.Tu) * dzfi_0);
    if (CRF) conv = conv + 0.5 * u_crf * (ue - uw) * _dx_inv;
    visc = ((dqe - dqw) * _dx_inv + (dqn - dqs) * _dy_inv + (top.Du - bot.Du) * dzfi_0) * _re_inv;
    r.u = visc - conv;
  }
  // v component
  {
    const double vp00 = V(1, 0, 0), vm00 = V(-1, 0, 0), v0p0 = V(0, 1, 0),
                 v0m0 = V(0, -1, 0), v00p = V(0, 0, 1);
    ve = (v000 + vp00);
    vw = (vm00 + v000);
    vn = (v000 + v0p0);
    vs = (v0m0 + v000);
    vt = (v000 * dzf_p + v00p * dzf_0) * dzci_0;
    ue = (u000 + U(0, 1, 0));
    uw = (U(-1, 0, 0) + U(-1, 1, 0));
    wt = (w000 + W(0, 1, 0));
    dqe = (vp00 - v000) * _dx_inv;
    dqw = (v000 - vm00) * _dx_inv;
    dqn = (v0p0 - v000) * _dy_inv;
    dqs = (v000 - v0m0) * _dy_inv;
    top.Dv = (v00p - v000) * dzci_0;
    top.Tv = wt * vt;
    conv = 0.25 * ((ue * ve - uw * vw) * _dx_inv + (vn * vn - vs * vs) * _dy_inv +
                   (top.Tv - bot.Tv) * dzfi_0);
    if (CRF) conv = conv + 0.5 * u_crf * (ve - vw) * _dx_inv;
    visc = ((dqe - dqw) * _dx_inv + (dqn - dqs) * _dy_inv + (top.Dv - bot.Dv) * dzfi_0) * _re_inv;
    r.v = visc - conv;
  }
  // w component
  {
    const double wp00 = W(1, 0, 0), wm00 = W(-1, 0, 0), w0p0 = W(0, 1, 0),
                 w0m0 = W(0, -1, 0), w00p = W(0, 0, 1);
    we = (w000 + wp00);
    ww = (wm00 + w000);
    wn = (w000 + w0p0);
    ws = (w0m0 + w000);
    wt = (w000 + w00p);
    ue = (u000 * dzf_p + U(0, 0, 1) * dzf_0) * dzci_0;
    uw = (U(-1, 0, 0) * dzf_p + U(-1, 0, 1) * dzf_0) * dzci_0;
    vn = (v000 * dzf_p + V(0, 0, 1) * dzf_0) * dzci_0;
    vs = (V(0, -1, 0) * dzf_p + V(0, -1, 1) * dzf_0) * dzci_0;
    dqe = (wp00 - w000) * _dx_inv;
    dqw = (w000 - wm00) * _dx_inv;
    dqn = (w0p0 - w000) * _dy_inv;
    dqs = (w000 - w0m0) * _dy_inv;
    top.Dw = (w00p - w000) * dzfi_p;
    top.Tw = wt * wt;
    conv = 0.25 * ((ue * we - uw * ww) * _dx_inv + (vn * wn - vs * ws) * _dy_inv +
                   (top.Tw - bot.Tw) * dzci_0);
    if (CRF) conv = conv + 0.5 * u_crf * (we - ww) * _dx_inv;
    visc = ((dqe - dqw) * _dx_inv + (dqn - dqs) * _dy_inv + (top.Dw - bot.Dw) * dzci_0) * _re_inv;
    r.w = visc - conv;
  }
#undef U
#undef V
#undef W
  return r;
}

// RK1 (STAGE 1, mod_calcVel.cc:27-129):  o = q + dt*F(q)
// RK2 (STAGE 2, mod_calcVel.cc:140-242): o = (q + dt*F(q) + o)*0.5, q = u1
template <int STAGE, bool FUSE>
__global__ void __launch_bounds__(BX *BY) k_rk(Geo g, const StepConst *__restrict__ sc,
                                               double u_crf, const double *__restrict__ qu,
                                               const double *__restrict__ qv,
                                               const double *__restrict__ qw, double *ou,
                                               double *ov, double *ow) {
  const int i = blockIdx.x * BX + threadIdx.x + 1;
  const int j = blockIdx.y * BY + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  if (i > g.nx || j > g.ny) return;
  const double dt = sc->dt;
  const long long c = g.at(i, j, k);
  const Rhs3 r = momentum_rhs(g, u_crf, GlobalAcc{qu, qv, qw, c, g.X, g.XY}, zmetric(g, k));
  double nu, nv, nw;
  if (STAGE == 1) {
    nu = qu[c] + dt * r.u;
    nv = qv[c] + dt * r.v;
    nw = qw[c] + dt * r.w;
  } else {
    nu = (qu[c] + dt * r.u + ou[c]) * 0.5;
    nv = (qv[c] + dt * r.v + ov[c]) * 0.5;
    nw = (qw[c] + dt * r.w + ow[c]) * 0.5;
  }
  if (FUSE) {
    store_with_halo(ou, g, i, j, k, nu, BC_CENTRED, 0.0 - u_crf);
    store_with_halo(ov, g, i, j, k, nv, BC_CENTRED, 0.0);
    store_with_halo(ow, g, i, j, k, nw, BC_FACE, 0.0);
  } else {
    ou[c] = nu;
    ov[c] = nv;
    ow[c] = nw;
  }
}

// ---------------------------------------------------------------------------
// RK stages as z-marching kernels fed by TMA.
//
// A block of 32 x 8 threads owns a 32 x 16 tile of interior (i, j) columns --
// each thread two rows of one column -- and a chunk of z planes.  For each
// operand field the (32+2) x (16+2) halo tile of every plane is brought into a
// 6-slot shared-memory ring by one 3-D bulk tensor copy (cp.async.bulk.tensor,
// completion on a "full" mbarrier), three planes ahead of the plane being
// computed, so every operand value crosses HBM once per block and the copies
// overlap the arithmetic.  There is no block-wide barrier in the
// march: every thread waits on the full barrier of the plane it is about to
// read, each warp arrives on the slot's "empty" mbarrier when it has read the
// plane for the last time, and thread 0 refills a slot once its empty barrier
// completed.  Every wait is bounded (a timeout raises *err and the thread
// leaves the march; the others' waits run out in turn).  The expression trees
// are those of momentum_rhs, so the results are bit-identical to the
// global-load kernel above.
// ---------------------------------------------------------------------------
constexpr int RX = 32, TY = 8, RY = 2 * TY;    // interior tile 32 x 16: two rows per thread
constexpr int HX = RX + 2, HY = RY + 2;         // halo tile (34 x 18)
constexpr int PLANE = HX * HY;                  // doubles per field-plane
constexpr int SLOT = ((PLANE * 8 + 127) / 128) * 128 / 8;  // doubles, 128-B aligned
constexpr int NSLOT = 6;
constexpr unsigned PLANE_TX_BYTES = 3u * PLANE * 8u;  // three fields per plane
constexpr long long kWaitLimit = 1ll << 22;            // try_wait polls before giving up

__device__ __forceinline__ unsigned smem_addr(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void tma_load_plane(double *dst, const CUtensorMap *map, int x, int y,
                                               int z, unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z),
      "r"(smem_addr(bar))
      : "memory");
}

// Operand access from the three plane slots (k-1, k, k+1) of each field: the
// u slots start at base, the v and w slots NSLOT*SLOT and 2*NSLOT*SLOT later.
struct SmemAcc {
  const double *base;
  int off[3];  // slot offset of planes k-1, k, k+1 plus the thread's point
  __device__ __forceinline__ double U(int di, int dj, int dk) const {
    return base[off[dk + 1] + di + dj * HX];
  }
  __device__ __forceinline__ double V(int di, int dj, int dk) const {
    return base[NSLOT * SLOT + off[dk + 1] + di + dj * HX];
  }
  __device__ __forceinline__ double W(int di, int dj, int dk) const {
    return base[2 * NSLOT * SLOT + off[dk + 1] + di + dj * HX];
  }
};

constexpr int KCHUNK_TMA = 32;  // planes per block (at most)
size_t rk_tma_smem_bytes() {
  return (size_t)3 * NSLOT * SLOT * 8 + KCHUNK_TMA * sizeof(ZMetric) + 2 * NSLOT * 8 + 128;
}

template <int STAGE, bool FUSE, bool CRF>
__global__ void __launch_bounds__(RX *TY, 2)
    k_rk_tma(const __grid_constant__ CUtensorMap mu, const __grid_constant__ CUtensorMap mv,
             const __grid_constant__ CUtensorMap mw, Geo g, const StepConst *__restrict__ sc,
             double u_crf, double *ou, double *ov, double *ow, int kchunk, int *err, int rev) {
  extern __shared__ unsigned char smem_raw[];
  double *base = reinterpret_cast<double *>(
      (reinterpret_cast<unsigned long long>(smem_raw) + 127ull) & ~127ull);
  double *slot_u = base, *slot_v = base + NSLOT * SLOT, *slot_w = base + 2 * NSLOT * SLOT;
  ZMetric *zrow = reinterpret_cast<ZMetric *>(base + 3 * NSLOT * SLOT);  // planes kb..ke
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(zrow + KCHUNK_TMA);
  unsigned long long *empty = bar + NSLOT;
  constexpr unsigned kWarps = RX * TY / 32;

  // the first stage carries the z-face terms from plane to plane (ZFace64;
  // RK1 0.940 -> 0.876 ms at 768 x 384 x 256, bit-identical); the second,
  // which also holds the base values of two planes, measured slower with
  // the carry (1.07 -> 1.24 ms) and evaluates them afresh
  constexpr bool kCarry = (STAGE == 1);
  ZFace64 fa_c{}, fb_c{};
  const int tid = threadIdx.x;
  const int tx = tid & (RX - 1), ty = tid / RX;
  const int x0 = blockIdx.x * RX, y0 = blockIdx.y * RY;  // halo'd coords of the tile corner
  // rows ja and jb = ja + 1 of column i; the second row shares the first's
  // north-face terms as its south-face terms
  const int i = x0 + tx + 1, ja = y0 + 2 * ty + 1, jb = ja + 1;
  const bool act_a = (i <= g.nx) && (ja <= g.ny);
  const bool act_b = act_a && (jb <= g.ny);
  const int zc = rev ? (int)gridDim.z - 1 - (int)blockIdx.z : (int)blockIdx.z;  // plane order
  const int kb = zc * kchunk + 1;
  const int ke = min(kb + kchunk - 1, g.nz);
  const int plast = ke + 1;  // last plane to bring in

  auto issue = [&](int p) {  // thread 0 only
    const int rel = p - (kb - 1);
    const int s = rel % NSLOT;
    mbar_expect_tx(&bar[s], PLANE_TX_BYTES);
    tma_load_plane(slot_u + s * SLOT, &mu, x0, y0, p, &bar[s]);
    tma_load_plane(slot_v + s * SLOT, &mv, x0, y0, p, &bar[s]);
    tma_load_plane(slot_w + s * SLOT, &mw, x0, y0, p, &bar[s]);
  };
  // bounded waits for plane p's copy to land (full) or to be read by every
  // warp for the last time (empty)
  auto wait_on = [&](unsigned long long *b, int p, long long limit) -> bool {
    const int rel = p - (kb - 1);
    const unsigned parity = (unsigned)((rel / NSLOT) & 1);
    for (long long it = 0; it < limit; ++it)
      if (mbar_try_wait(&b[rel % NSLOT], parity)) return true;
    return false;
  };

  int issued = min(kb + 2, plast);  // thread 0: the last plane copied
  if (tid == 0) {
    for (int s = 0; s < NSLOT; ++s) {
      mbar_init(&bar[s], 1);
      mbar_init(&empty[s], kWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int p = kb - 1; p <= issued; ++p) issue(p);
  }
  // metric factors of the block's planes, read once (a plane's row is four
  // 16-byte shared loads, the same for every thread)
  for (int k = kb + tid; k <= ke; k += blockDim.x) zrow[k - kb] = zmetric(g, k);
  __syncthreads();

  const double dt = sc->dt;
  const long long X = g.X, XY = g.XY;
  long long c = g.at(act_a ? i : 1, act_a ? ja : 1, kb);  // point a; point b is c + X
  // RK2 base values (u, v, w) of plane k at points a and b
  double ba[3] = {0.0, 0.0, 0.0}, bb[3] = {0.0, 0.0, 0.0};
  if (STAGE == 2 && act_a) {
    ba[0] = ou[c];
    ba[1] = ov[c];
    ba[2] = ow[c];
    if (act_b) {
      bb[0] = ou[c + X];
      bb[1] = ov[c + X];
      bb[2] = ow[c + X];
    }
  }
  const HaloCol ha = halo_col(g, i, ja), hb = halo_col(g, i, jb);
  const bool xy_edge = (ha.dx | ha.dy | hb.dx | hb.dy) != 0;  // images in x or y
  const int o = (2 * ty + 1) * HX + (tx + 1);                 // point a in a slot
  int sm = 0, s0 = 1, sp = 2;                                 // slots of planes k-1, k, k+1
  for (int k = kb; k <= ke; ++k) {
    bool ok = true;
    if (tid == 0 && k + 3 <= plast) {
      // the slot of plane k+3 last held plane k+3-NSLOT
      if (k + 3 - NSLOT >= kb - 1) ok = wait_on(empty, k + 3 - NSLOT, kWaitLimit);
      if (ok) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue(k + 3);
        issued = k + 3;
      }
    }
    if (ok && k == kb) ok = wait_on(bar, kb - 1, kWaitLimit) && wait_on(bar, kb, kWaitLimit);
    ok = ok && wait_on(bar, k + 1, kWaitLimit);
    if (!ok) {
      atomicExch(err, 1);
      break;  // the other threads' waits run out as well
    }
    double na[3] = {0.0, 0.0, 0.0}, nb[3] = {0.0, 0.0, 0.0};  // base values of plane k+1
    if (STAGE == 2 && act_a && k < ke) {
      na[0] = ou[c + XY];
      na[1] = ov[c + XY];
      na[2] = ow[c + XY];
      if (act_b) {
        nb[0] = ou[c + X + XY];
        nb[1] = ov[c + X + XY];
        nb[2] = ow[c + X + XY];
      }
    }
    if (act_a) {
      SmemAcc a;
      a.base = slot_u;
      a.off[0] = sm * SLOT + o;
      a.off[1] = s0 * SLOT + o;
      a.off[2] = sp * SLOT + o;
      SmemAcc b = a;
      b.off[0] += HX;
      b.off[1] += HX;
      b.off[2] += HX;
      const ZMetric zm = zrow[k - kb];
      Rhs3 ra, rb;
      if constexpr (kCarry) {
        if (k == kb) {
          ra = momentum_rhs_c<CRF, true>(g, u_crf, a, zm, fa_c, fa_c);
          rb = momentum_rhs_c<CRF, true>(g, u_crf, b, zm, fb_c, fb_c);
        } else {
          ra = momentum_rhs_c<CRF, false>(g, u_crf, a, zm, fa_c, fa_c);
          rb = momentum_rhs_c<CRF, false>(g, u_crf, b, zm, fb_c, fb_c);
        }
      } else {
        ra = momentum_rhs<CRF>(g, u_crf, a, zm);
        rb = momentum_rhs<CRF>(g, u_crf, b, zm);
      }
      const double fa[3] = {ra.u, ra.v, ra.w}, fb[3] = {rb.u, rb.v, rb.w};
      const double qa[3] = {a.U(0, 0, 0), a.V(0, 0, 0), a.W(0, 0, 0)};
      const double qb[3] = {b.U(0, 0, 0), b.V(0, 0, 0), b.W(0, 0, 0)};
      double va[3], vb[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if (STAGE == 1) {
          va[d] = qa[d] + dt * fa[d];
          vb[d] = qb[d] + dt * fb[d];
        } else {
          va[d] = (qa[d] + dt * fa[d] + ba[d]) * 0.5;
          vb[d] = (qb[d] + dt * fb[d] + bb[d]) * 0.5;
        }
      }
      if (FUSE && (xy_edge || k == 1 || k == g.nz)) {
        store_point(ou, g, ha, c, k, va[0], BC_CENTRED, 0.0 - u_crf);
        store_point(ov, g, ha, c, k, va[1], BC_CENTRED, 0.0);
        store_point(ow, g, ha, c, k, va[2], BC_FACE, 0.0);
        if (act_b) {
          store_point(ou, g, hb, c + X, k, vb[0], BC_CENTRED, 0.0 - u_crf);
          store_point(ov, g, hb, c + X, k, vb[1], BC_CENTRED, 0.0);
          store_point(ow, g, hb, c + X, k, vb[2], BC_FACE, 0.0);
        }
      } else {  // no image or ghost to write
        ou[c] = va[0];
        ov[c] = va[1];
        ow[c] = va[2];
        if (act_b) {
          ou[c + X] = vb[0];
          ov[c + X] = vb[1];
          ow[c + X] = vb[2];
        }
      }
    }
    // this warp is done with plane k-1 (slot sm)
    __syncwarp();
    if ((tid & 31) == 0) mbar_arrive(&empty[sm]);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      ba[d] = na[d];
      bb[d] = nb[d];
    }
    sm = s0;
    s0 = sp;
    sp = (sp + 1 == NSLOT) ? 0 : sp + 1;
    c += XY;
  }
  if (tid == 0) {
    // no copy may still be writing into shared memory when the block leaves
    // (after an error; on the normal path every copy has been waited for)
    for (int p = max(kb - 1, issued - NSLOT + 1); p <= issued; ++p) wait_on(bar, p, 1 << 20);
  }
}

// calcRHS, mod_calcRHS.cc:7-33
__global__ void __launch_bounds__(BX *BY) k_calc_rhs(Geo g, const StepConst *__restrict__ sc,
                                                     const double *__restrict__ u,
                                                     const double *__restrict__ v,
                                                     const double *__restrict__ w,
                                                     double *__restrict__ rhs) {
  const int i = blockIdx.x * BX + threadIdx.x + 1;
  const int j = blockIdx.y * BY + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  if (i > g.nx || j > g.ny) return;
  const double dti = sc->dti, dtidxi = sc->dtidxi, dtidyi = sc->dtidyi;
  const long long c = g.at(i, j, k);
  rhs[c] = (u[c] - u[c - 1]) * dtidxi + (v[c] - v[c - g.X]) * dtidyi +
           (w[c] - w[c - g.XY]) * dti * __ldg(g.dzf_inv + k);
}

// ---------------------------------------------------------------------------
// Order-independent block and grid sums.  Values are accumulated in
// double-double (Knuth's error-free TwoSum); the rounded total hi + lo is the
// correctly rounded sum except when the exact sum lies within ~n*2^-106 of a
// rounding boundary, so it does not depend on the summation order and equals
// the CPU restatement's value bit for bit.
// ---------------------------------------------------------------------------
struct DD {
  double hi, lo;
};

__device__ __forceinline__ void dd_add(DD &a, double x) {
  const double s = a.hi + x;
  const double bb = s - a.hi;
  const double e = (a.hi - (s - bb)) + (x - bb);
  a.hi = s;
  a.lo += e;
}

__device__ __forceinline__ void dd_merge(DD &a, double bhi, double blo) {
  const double s = a.hi + bhi;
  const double bb = s - a.hi;
  const double e = (a.hi - (s - bb)) + (bhi - bb);
  a.hi = s;
  a.lo = (a.lo + blo) + e;
}

template <int NV>
__device__ __forceinline__ void block_sum(DD (&v)[NV], double *smem /*2*NV*32*/) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    DD x = v[q];
    for (int o = 16; o > 0; o >>= 1) {
      const double h = __shfl_down_sync(0xffffffffu, x.hi, o);
      const double l = __shfl_down_sync(0xffffffffu, x.lo, o);
      dd_merge(x, h, l);
    }
    if (lane == 0) {
      smem[(2 * q) * 32 + wid] = x.hi;
      smem[(2 * q + 1) * 32 + wid] = x.lo;
    }
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      DD x{0.0, 0.0};
      if (lane < nw) x = DD{smem[(2 * q) * 32 + lane], smem[(2 * q + 1) * 32 + lane]};
      for (int o = 16; o > 0; o >>= 1) {
        const double h = __shfl_down_sync(0xffffffffu, x.hi, o);
        const double l = __shfl_down_sync(0xffffffffu, x.lo, o);
        dd_merge(x, h, l);
      }
      v[q] = x;  // valid in thread 0
    }
  }
  __syncthreads();
}

// After every block wrote its partial sums, the last block to arrive merges
// the partials and returns true in thread 0 with the totals.
template <int NV>
__device__ bool grid_sum_last(DD (&v)[NV], double *partials, unsigned int *counter, int nblocks,
                              int blin, double *smem) {
  __shared__ bool am_last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      partials[(2 * q) * kMaxBlocksReduce + blin] = v[q].hi;
      partials[(2 * q + 1) * kMaxBlocksReduce + blin] = v[q].lo;
    }
    __threadfence();
    const unsigned int t = atomicAdd(counter, 1u);
    am_last = (t == (unsigned)nblocks - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  DD acc[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    acc[q] = DD{0.0, 0.0};
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
      dd_merge(acc[q], __ldcg(partials + (2 * q) * kMaxBlocksReduce + b),
               __ldcg(partials + (2 * q + 1) * kMaxBlocksReduce + b));
  }
  block_sum<NV>(acc, smem);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = acc[q];
    *counter = 0u;  // ready for the next launch
  }
  return threadIdx.x == 0;
}

// Mean (mod_utils.cc:30-51): sum(var*dzflzi) / nxg / nyg -> sc->mean[comp]
// (products and sums in FP64 also for an FP32 field)
template <class T>
__global__ void __launch_bounds__(256) k_mean(Geo g, StepConst *sc, int comp, int nxg, int nyg,
                                              const T *__restrict__ var, double *partials,
                                              unsigned int *counter) {
  __shared__ double smem[2 * 32];
  DD s[1] = {{0.0, 0.0}};
  // interior rows over the blocks, their x points over the threads (the
  // double-double sum does not depend on the order)
  const int nrows = g.ny * g.nz;
  for (int row = blockIdx.x; row < nrows; row += gridDim.x) {
    const int k = row / g.ny + 1, j = row - (k - 1) * g.ny + 1;
    const double wz = __ldg(g.dzflzi + k);
    for (int i = threadIdx.x + 1; i <= g.nx; i += blockDim.x)
      dd_add(s[0], double(var[g.at(i, j, k)]) * wz);
  }
  block_sum<1>(s, smem);
  if (grid_sum_last<1>(s, partials, counter, gridDim.x, blockIdx.x, smem)) {
    const double total = s[0].hi + s[0].lo;
    sc->mean[comp] = total / nxg / nyg;
  }
}

// correctVel (mod_calcVel.cc:253-278), interior only.  T = float: the
// mixed form's plain correction (the projection of plc_project).
template <class T>
__global__ void __launch_bounds__(BX *BY) k_correct(Geo g, const StepConst *__restrict__ sc,
                                                    const T *__restrict__ p, T *u, T *v, T *w) {
  const int i = blockIdx.x * BX + threadIdx.x + 1;
  const int j = blockIdx.y * BY + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  if (i > g.nx || j > g.ny) return;
  const long long c = g.at(i, j, k);
  const T pc = p[c];
  u[c] -= (p[c + 1] - pc) * T(sc->dtdxi);
  v[c] -= (p[c + g.X] - pc) * T(sc->dtdyi);
  w[c] -= (p[c + g.XY] - pc) * T(sc->dt) * T(__ldg(g.dzc_inv + k));
}

// Fused correction of the step: correctVel, the halo images of every
// component that is not forced, and the bulk mean of every forced component
// (after correction).  The last block turns the means into the forcing values
// sc->force[d] = vel_force[d] - mean[d] (mod_calcVel.cc:280-301).
struct ForceCfg {
  int forced[3];
  double vel_force[3];
  double u_crf;
};

// One wave of persistent blocks walks work items of 32 x 8 interior columns
// by KZ planes; each thread issues all loads of its column segment (p at
// KZ+1 planes, its x and y neighbours, u, v, w) before the arithmetic, so
// p(k+1) is read once for planes k and k+1 and ~6 loads per thread and plane
// are in flight.  The block reduces once at the end (a reduction tail per
// short-lived block would cost more than the correction itself).
// T = double: the reference's arithmetic.  T = float (mixed form): the
// correction in FP32, the bulk sums of the forced components in FP64.
template <class T, int KZ>
__global__ void __launch_bounds__(256, 2) k_correct_fused(Geo g, StepConst *sc, ForceCfg fc,
                                                          const T *__restrict__ p, T *u, T *v,
                                                          T *w, double *partials,
                                                          unsigned int *counter) {
  __shared__ double smem[2 * 3 * 32];
  const T dtdxi = T(sc->dtdxi), dtdyi = T(sc->dtdyi), dt = T(sc->dt);
  const int tiles_x = (g.nx + 31) / 32, tiles_y = (g.ny + 7) / 8;
  const int per_chunk = tiles_x * tiles_y;
  const int items = per_chunk * ((g.nz + KZ - 1) / KZ);
  const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;
  const long long X = g.X, XY = g.XY;
  DD s[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
  // FP64: error-free double-double terms (the order-independent sum of the
  // reference restatement); FP32 fields: a plain FP64 sum of the FP32 values
  auto acc = [](DD &a, double x) {
    if constexpr (sizeof(T) == 8)
      dd_add(a, x);
    else
      a.hi += x;
  };
  for (int item = blockIdx.x; item < items; item += gridDim.x) {
    const int kc = item / per_chunk, r = item - kc * per_chunk;
    const int jt = r / tiles_x, it = r - jt * tiles_x;
    const int i = it * 32 + lx + 1, j = jt * 8 + ly + 1, k0 = kc * KZ + 1;
    if (i > g.nx || j > g.ny) continue;
    const int nk = min(KZ, g.nz - k0 + 1);
    const long long c0 = g.at(i, j, k0);
    const HaloCol h = halo_col(g, i, j);
    T pc[KZ + 1], px[KZ], py[KZ], uu[KZ], vv[KZ], ww[KZ];
#pragma unroll
    for (int q = 0; q < KZ; ++q)
      if (q < nk) {
        const long long c = c0 + q * XY;
        pc[q] = p[c];
        px[q] = p[c + 1];
        py[q] = p[c + X];
        uu[q] = u[c];
        vv[q] = v[c];
        ww[q] = w[c];
      }
    // p(k+1) of the last plane (k0+nk <= nz+1, a halo plane at most)
#pragma unroll
    for (int q = 1; q <= KZ; ++q)
      if (q == nk) pc[q] = p[c0 + q * XY];
#pragma unroll
    for (int q = 0; q < KZ; ++q)
      if (q < nk) {
        const int k = k0 + q;
        const long long c = c0 + q * XY;
        // correctVel, mod_calcVel.cc:272-274
        const T nu = uu[q] - (px[q] - pc[q]) * dtdxi;
        const T nv = vv[q] - (py[q] - pc[q]) * dtdyi;
        const T nw = ww[q] - (pc[q + 1] - pc[q]) * dt * T(__ldg(g.dzc_inv + k));
        const double dzl = __ldg(g.dzflzi + k);
        if (fc.forced[0]) {
          u[c] = nu;
          acc(s[0], double(nu) * dzl);
        } else {
          store_point(u, g, h, c, k, nu, BC_CENTRED, T(0.0 - fc.u_crf));
        }
        if (fc.forced[1]) {
          v[c] = nv;
          acc(s[1], double(nv) * dzl);
        } else {
          store_point(v, g, h, c, k, nv, BC_CENTRED, T(0));
        }
        if (fc.forced[2]) {
          w[c] = nw;
          acc(s[2], double(nw) * dzl);
        } else {
          store_point(w, g, h, c, k, nw, BC_FACE, T(0));
        }
      }
  }
  block_sum<3>(s, smem);
  if (grid_sum_last<3>(s, partials, counter, gridDim.x, blockIdx.x, smem)) {
    for (int d = 0; d < 3; ++d) {
      if (fc.forced[d]) {
        const double mean = (s[d].hi + s[d].lo) / g.nx / g.ny;
        sc->mean[d] = mean;
        sc->force[d] = fc.vel_force[d] - mean;
      } else {
        sc->mean[d] = 0.0;
        sc->force[d] = 0.0;
      }
    }
  }
}

// The mixed form's fused correction: correctVel (mod_calcVel.cc:272-274) plus
// the forcing sc->force[d] that its fused RK2 stage has already reduced
// (0 for unforced components), written with the halo images and wall ghosts.
// No reduction, so a plain grid: each thread takes KZ planes of one column
// (p(k+1) of a plane is p(k) of the next) with all loads issued first.
template <class T, int KZ>
__global__ void __launch_bounds__(BX *BY) k_correct_forced(Geo g, const StepConst *__restrict__ sc,
                                                           double u_crf, const T *__restrict__ p,
                                                           T *u, T *v, T *w) {
  const int i = blockIdx.x * BX + threadIdx.x + 1;
  const int j = blockIdx.y * BY + threadIdx.y + 1;
  const int k0 = blockIdx.z * KZ + 1;
  if (i > g.nx || j > g.ny) return;
  const int nk = min(KZ, g.nz - k0 + 1);
  const T dtdxi = T(sc->dtdxi), dtdyi = T(sc->dtdyi), dt = T(sc->dt);
  const T fu = T(sc->force[0]), fv = T(sc->force[1]), fw = T(sc->force[2]);
  const long long c0 = g.at(i, j, k0), X = g.X, XY = g.XY;
  const HaloCol h = halo_col(g, i, j);
  T pc[KZ + 1], px[KZ], py[KZ], uu[KZ], vv[KZ], ww[KZ];
#pragma unroll
  for (int q = 0; q < KZ; ++q)
    if (q < nk) {
      const long long c = c0 + q * XY;
      pc[q] = p[c];
      px[q] = p[c + 1];
      py[q] = p[c + X];
      uu[q] = u[c];
      vv[q] = v[c];
      ww[q] = w[c];
    }
#pragma unroll
  for (int q = 1; q <= KZ; ++q)
    if (q == nk) pc[q] = p[c0 + q * XY];
#pragma unroll
  for (int q = 0; q < KZ; ++q)
    if (q < nk) {
      const int k = k0 + q;
      const long long c = c0 + q * XY;
      const T nu = uu[q] - (px[q] - pc[q]) * dtdxi + fu;
      const T nv = vv[q] - (py[q] - pc[q]) * dtdyi + fv;
      const T nw = ww[q] - (pc[q + 1] - pc[q]) * dt * T(__ldg(g.dzc_inv + k)) + fw;
      store_point(u, g, h, c, k, nu, BC_CENTRED, T(0.0 - u_crf));
      store_point(v, g, h, c, k, nv, BC_CENTRED, T(0));
      store_point(w, g, h, c, k, nw, BC_FACE, T(0));
    }
}

// The same for one block of a batched launch over several channels (the
// block's coordinates from the work list).  The single-channel kernel keeps
// its own copy of these lines: a body shared between the two changed the
// single-channel kernel's code generation and made it slower.
template <class T, int KZ>
__device__ __forceinline__ void correct_forced_body(Geo g, const StepConst *__restrict__ sc,
                                                    double u_crf, const T *__restrict__ p, T *u,
                                                    T *v, T *w, VBlk vb) {
  const int i = vb.x() * BX + threadIdx.x + 1;
  const int j = vb.y() * BY + threadIdx.y + 1;
  const int k0 = vb.z() * KZ + 1;
  if (i > g.nx || j > g.ny) return;
  const int nk = min(KZ, g.nz - k0 + 1);
  const T dtdxi = T(sc->dtdxi), dtdyi = T(sc->dtdyi), dt = T(sc->dt);
  const T fu = T(sc->force[0]), fv = T(sc->force[1]), fw = T(sc->force[2]);
  const long long c0 = g.at(i, j, k0), X = g.X, XY = g.XY;
  const HaloCol h = halo_col(g, i, j);
  T pc[KZ + 1], px[KZ], py[KZ], uu[KZ], vv[KZ], ww[KZ];
#pragma unroll
  for (int q = 0; q < KZ; ++q)
    if (q < nk) {
      const long long c = c0 + q * XY;
      pc[q] = p[c];
      px[q] = p[c + 1];
      py[q] = p[c + X];
      uu[q] = u[c];
      vv[q] = v[c];
      ww[q] = w[c];
    }
#pragma unroll
  for (int q = 1; q <= KZ; ++q)
    if (q == nk) pc[q] = p[c0 + q * XY];
#pragma unroll
  for (int q = 0; q < KZ; ++q)
    if (q < nk) {
      const int k = k0 + q;
      const long long c = c0 + q * XY;
      const T nu = uu[q] - (px[q] - pc[q]) * dtdxi + fu;
      const T nv = vv[q] - (py[q] - pc[q]) * dtdyi + fv;
      const T nw = ww[q] - (pc[q + 1] - pc[q]) * dt * T(__ldg(g.dzc_inv + k)) + fw;
      // inline image stores: in small channels most warps have boundary lanes
      store_point_inline(u, g, h, c, k, nu, BC_CENTRED, T(0.0 - u_crf));
      store_point_inline(v, g, h, c, k, nv, BC_CENTRED, T(0));
      store_point_inline(w, g, h, c, k, nw, BC_FACE, T(0));
    }
}

// The same over the mixed-form channels of an ensemble in one launch (the
// arguments of each channel in the parameters; block b works for channel m,
// start[m] <= b < start[m + 1], as block b - start[m] of its own grid).
struct CorrMember {
  Geo g;
  const StepConst *sc;
  double u_crf;
  const float *p;
  float *u, *v, *w;
  int gx, gy, gz;
};
struct CorrBatch {
  int n;
  int start[kBatchMax + 1];
  CorrMember m[kBatchMax];
};
static_assert(sizeof(CorrBatch) <= 32000, "kernel parameters are limited to 32764 bytes");
template <int KZ>
__global__ void __launch_bounds__(BX *BY) k_correct_forced_batch(const __grid_constant__ CorrBatch b) {
  batch_grid_sync();
  const int q = batch_member(b.start, b.n, (int)blockIdx.x);
  const CorrMember &a = b.m[q];
  correct_forced_body<float, KZ>(a.g, a.sc, a.u_crf, a.p, a.u, a.v, a.w,
                                 VBlk::of((int)blockIdx.x - b.start[q], a.gx, a.gy, a.gz));
}

// Adds sc->force[d] to the interior of each forced component
// (mod_calcVel.cc:296-316); with FUSE the halos of those components are
// refreshed from the new interior values (the final updateBoundVel of
// main.cc:153).
// Each thread walks kz planes of one column; all its loads are issued first.
template <class T, bool FUSE>
__global__ void __launch_bounds__(BX *BY) k_force_apply(Geo g, const StepConst *__restrict__ sc,
                                                        ForceCfg fc, T *u, T *v, T *w, int kz) {
  constexpr int KMAX = 8;
  const int i = blockIdx.x * BX + threadIdx.x + 1;
  const int j = blockIdx.y * BY + threadIdx.y + 1;
  const int kb = blockIdx.z * kz + 1;
  const int nk = min(kz, g.nz - kb + 1);
  if (i > g.nx || j > g.ny) return;
  const long long c0 = g.at(i, j, kb);
  T *q[3] = {u, v, w};
  const int kind[3] = {BC_CENTRED, BC_CENTRED, BC_FACE};
  const T bc[3] = {T(0.0 - fc.u_crf), T(0), T(0)};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (!fc.forced[d]) continue;
    const T f = T(sc->force[d]);
    for (int k0 = 0; k0 < nk; k0 += KMAX) {
      T x[KMAX];
#pragma unroll
      for (int s = 0; s < KMAX; ++s)
        if (k0 + s < nk) x[s] = q[d][c0 + (long long)(k0 + s) * g.XY];
#pragma unroll
      for (int s = 0; s < KMAX; ++s)
        if (k0 + s < nk) {
          const T nv = x[s] + f;
          if (FUSE)
            store_with_halo(q[d], g, i, j, kb + k0 + s, nv, kind[d], bc[d]);
          else
            q[d][c0 + (long long)(k0 + s) * g.XY] = nv;
        }
    }
  }
}

// Boundary update of the velocity (mod_updateBound.cc:263-285) as one kernel
// over the interior: every interior point rewrites its own halo images.
template <class T>
__global__ void __launch_bounds__(BX *BY) k_bound_vel(Geo g, double u_crf, T *u, T *v, T *w) {
  const int i = blockIdx.x * BX + threadIdx.x + 1;
  const int j = blockIdx.y * BY + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  if (i > g.nx || j > g.ny) return;
  // only points that own an image do any work
  if (!(i == 1 || i == g.nx || j == 1 || j == g.ny || k == 1 || k == g.nz)) return;
  const long long c = g.at(i, j, k);
  store_with_halo(u, g, i, j, k, u[c], BC_CENTRED, T(0.0 - u_crf));
  store_with_halo(v, g, i, j, k, v[c], BC_CENTRED, T(0));
  store_with_halo(w, g, i, j, k, w[c], BC_FACE, T(0));
}

template <class T>
__global__ void __launch_bounds__(BX *BY) k_bound_p(Geo g, T *p) {
  const int i = blockIdx.x * BX + threadIdx.x + 1;
  const int j = blockIdx.y * BY + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  if (i > g.nx || j > g.ny) return;
  if (!(i == 1 || i == g.nx || j == 1 || j == g.ny || k == 1 || k == g.nz)) return;
  store_with_halo(p, g, i, j, k, p[g.at(i, j, k)], BC_ZEROGRAD, T(0));
}

// var -= delta on the interior (transform2CRF, mod_calcVel.cc:13-25)
template <class T>
__global__ void k_shift(Geo g, T *var, double delta) {
  const int i = blockIdx.x * BX + threadIdx.x + 1;
  const int j = blockIdx.y * BY + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  if (i > g.nx || j > g.ny) return;
  const long long c = g.at(i, j, k);
  var[c] = T(var[c] - delta);
}

// var *= *mult on the interior (bulk rescale of initFlow, mod_initFlow.cc:108-118)
template <class T>
__global__ void k_scale(Geo g, T *var, const double *mult) {
  const int i = blockIdx.x * BX + threadIdx.x + 1;
  const int j = blockIdx.y * BY + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  if (i > g.nx || j > g.ny) return;
  const double m = *mult;
  const long long c = g.at(i, j, k);
  var[c] = T(var[c] * m);
}

// Project noise generator: minstd (48271, 2^31-1) seeded with `seed` and
// jumped ahead to output number offset+1, mapped to [0,1).
__device__ __forceinline__ double noise_uniform(int seed, long long offset) {
  const unsigned long long m = 2147483647ull;
  unsigned long long x = (unsigned long long)((long long)seed % (long long)m);
  if (x == 0) x = 1;
  unsigned long long e = (unsigned long long)offset + 1ull, base = 48271ull, mult = 1ull;
  while (e) {
    if (e & 1ull) mult = (mult * base) % m;
    base = (base * base) % m;
    e >>= 1;
  }
  x = (x * mult) % m;
  return (double)(x - 1ull) / (double)(m - 1ull);
}

// initFlow (mod_initFlow.cc:47-106) before the bulk rescale: u = profile(k)
// plus noise, v and w noise only; halos untouched (zero).
// (computed in FP64 and stored in T)
template <class T>
__global__ void k_init_flow(Geo g, const double *__restrict__ prof, int with_noise, double norm,
                            T *u, T *v, T *w) {
  const int i = blockIdx.x * BX + threadIdx.x + 1;
  const int j = blockIdx.y * BY + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  if (i > g.nx || j > g.ny) return;
  const long long c = g.at(i, j, k);
  double uu = prof[k], vv = 0.0, ww = 0.0;
  if (with_noise) {
    const long long off = ((long long)(k - 1) * g.ny + (j - 1)) * g.nx + (i - 1);
    // explicit roundings (no contraction) so that the field is bit-identical
    // to var += 2.0*(x - 0.5)*norm evaluated term by term
    uu = __dadd_rn(uu, __dmul_rn(__dmul_rn(2.0, __dsub_rn(noise_uniform(123, off), 0.5)), norm));
    vv = __dadd_rn(vv, __dmul_rn(__dmul_rn(2.0, __dsub_rn(noise_uniform(456, off), 0.5)), norm));
    ww = __dadd_rn(ww, __dmul_rn(__dmul_rn(2.0, __dsub_rn(noise_uniform(789, off), 0.5)), norm));
  }
  u[c] = T(uu);
  v[c] = T(vv);
  w[c] = T(ww);
}

// Streamwise vortices added to v, w (plc_init_flow with init_vortex_amp):
// psi(j, k) at the cell edge (y = j dy, z = zf[k]); v(j,k) = dpsi/dz and
// w(j,k) = -dpsi/dy as differences over the cell, so that the discrete
// divergence of the perturbation vanishes; psi and dpsi/dz are zero at the
// walls.
__device__ __forceinline__ double vortex_psi(double amp, double ky, double dy, const double *zf,
                                             double lz, int j, int k) {
  const double zeta = 2.0 * zf[k] / lz - 1.0;
  const double e = 1.0 - zeta * zeta;
  return amp * sin(ky * j * dy) * e * e;
}

template <class T>
__global__ void k_add_vortices(Geo g, const double *__restrict__ zf, double amp, double kx,
                               double ky, double dx, double dy, double lz, T *v, T *w) {
  const int i = blockIdx.x * BX + threadIdx.x + 1;
  const int j = blockIdx.y * BY + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  if (i > g.nx || j > g.ny) return;
  const long long c = g.at(i, j, k);
  const double fx = 1.0 + 0.5 * cos(kx * i * dx);
  const double p = vortex_psi(amp, ky, dy, zf, lz, j, k);
  const double pz = vortex_psi(amp, ky, dy, zf, lz, j, k - 1);
  const double py = vortex_psi(amp, ky, dy, zf, lz, j - 1, k);
  v[c] = T(double(v[c]) + (p - pz) * g.dzf_inv[k] * fx);
  w[c] = T(double(w[c]) - (p - py) / dy * fx);
}

// ---------------------------------------------------------------------------
// NaN / CFL / divergence check (mod_utils.cc:77-205).  what: bit 0 NaN of u
// (halos included), bit 1 CFL, bit 2 divergence.  Max with the smallest
// linear index on ties, i.e. the first maximum of the reference's k,j,i scan.
// ---------------------------------------------------------------------------
struct MaxIdx {
  double v;
  long long i;
};
__device__ __forceinline__ void max_combine(MaxIdx &a, double v, long long i) {
  if (v > a.v || (v == a.v && i < a.i)) {
    a.v = v;
    a.i = i;
  }
}

__device__ void block_max(MaxIdx &a, MaxIdx *smem) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    double v = __shfl_down_sync(0xffffffffu, a.v, o);
    long long i = __shfl_down_sync(0xffffffffu, a.i, o);
    max_combine(a, v, i);
  }
  if (lane == 0) smem[wid] = a;
  __syncthreads();
  if (wid == 0) {
    MaxIdx b = (lane < nw) ? smem[lane] : MaxIdx{0.0, 0x7fffffffffffffffll};
    for (int o = 16; o > 0; o >>= 1) {
      double v = __shfl_down_sync(0xffffffffu, b.v, o);
      long long i = __shfl_down_sync(0xffffffffu, b.i, o);
      max_combine(b, v, i);
    }
    a = b;
  }
  __syncthreads();
}

// The scan of the checks of main.cc:156-178 over one channel by block lb of
// nb: NaN anywhere in u (what & 1), the CFL rate (what & 2) and the
// divergence (what & 4) at every interior point, FP32 fields in FP64
// arithmetic.  The interior rows (j, k) are cut into 64-point segments, one
// segment per warp at a time (two points per lane, all loads issued first),
// so that short rows keep every lane busy.  The maxima keep the lowest index
// among equal values: the result does not depend on the partition.
template <class T>
__device__ __forceinline__ void check_scan(const Geo &g, int what, const T *__restrict__ u,
                                           const T *__restrict__ v, const T *__restrict__ w,
                                           int lb, int nb, MaxIdx &cfl, MaxIdx &div,
                                           int &nan_found) {
  if (what & 1) {
    const long long nall = g.XY * (g.nz + 2);
    const long long stride = (long long)nb * blockDim.x;
    long long t = (long long)lb * blockDim.x + threadIdx.x;
    for (; t + 3 * stride < nall; t += 4 * stride) {
      const T a0 = u[t], a1 = u[t + stride], a2 = u[t + 2 * stride], a3 = u[t + 3 * stride];
      if (isnan(a0) || isnan(a1) || isnan(a2) || isnan(a3)) nan_found = 1;
    }
    for (; t < nall; t += stride)
      if (isnan(u[t])) nan_found = 1;
  }
  if (what & 6) {
    constexpr int SEG = 64;
    const int segs = (g.nx + SEG - 1) / SEG;
    // ny * nz * segs stays far below 2^31 for any channel whose fields fit in memory
    const int ntask = g.ny * g.nz * segs;
    const int wpb = (int)(blockDim.x >> 5), lane = (int)(threadIdx.x & 31);
    for (int task = lb * wpb + (int)(threadIdx.x >> 5); task < ntask; task += nb * wpb) {
      const int row = task / segs, sg = task - row * segs;
      const int k = row / g.ny + 1, j = row - (k - 1) * g.ny + 1;
      const double dzfi = __ldg(g.dzf_inv + k);
      double uc[2], um[2], vc[2], vm[2], wc[2], wm[2];
      long long cc[2];
      bool in[2];
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int i = sg * SEG + 32 * r + lane + 1;
        in[r] = i <= g.nx;
        const long long c = g.at(in[r] ? i : 1, j, k);
        cc[r] = c;
        uc[r] = u[c];
        um[r] = u[c - 1];
        vc[r] = v[c];
        vm[r] = v[c - g.X];
        wc[r] = w[c];
        wm[r] = w[c - g.XY];
      }
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        if (!in[r]) continue;
        if (what & 2) {
          const double q = fabs((uc[r] + um[r]) * 0.5) * g.dx_inv +
                           fabs((vc[r] + vm[r]) * 0.5) * g.dy_inv + fabs((wc[r] + wm[r]) * 0.5) * dzfi;
          max_combine(cfl, q, cc[r]);
        }
        if (what & 4) {
          const double d =
              fabs((uc[r] - um[r]) * g.dx_inv + (vc[r] - vm[r]) * g.dy_inv + (wc[r] - wm[r]) * dzfi);
          max_combine(div, d, cc[r]);
        }
      }
    }
  }
}

// (an FP32 field is checked in FP64 arithmetic)
template <class T>
__global__ void __launch_bounds__(256) k_check(Geo g, int what, const T *__restrict__ u,
                                               const T *__restrict__ v, const T *__restrict__ w,
                                               double *partials, unsigned int *counter,
                                               CheckResult *out) {
  __shared__ MaxIdx smem[32];
  __shared__ int nan_s;
  __shared__ bool am_last;
  if (threadIdx.x == 0) nan_s = 0;
  __syncthreads();
  const long long first = g.at(1, 1, 1);
  MaxIdx cfl{0.0, first}, div{0.0, first};
  int nan_found = 0;
  if (what & 1) {
    const long long nall = (long long)g.XY * (g.nz + 2);
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nall;
         t += (long long)gridDim.x * blockDim.x)
      if (isnan(u[t])) nan_found = 1;
  }
  if (what & 6) {
    // interior rows (j, k) over the blocks, the x points of a row over the
    // threads: one division per row instead of two per point
    const int nrows = g.ny * g.nz;
    for (int row = blockIdx.x; row < nrows; row += gridDim.x) {
      const int k = row / g.ny + 1, j = row - (k - 1) * g.ny + 1;
      const double dzfi = __ldg(g.dzf_inv + k);
      for (int i = threadIdx.x + 1; i <= g.nx; i += blockDim.x) {
        const long long c = g.at(i, j, k);
        const double uc = u[c], um = u[c - 1], vc = v[c], vm = v[c - g.X], wc = w[c],
                     wm = w[c - g.XY];
        if (what & 2) {
          const double r = fabs((uc + um) * 0.5) * g.dx_inv + fabs((vc + vm) * 0.5) * g.dy_inv +
                           fabs((wc + wm) * 0.5) * dzfi;
          max_combine(cfl, r, c);
        }
        if (what & 4) {
          const double d = fabs((uc - um) * g.dx_inv + (vc - vm) * g.dy_inv + (wc - wm) * dzfi);
          max_combine(div, d, c);
        }
      }
    }
  }
  if (nan_found) atomicOr(&nan_s, 1);
  block_max(cfl, smem);
  block_max(div, smem);
  // partial layout: [0] cfl value, [1] cfl index, [2] div value, [3] div index (as double bits)
  if (threadIdx.x == 0) {
    partials[0 * kMaxBlocksReduce + blockIdx.x] = cfl.v;
    partials[1 * kMaxBlocksReduce + blockIdx.x] = __longlong_as_double(cfl.i);
    partials[2 * kMaxBlocksReduce + blockIdx.x] = div.v;
    partials[3 * kMaxBlocksReduce + blockIdx.x] = __longlong_as_double(div.i);
    if (nan_s) atomicOr(&out->nan_found, 1);
    __threadfence();
    const unsigned int t = atomicAdd(counter, 1u);
    am_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  MaxIdx c2{0.0, first}, d2{0.0, first};
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
    max_combine(c2, __ldcg(partials + b), __double_as_longlong(__ldcg(partials + kMaxBlocksReduce + b)));
    max_combine(d2, __ldcg(partials + 2 * kMaxBlocksReduce + b),
                __double_as_longlong(__ldcg(partials + 3 * kMaxBlocksReduce + b)));
  }
  block_max(c2, smem);
  block_max(d2, smem);
  if (threadIdx.x == 0) {
    out->cfl = c2.v;
    out->cfl_idx = c2.i;
    out->div = d2.v;
    out->div_idx = d2.i;
    *counter = 0u;
  }
}

// The full check (what = 7) of the mixed-form channels of an ensemble in one
// launch, with what each channel's check step does after it: block b works
// as block b - start[m] of nb blocks of channel m (start[m] <= b <
// start[m + 1]); the last block of a channel writes its result to the
// device and to the channel's pinned host copy, and, under CFL control, the
// new dt and its derived factors (the host's arithmetic: one division, then
// the products).  The same maxima and indices as k_check (ties to the
// lowest index); the NaN flag travels in the partials, so nothing has to be
// cleared first.
struct ChkMember {
  Geo g;
  const float *u, *v, *w;
  double *partials;
  unsigned int *counter;
  CheckResult *out, *out_host;
  StepConst *sc;
  double cfl_target;
  int nb;
};
struct ChkBatch {
  int n;
  int start[kBatchMax + 1];
  ChkMember m[kBatchMax];
};
static_assert(sizeof(ChkBatch) <= 32000, "kernel parameters are limited to 32764 bytes");
__global__ void __launch_bounds__(256) k_check_batch(const __grid_constant__ ChkBatch bt) {
  batch_grid_sync();
  __shared__ MaxIdx smem[32];
  __shared__ int nan_s;
  __shared__ bool am_last;
  const int q = batch_member(bt.start, bt.n, (int)blockIdx.x);
  const ChkMember &M = bt.m[q];
  const Geo g = M.g;
  const int lb = (int)blockIdx.x - bt.start[q], nb = M.nb;
  if (threadIdx.x == 0) nan_s = 0;
  __syncthreads();
  const long long first = g.at(1, 1, 1);
  MaxIdx cfl{0.0, first}, div{0.0, first};
  int nan_found = 0;
  check_scan<float>(g, 7, M.u, M.v, M.w, lb, nb, cfl, div, nan_found);
  if (nan_found) atomicOr(&nan_s, 1);
  block_max(cfl, smem);
  block_max(div, smem);
  double *partials = M.partials;
  if (threadIdx.x == 0) {
    partials[0 * kMaxBlocksReduce + lb] = cfl.v;
    partials[1 * kMaxBlocksReduce + lb] = __longlong_as_double(cfl.i);
    partials[2 * kMaxBlocksReduce + lb] = div.v;
    partials[3 * kMaxBlocksReduce + lb] = __longlong_as_double(div.i);
    partials[4 * kMaxBlocksReduce + lb] = nan_s ? 1.0 : 0.0;
    __threadfence();
    const unsigned int t = atomicAdd(M.counter, 1u);
    am_last = (t == (unsigned)nb - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  MaxIdx c2{0.0, first}, d2{0.0, first};
  int nan_any = 0;
  for (int b2 = threadIdx.x; b2 < nb; b2 += blockDim.x) {
    max_combine(c2, __ldcg(partials + b2), __double_as_longlong(__ldcg(partials + kMaxBlocksReduce + b2)));
    max_combine(d2, __ldcg(partials + 2 * kMaxBlocksReduce + b2),
                __double_as_longlong(__ldcg(partials + 3 * kMaxBlocksReduce + b2)));
    if (__ldcg(partials + 4 * kMaxBlocksReduce + b2) != 0.0) nan_any = 1;
  }
  if (threadIdx.x == 0) nan_s = 0;
  __syncthreads();
  if (nan_any) atomicOr(&nan_s, 1);
  block_max(c2, smem);
  block_max(d2, smem);
  if (threadIdx.x == 0) {
    CheckResult res;
    res.nan_found = nan_s;
    res.pad = 0;
    res.cfl = c2.v;
    res.cfl_idx = c2.i;
    res.div = d2.v;
    res.div_idx = d2.i;
    *M.out = res;
    *M.out_host = res;
    if (M.cfl_target > 0.0 && c2.v > 0.0) {
      const double dt = M.cfl_target / c2.v;
      const double dti = 1.0 / dt;
      M.sc->dt = dt;
      M.sc->dti = dti;
      M.sc->dtidxi = dti * g.dx_inv;
      M.sc->dtidyi = dti * g.dy_inv;
      M.sc->dtdxi = dt * g.dx_inv;
      M.sc->dtdyi = dt * g.dy_inv;
    }
    *M.counter = 0u;
  }
}

inline dim3 interior_grid(const plc_ctx *c) {
  return dim3((c->nx + BX - 1) / BX, (c->ny + BY - 1) / BY, c->nz);
}

inline int reduce_blocks(const plc_ctx *c) {
  long long n = (long long)c->nx * c->ny * c->nz;
  long long b = (n + 255) / 256;
  if (b > 148 * 8) b = 148 * 8;
  if (b < 1) b = 1;
  return (int)b;
}

inline ForceCfg force_cfg(const plc_ctx *c) {
  ForceCfg fc;
  for (int d = 0; d < 3; ++d) {
    fc.forced[d] = c->prm.is_forced[d] ? 1 : 0;
    fc.vel_force[d] = c->prm.vel_force[d];
  }
  fc.u_crf = c->prm.u_crf;
  return fc;
}

}  // namespace

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library does not link libcuda directly).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = []() {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

namespace {

// Tensor map of one halo'd field: dims (X, Y, Z), box = one 34 x 18 halo tile
// of one plane.  Base and strides are multiples of 16 bytes (X is even); the
// tile's x origin 32*bx is even, i.e. 16-byte aligned.
bool field_tensor_map(CUtensorMap *m, const double *ptr, const Geo &g) {
  auto enc = tensor_map_encoder();
  if (!enc || (reinterpret_cast<unsigned long long>(ptr) & 15ull)) return false;
  cuuint64_t dims[3] = {(cuuint64_t)g.X, (cuuint64_t)g.Y, (cuuint64_t)(g.nz + 2)};
  cuuint64_t strides[2] = {(cuuint64_t)g.X * 8ull, (cuuint64_t)g.XY * 8ull};
  cuuint32_t box[3] = {(cuuint32_t)HX, (cuuint32_t)HY, 1u};
  cuuint32_t estr[3] = {1u, 1u, 1u};
  const CUresult r =
      enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double *>(ptr), dims, strides, box,
          estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <int STAGE, bool FUSE>
cudaError_t launch_rk_tma(const plc_ctx *c, const CUtensorMap &mu, const CUtensorMap &mv,
                          const CUtensorMap &mw, double u_crf, double *ou, double *ov, double *ow,
                          cudaStream_t s) {
  const int kchunk = rk_chunk(c, KCHUNK_TMA);
  dim3 grid((c->nx + RX - 1) / RX, (c->ny + RY - 1) / RY, (c->nz + kchunk - 1) / kchunk);
  if (u_crf != 0.0)
    k_rk_tma<STAGE, FUSE, true><<<grid, RX * TY, rk_tma_smem_bytes(), s>>>(
        mu, mv, mw, c->geo(), c->d_sc, u_crf, ou, ov, ow, kchunk, c->d_err,
        STAGE == 2 ? c->order[SK_RK2] : 0);
  else
    k_rk_tma<STAGE, FUSE, false><<<grid, RX * TY, rk_tma_smem_bytes(), s>>>(
        mu, mv, mw, c->geo(), c->d_sc, u_crf, ou, ov, ow, kchunk, c->d_err,
        STAGE == 2 ? c->order[SK_RK2] : 0);
  return cudaGetLastError();
}

}  // namespace

// Raises the dynamic shared-memory limit of the FP64 RK kernels (~51 KB) on
// the current device.
cudaError_t rk_tma_configure() {
  const int bytes = (int)rk_tma_smem_bytes();
  cudaError_t e = cudaSuccess;
#define PLC_RK_ATTR(S, F, C)                                                                \
  if (e == cudaSuccess)                                                                     \
    e = cudaFuncSetAttribute(k_rk_tma<S, F, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                             bytes);
  PLC_RK_ATTR(1, true, true)
  PLC_RK_ATTR(1, true, false)
  PLC_RK_ATTR(1, false, true)
  PLC_RK_ATTR(1, false, false)
  PLC_RK_ATTR(2, true, true)
  PLC_RK_ATTR(2, true, false)
  PLC_RK_ATTR(2, false, true)
  PLC_RK_ATTR(2, false, false)
#undef PLC_RK_ATTR
  return e;
}

cudaError_t launch_rk(const plc_ctx *c, int stage, bool fuse_bc, double u_crf, const double *qu,
                      const double *qv, const double *qw, double *ou, double *ov, double *ow,
                      cudaStream_t s) {
  const Geo g = c->geo();
  CUtensorMap mu, mv, mw;
  if (field_tensor_map(&mu, qu, g) && field_tensor_map(&mv, qv, g) &&
      field_tensor_map(&mw, qw, g)) {
    if (stage == 1)
      return fuse_bc ? launch_rk_tma<1, true>(c, mu, mv, mw, u_crf, ou, ov, ow, s)
                     : launch_rk_tma<1, false>(c, mu, mv, mw, u_crf, ou, ov, ow, s);
    return fuse_bc ? launch_rk_tma<2, true>(c, mu, mv, mw, u_crf, ou, ov, ow, s)
                   : launch_rk_tma<2, false>(c, mu, mv, mw, u_crf, ou, ov, ow, s);
  }
  // operands not 16-byte aligned: the global-load kernel
  dim3 grid = interior_grid(c), block(BX, BY);
  if (stage == 1) {
    if (fuse_bc)
      k_rk<1, true><<<grid, block, 0, s>>>(g, c->d_sc, u_crf, qu, qv, qw, ou, ov, ow);
    else
      k_rk<1, false><<<grid, block, 0, s>>>(g, c->d_sc, u_crf, qu, qv, qw, ou, ov, ow);
  } else {
    if (fuse_bc)
      k_rk<2, true><<<grid, block, 0, s>>>(g, c->d_sc, u_crf, qu, qv, qw, ou, ov, ow);
    else
      k_rk<2, false><<<grid, block, 0, s>>>(g, c->d_sc, u_crf, qu, qv, qw, ou, ov, ow);
  }
  return cudaGetLastError();
}

cudaError_t launch_calc_rhs(const plc_ctx *c, const double *u, const double *v, const double *w,
                            double *rhs, cudaStream_t s) {
  k_calc_rhs<<<interior_grid(c), dim3(BX, BY), 0, s>>>(c->geo(), c->d_sc, u, v, w, rhs);
  return cudaGetLastError();
}

namespace {
// planes a thread of the mixed form's correction takes: 8 (0.418 ms against
// 0.437 for 4, FP32, 768x384x256)
constexpr int kCorrKzMixed = 8;

template <class T>
cudaError_t correct_fused_t(const plc_ctx *c, const T *p, T *u, T *v, T *w, cudaStream_t s) {
  // KZ planes per work item (the loads of one item live in registers): 6 in
  // FP32, 4 in FP64; 2 resident blocks per SM (launch bounds)
  constexpr int KZ = sizeof(T) == 4 ? 6 : 4;
  constexpr int kBlocksPerSm = 2;
  // one wave of resident blocks, at most the items
  const long long items =
      (long long)((c->nx + 31) / 32) * ((c->ny + 7) / 8) * ((c->nz + KZ - 1) / KZ);
  long long nb = (long long)kBlocksPerSm * c->num_sms;
  if (nb > items) nb = items;
  if (nb > kMaxBlocksReduce) nb = kMaxBlocksReduce;
  if (c->mixed) {
    // the mixed form's fused RK2 stage has reduced the forcing already
    constexpr int KZF = kCorrKzMixed;
    dim3 grid((c->nx + BX - 1) / BX, (c->ny + BY - 1) / BY, (c->nz + KZF - 1) / KZF);
    k_correct_forced<T, KZF><<<grid, dim3(BX, BY), 0, s>>>(c->geo(), c->d_sc, c->prm.u_crf, p, u,
                                                          v, w);
  } else {
    k_correct_fused<T, KZ><<<(unsigned)nb, 256, 0, s>>>(c->geo(), c->d_sc, force_cfg(c), p, u, v,
                                                         w, c->d_partials, c->d_counter);
  }
  return cudaGetLastError();
}

template <class T>
cudaError_t force_apply_t(const plc_ctx *c, bool fuse_bc, T *u, T *v, T *w, cudaStream_t s) {
  const ForceCfg fc = force_cfg(c);
  if (!fc.forced[0] && !fc.forced[1] && !fc.forced[2]) return cudaSuccess;
  const int kz = 8;
  dim3 grid((c->nx + BX - 1) / BX, (c->ny + BY - 1) / BY, (c->nz + kz - 1) / kz);
  if (fuse_bc)
    k_force_apply<T, true><<<grid, dim3(BX, BY), 0, s>>>(c->geo(), c->d_sc, fc, u, v, w, kz);
  else
    k_force_apply<T, false><<<grid, dim3(BX, BY), 0, s>>>(c->geo(), c->d_sc, fc, u, v, w, kz);
  return cudaGetLastError();
}

template <class T>
cudaError_t check_t(const plc_ctx *c, const T *u, const T *v, const T *w, int what,
                    cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(c->d_check, 0, sizeof(CheckResult), s);
  if (e != cudaSuccess) return e;
  k_check<T><<<reduce_blocks(c), 256, 0, s>>>(c->geo(), what, u, v, w, c->d_partials,
                                              c->d_counter + 2, c->d_check);
  return cudaGetLastError();
}
}  // namespace

cudaError_t launch_correct(const plc_ctx *c, bool fused, const double *p, double *u, double *v,
                           double *w, cudaStream_t s) {
  if (fused) return correct_fused_t<double>(c, p, u, v, w, s);
  k_correct<double><<<interior_grid(c), dim3(BX, BY), 0, s>>>(c->geo(), c->d_sc, p, u, v, w);
  return cudaGetLastError();
}
// mixed form: the fused correction of the step, or the plain one
cudaError_t launch_correct(const plc_ctx *c, bool fused, const float *p, float *u, float *v,
                           float *w, cudaStream_t s) {
  if (fused) return correct_fused_t<float>(c, p, u, v, w, s);
  k_correct<float><<<interior_grid(c), dim3(BX, BY), 0, s>>>(c->geo(), c->d_sc, p, u, v, w);
  return cudaGetLastError();
}

cudaError_t launch_force_apply(const plc_ctx *c, bool fuse_bc, double *u, double *v, double *w,
                               cudaStream_t s) {
  return force_apply_t<double>(c, fuse_bc, u, v, w, s);
}
cudaError_t launch_force_apply(const plc_ctx *c, bool fuse_bc, float *u, float *v, float *w,
                               cudaStream_t s) {
  return force_apply_t<float>(c, fuse_bc, u, v, w, s);
}

cudaError_t launch_mean(const plc_ctx *c, int comp, int nxg, int nyg, const double *var,
                        cudaStream_t s) {
  k_mean<double><<<reduce_blocks(c), 256, 0, s>>>(c->geo(), c->d_sc, comp, nxg, nyg, var,
                                                  c->d_partials, c->d_counter + 1);
  return cudaGetLastError();
}
cudaError_t launch_mean(const plc_ctx *c, int comp, int nxg, int nyg, const float *var,
                        cudaStream_t s) {
  k_mean<float><<<reduce_blocks(c), 256, 0, s>>>(c->geo(), c->d_sc, comp, nxg, nyg, var,
                                                 c->d_partials, c->d_counter + 1);
  return cudaGetLastError();
}

cudaError_t launch_bound_vel(const plc_ctx *c, double u_crf, double *u, double *v, double *w,
                             cudaStream_t s) {
  k_bound_vel<double><<<interior_grid(c), dim3(BX, BY), 0, s>>>(c->geo(), u_crf, u, v, w);
  return cudaGetLastError();
}
cudaError_t launch_bound_vel(const plc_ctx *c, double u_crf, float *u, float *v, float *w,
                             cudaStream_t s) {
  k_bound_vel<float><<<interior_grid(c), dim3(BX, BY), 0, s>>>(c->geo(), u_crf, u, v, w);
  return cudaGetLastError();
}

cudaError_t launch_bound_p(const plc_ctx *c, double *p, cudaStream_t s) {
  k_bound_p<double><<<interior_grid(c), dim3(BX, BY), 0, s>>>(c->geo(), p);
  return cudaGetLastError();
}
cudaError_t launch_bound_p(const plc_ctx *c, float *p, cudaStream_t s) {
  k_bound_p<float><<<interior_grid(c), dim3(BX, BY), 0, s>>>(c->geo(), p);
  return cudaGetLastError();
}

cudaError_t launch_shift(const plc_ctx *c, double *var, double delta, cudaStream_t s) {
  k_shift<double><<<interior_grid(c), dim3(BX, BY), 0, s>>>(c->geo(), var, delta);
  return cudaGetLastError();
}
cudaError_t launch_shift(const plc_ctx *c, float *var, double delta, cudaStream_t s) {
  k_shift<float><<<interior_grid(c), dim3(BX, BY), 0, s>>>(c->geo(), var, delta);
  return cudaGetLastError();
}

cudaError_t launch_scale(const plc_ctx *c, double *var, const double *d_mult, cudaStream_t s) {
  k_scale<double><<<interior_grid(c), dim3(BX, BY), 0, s>>>(c->geo(), var, d_mult);
  return cudaGetLastError();
}
cudaError_t launch_scale(const plc_ctx *c, float *var, const double *d_mult, cudaStream_t s) {
  k_scale<float><<<interior_grid(c), dim3(BX, BY), 0, s>>>(c->geo(), var, d_mult);
  return cudaGetLastError();
}

cudaError_t launch_check(const plc_ctx *c, const double *u, const double *v, const double *w,
                         int what, cudaStream_t s) {
  return check_t<double>(c, u, v, w, what, s);
}
cudaError_t launch_check(const plc_ctx *c, const float *u, const float *v, const float *w,
                         int what, cudaStream_t s) {
  return check_t<float>(c, u, v, w, what, s);
}

cudaError_t launch_init_flow(const plc_ctx *c, double *u, double *v, double *w,
                             const double *d_prof, cudaStream_t s) {
  k_init_flow<double><<<interior_grid(c), dim3(BX, BY), 0, s>>>(
      c->geo(), d_prof, c->prm.init_with_noise, c->prm.noise_intensity, u, v, w);
  return cudaGetLastError();
}
cudaError_t launch_init_flow(const plc_ctx *c, float *u, float *v, float *w,
                             const double *d_prof, cudaStream_t s) {
  k_init_flow<float><<<interior_grid(c), dim3(BX, BY), 0, s>>>(
      c->geo(), d_prof, c->prm.init_with_noise, c->prm.noise_intensity, u, v, w);
  return cudaGetLastError();
}

template <class T>
cudaError_t vortices_t(const plc_ctx *c, T *v, T *w, const double *d_zf, cudaStream_t s) {
  const plc_params &P = c->prm;
  const double pi = 3.14159265358979323846;
  const double ny_pairs = fmax(1.0, nearbyint(3.0 * P.ly / (2.0 * pi)));
  const double nx_mod = fmax(1.0, nearbyint(2.0 * P.lx / (4.0 * pi)));
  k_add_vortices<T><<<interior_grid(c), dim3(BX, BY), 0, s>>>(
      c->geo(), d_zf, P.init_vortex_amp, 2.0 * pi * nx_mod / P.lx, 2.0 * pi * ny_pairs / P.ly,
      c->dx, c->dy, P.lz, v, w);
  return cudaGetLastError();
}
cudaError_t launch_add_vortices(const plc_ctx *c, double *v, double *w, const double *d_zf,
                                cudaStream_t s) {
  return vortices_t(c, v, w, d_zf, s);
}
cudaError_t launch_add_vortices(const plc_ctx *c, float *v, float *w, const double *d_zf,
                                cudaStream_t s) {
  return vortices_t(c, v, w, d_zf, s);
}

// The mixed form's correction (with the forcing and halos) of n channels in
// launches of up to kBatchMax channels.
cudaError_t launch_correct_batch(plc_ctx *const *cs, int n, cudaStream_t s, bool pdl) {
  constexpr int KZ = kCorrKzMixed;
  for (int q0 = 0; q0 < n; q0 += kBatchMax) {
    CorrBatch b;
    std::memset(&b, 0, sizeof b);
    b.n = std::min(kBatchMax, n - q0);
    int tot = 0;
    for (int q = 0; q < b.n; ++q) {
      const plc_ctx *c = cs[q0 + q];
      if (!c->mixed) return cudaErrorInvalidValue;
      CorrMember &a = b.m[q];
      a.g = c->geo();
      a.sc = c->d_sc;
      a.u_crf = c->prm.u_crf;
      a.p = c->f_field[PLC_P];
      a.u = c->f_field[PLC_U];
      a.v = c->f_field[PLC_V];
      a.w = c->f_field[PLC_W];
      a.gx = (c->nx + BX - 1) / BX;
      a.gy = (c->ny + BY - 1) / BY;
      a.gz = (c->nz + KZ - 1) / KZ;
      b.start[q] = tot;
      tot += a.gx * a.gy * a.gz;
    }
    b.start[b.n] = tot;
    const cudaError_t e =
        launch_batched(k_correct_forced_batch<KZ>, (unsigned)tot, dim3(BX, BY), 0, s, b, pdl);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// The full checks of n mixed-form channels, their CFL-controlled dt and the
// results in their pinned host copies, in launches of up to kBatchMax
// channels (the check step of a graph that carries its checks).
cudaError_t launch_check_batch(plc_ctx *const *cs, int n, cudaStream_t s, bool pdl) {
  for (int q0 = 0; q0 < n; q0 += kBatchMax) {
    ChkBatch b;
    std::memset(&b, 0, sizeof b);
    b.n = std::min(kBatchMax, n - q0);
    int tot = 0;
    for (int q = 0; q < b.n; ++q) {
      plc_ctx *c = cs[q0 + q];
      if (!c->mixed) return cudaErrorInvalidValue;
      ChkMember &a = b.m[q];
      a.g = c->geo();
      a.u = c->f_field[PLC_U];
      a.v = c->f_field[PLC_V];
      a.w = c->f_field[PLC_W];
      a.partials = c->d_partials;
      a.counter = c->d_counter + 2;
      a.out = c->d_check;
      void *hp = nullptr;
      const cudaError_t e = cudaHostGetDevicePointer(&hp, c->h_check, 0);
      if (e != cudaSuccess) return e;
      a.out_host = static_cast<CheckResult *>(hp);
      a.sc = c->d_sc;
      a.cfl_target = c->prm.cfl_target;
      a.nb = reduce_blocks(c);
      b.start[q] = tot;
      tot += a.nb;
    }
    b.start[b.n] = tot;
    const cudaError_t e = launch_batched(k_check_batch, (unsigned)tot, dim3(256), 0, s, b, pdl);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace plc
