// FP32 kernels of the mixed-precision form: the two RK stages and the
// conversions between the reference's FP64 host layout and the context's
// FP32 fields.
//
// The mixed form stores u, v, w, u1, v1, w1, p and the spectral array in
// FP32; the halo'd fields keep the reference's (i, j, k) layout but with the
// x row padded to a multiple of 4 elements (16 bytes), so that every row and
// plane starts on a 16-byte boundary for the bulk tensor copies.  Scalars
// (dt, the forcing), reductions (bulk mean, NaN/CFL/divergence checks) and
// the tridiagonal sweep stay FP64.
//
// RK stages (mod_calcVel.cc:27-129 and :140-242): the same z-marching
// structure as the FP64 kernel -- a block of (i, j) columns walks a chunk of
// z planes, each operand plane brought into a shared-memory ring by one
// cp.async.bulk.tensor copy per field three planes ahead -- but the
// momentum right-hand side is evaluated in FP32 with fused multiply-adds and
// with the z interpolation weights folded into ten per-plane coefficients
// (an algebraic rearrangement of the reference's expressions).  The fused RK2
// stage also sums the forced components for the bulk forcing.

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <type_traits>
#include <vector>

#include "plc_device.cuh"
#include "plc_internal.h"

namespace plc {

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

namespace {

constexpr int RX = 32;                  // interior columns of a tile (one warp)
constexpr int TY = 8;                   // thread rows of a block
constexpr int RY = 2 * TY;              // interior rows of a tile: two per thread
constexpr int HX = 36;                  // 34 columns used; TMA rows are whole 16-byte units
constexpr int HY = RY + 2;              // 18
constexpr int PLANE = HX * HY;          // floats per field-plane
constexpr int SLOT = ((PLANE * 4 + 127) / 128) * 128 / 4;  // floats, 128-B aligned
constexpr int NSLOT = 6;
constexpr unsigned PLANE_TX_BYTES = 3u * PLANE * 4u;
constexpr long long kWaitLimit = 1ll << 22;  // try_wait polls before giving up
constexpr int KCHUNK = 32;
constexpr int NCOEF = 12;               // per-plane coefficient row (10 used), 3 float4

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
__device__ __forceinline__ void tma_load_plane(float *dst, const CUtensorMap *map, int x, int y,
                                               int z, unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z),
      "r"(smem_addr(bar))
      : "memory");
}

// x/y constants of the momentum right-hand side
struct RkConst {
  float qx, qy;    // 0.25/dx, 0.25/dy (convection)
  float rx, ry;    // re_inv/dx^2, re_inv/dy^2 (diffusion)
  float crf;       // 0.5*u_crf/dx (convecting frame; 0 when u_crf = 0)
};

// Per-plane coefficient row k (FP64 on the host, rounded once):
//   [0] at = dzf(k+1)/dzc(k)   [1] bt = dzf(k)/dzc(k)      z interpolation to the
//   [2] ab = dzf(k-1)/dzc(k-1) [3] bb = dzf(k)/dzc(k-1)    top/bottom faces
//   [4] cz = 0.25/dzf(k)       [5] cw = 0.25/dzc(k)        convection, centred / w
//   [6] vt = re_inv/(dzf(k) dzc(k))     [7] vb = re_inv/(dzf(k) dzc(k-1))
//   [8] wt = re_inv/(dzc(k) dzf(k+1))   [9] wb = re_inv/(dzc(k) dzf(k))
struct alignas(16) Coef {
  float at, bt, ab, bb, cz, cw, vt, vb, wt, wb, pad0, pad1;
};

struct Rhs3f {
  float u, v, w;
};

// (visc - conv) at one point (the RK1 stage); P(f, di, dj, dk) reads field f (0 u, 1 v, 2 w)
// at offset (di, dj, dk) from the point.
template <bool CRF, class Acc>
__device__ __forceinline__ Rhs3f momentum_rhs32(const RkConst &K, const Coef &z, const Acc &P) {
  const float u0 = P(0, 0, 0, 0), v0 = P(1, 0, 0, 0), w0 = P(2, 0, 0, 0);
  Rhs3f r;
  {
    const float upx = P(0, 1, 0, 0), umx = P(0, -1, 0, 0), upy = P(0, 0, 1, 0),
                umy = P(0, 0, -1, 0), uzp = P(0, 0, 0, 1), uzm = P(0, 0, 0, -1);
    const float ue = u0 + upx, uw = umx + u0, un = u0 + upy, us = umy + u0;
    const float ut = fmaf(u0, z.at, uzp * z.bt), ub = fmaf(u0, z.ab, uzm * z.bb);
    const float vn = v0 + P(1, 1, 0, 0), vs = P(1, 0, -1, 0) + P(1, 1, -1, 0);
    const float wt = w0 + P(2, 1, 0, 0), wb = P(2, 0, 0, -1) + P(2, 1, 0, -1);
    float conv = K.qx * (ue * ue - uw * uw) + K.qy * (un * vn - us * vs) +
                 z.cz * (ut * wt - ub * wb);
    if (CRF) conv = fmaf(K.crf, ue - uw, conv);
    const float visc = K.rx * ((upx - u0) - (u0 - umx)) + K.ry * ((upy - u0) - (u0 - umy)) +
                       (z.vt * (uzp - u0) - z.vb * (u0 - uzm));
    r.u = visc - conv;
  }
  {
    const float vpx = P(1, 1, 0, 0), vmx = P(1, -1, 0, 0), vpy = P(1, 0, 1, 0),
                vmy = P(1, 0, -1, 0), vzp = P(1, 0, 0, 1), vzm = P(1, 0, 0, -1);
    const float ve = v0 + vpx, vw = vmx + v0, vn = v0 + vpy, vs = vmy + v0;
    const float vt = fmaf(v0, z.at, vzp * z.bt), vb = fmaf(v0, z.ab, vzm * z.bb);
    const float ue = u0 + P(0, 0, 1, 0), uw = P(0, -1, 0, 0) + P(0, -1, 1, 0);
    const float wt = w0 + P(2, 0, 1, 0), wb = P(2, 0, 0, -1) + P(2, 0, 1, -1);
    float conv = K.qx * (ue * ve - uw * vw) + K.qy * (vn * vn - vs * vs) +
                 z.cz * (wt * vt - wb * vb);
    if (CRF) conv = fmaf(K.crf, ve - vw, conv);
    const float visc = K.rx * ((vpx - v0) - (v0 - vmx)) + K.ry * ((vpy - v0) - (v0 - vmy)) +
                       (z.vt * (vzp - v0) - z.vb * (v0 - vzm));
    r.v = visc - conv;
  }
  {
    const float wpx = P(2, 1, 0, 0), wmx = P(2, -1, 0, 0), wpy = P(2, 0, 1, 0),
                wmy = P(2, 0, -1, 0), wzp = P(2, 0, 0, 1), wzm = P(2, 0, 0, -1);
    const float we = w0 + wpx, ww = wmx + w0, wn = w0 + wpy, ws = wmy + w0;
    const float wt = w0 + wzp, wb = w0 + wzm;
    const float ue = fmaf(u0, z.at, P(0, 0, 0, 1) * z.bt);
    const float uw = fmaf(P(0, -1, 0, 0), z.at, P(0, -1, 0, 1) * z.bt);
    const float vn = fmaf(v0, z.at, P(1, 0, 0, 1) * z.bt);
    const float vs = fmaf(P(1, 0, -1, 0), z.at, P(1, 0, -1, 1) * z.bt);
    float conv = K.qx * (ue * we - uw * ww) + K.qy * (vn * wn - vs * ws) +
                 z.cw * (wt * wt - wb * wb);
    if (CRF) conv = fmaf(K.crf, we - ww, conv);
    const float visc = K.rx * ((wpx - w0) - (w0 - wmx)) + K.ry * ((wpy - w0) - (w0 - wmy)) +
                       (z.wt * (wzp - w0) - z.wb * (w0 - wzm));
    r.w = visc - conv;
  }
  return r;
}

// The z-face terms of the three components at one point: the top-face
// convective products and gradients of plane k are the bottom-face ones of
// plane k+1 (the face values are the same interpolations and sums: the
// interpolation weights of the top face of k are those of the bottom face of
// k+1, with the fused multiply-add on the other product; the sums and
// differences are the same operations).  Tu = ut*wt, Tv = wt*vt, Tw = wt*wt
// and Du = u(k+1)-u(k), Dv, Dw.
struct ZFace {
  float Tu, Tv, Tw, Du, Dv, Dw;
};

// (visc - conv) at one point with the bottom-face terms carried from the
// plane below (bot), or, with FIRST, evaluated from plane k-1 as in
// momentum_rhs32; the top-face terms are returned in top for the plane above.
// Same expressions as momentum_rhs32 otherwise.
template <bool CRF, bool FIRST, class Acc>
__device__ __forceinline__ Rhs3f momentum_rhs32c(const RkConst &K, const Coef &z, const Acc &P,
                                                 const ZFace &bot_in, ZFace &top) {
  const float u0 = P(0, 0, 0, 0), v0 = P(1, 0, 0, 0), w0 = P(2, 0, 0, 0);
  ZFace bot = bot_in;
  if (FIRST) {
    const float uzm = P(0, 0, 0, -1), vzm = P(1, 0, 0, -1), wzm = P(2, 0, 0, -1);
    const float ub = fmaf(u0, z.ab, uzm * z.bb), wbu = wzm + P(2, 1, 0, -1);
    const float vb = fmaf(v0, z.ab, vzm * z.bb), wbv = wzm + P(2, 0, 1, -1);
    const float wbw = w0 + wzm;
    bot.Tu = ub * wbu;
    bot.Tv = wbv * vb;
    bot.Tw = wbw * wbw;
    bot.Du = u0 - uzm;
    bot.Dv = v0 - vzm;
    bot.Dw = w0 - wzm;
  }
  Rhs3f r;
  {
    const float upx = P(0, 1, 0, 0), umx = P(0, -1, 0, 0), upy = P(0, 0, 1, 0),
                umy = P(0, 0, -1, 0), uzp = P(0, 0, 0, 1);
    const float ue = u0 + upx, uw = umx + u0, un = u0 + upy, us = umy + u0;
    const float ut = fmaf(u0, z.at, uzp * z.bt);
    const float vn = v0 + P(1, 1, 0, 0), vs = P(1, 0, -1, 0) + P(1, 1, -1, 0);
    const float wt = w0 + P(2, 1, 0, 0);
    top.Tu = ut * wt;
    top.Du = uzp - u0;
    float conv = K.qx * (ue * ue - uw * uw) + K.qy * (un * vn - us * vs) + z.cz * (top.Tu - bot.Tu);
    if (CRF) conv = fmaf(K.crf, ue - uw, conv);
    const float visc = K.rx * ((upx - u0) - (u0 - umx)) + K.ry * ((upy - u0) - (u0 - umy)) +
                       (z.vt * top.Du - z.vb * bot.Du);
    r.u = visc - conv;
  }
  {
    const float vpx = P(1, 1, 0, 0), vmx = P(1, -1, 0, 0), vpy = P(1, 0, 1, 0),
                vmy = P(1, 0, -1, 0), vzp = P(1, 0, 0, 1);
    const float ve = v0 + vpx, vw = vmx + v0, vn = v0 + vpy, vs = vmy + v0;
    const float vt = fmaf(v0, z.at, vzp * z.bt);
    const float ue = u0 + P(0, 0, 1, 0), uw = P(0, -1, 0, 0) + P(0, -1, 1, 0);
    const float wt = w0 + P(2, 0, 1, 0);
    top.Tv = wt * vt;
    top.Dv = vzp - v0;
    float conv = K.qx * (ue * ve - uw * vw) + K.qy * (vn * vn - vs * vs) + z.cz * (top.Tv - bot.Tv);
    if (CRF) conv = fmaf(K.crf, ve - vw, conv);
    const float visc = K.rx * ((vpx - v0) - (v0 - vmx)) + K.ry * ((vpy - v0) - (v0 - vmy)) +
                       (z.vt * top.Dv - z.vb * bot.Dv);
    r.v = visc - conv;
  }
  {
    const float wpx = P(2, 1, 0, 0), wmx = P(2, -1, 0, 0), wpy = P(2, 0, 1, 0),
                wmy = P(2, 0, -1, 0), wzp = P(2, 0, 0, 1);
    const float we = w0 + wpx, ww = wmx + w0, wn = w0 + wpy, ws = wmy + w0;
    const float wt = w0 + wzp;
    const float ue = fmaf(u0, z.at, P(0, 0, 0, 1) * z.bt);
    const float uw = fmaf(P(0, -1, 0, 0), z.at, P(0, -1, 0, 1) * z.bt);
    const float vn = fmaf(v0, z.at, P(1, 0, 0, 1) * z.bt);
    const float vs = fmaf(P(1, 0, -1, 0), z.at, P(1, 0, -1, 1) * z.bt);
    top.Tw = wt * wt;
    top.Dw = wzp - w0;
    float conv = K.qx * (ue * we - uw * ww) + K.qy * (vn * wn - vs * ws) + z.cw * (top.Tw - bot.Tw);
    if (CRF) conv = fmaf(K.crf, we - ww, conv);
    const float visc = K.rx * ((wpx - w0) - (w0 - wmx)) + K.ry * ((wpy - w0) - (w0 - wmy)) +
                       (z.wt * top.Dw - z.wb * bot.Dw);
    r.w = visc - conv;
  }
  return r;
}

// Operand access from the three plane slots (k-1, k, k+1) of each field.
struct SmemAcc32 {
  const float *base;
  int off[3];  // slot offset of planes k-1, k, k+1 plus the thread's point
  __device__ __forceinline__ float operator()(int f, int di, int dj, int dk) const {
    return base[f * NSLOT * SLOT + off[dk + 1] + di + dj * HX];
  }
};

size_t rk32_smem_bytes() {
  return (size_t)3 * NSLOT * SLOT * 4 + (size_t)(KCHUNK + 2) * NCOEF * 4 + 2 * NSLOT * 8 + 128;
}

// Bulk mean of the forced components, summed by the mixed form's fused RK2
// stage (MEAN = STAGE 2 with FUSE) from the values it stores.  The correction
// that follows changes each x-line of u by -dt/dx times
// sum_i (p(i+1) - p(i)), zero on the periodic line, so this mean of the state
// after RK2 is the mean after the correction (forceVel,
// mod_calcVel.cc:280-301, up to rounding), and the correction adds the force.
// Threads sum in FP32 (a few hundred values), blocks write FP64 partials and
// k_bulk_force adds them in a fixed order.
struct BulkMean {
  int forced[3];
  double vel_force[3];
  double *partials;  // 3 * blocks
};

// RK1 (STAGE 1): o = q + dt*F(q);  RK2 (STAGE 2): o = (q + dt*F(q) + o)/2.
// FUSE: the halo images and wall ghosts of the result are written as well.
//
// A block of 32 x 8 threads owns a 32 x 16 tile of interior columns; each
// thread computes the two rows j, j+1 of its column pair (the operands the two
// points share are read from shared memory once).  The ring has no block-wide
// barrier: every slot has a "full" mbarrier (the copy's transaction bytes) that
// each thread waits on before it reads the plane, and an "empty" mbarrier on
// which each warp arrives once it has read the plane for the last time (at the
// end of iteration p+1 for plane p).  Thread 0 copies plane k+3 into the slot
// of plane k+3-NSLOT = k-3 after that slot's empty barrier completed, so warps
// drift apart by up to two planes without stalling the others.  RK2 reads the
// base values o of its two points one plane ahead from global memory.  Both
// stages run at 4 blocks per SM (64 registers, 50 KB of shared memory; RK1
// measured 0.56 ms at 4 blocks against 0.59 ms at 3, 768 x 384 x 256).
// C2: the second stage carries its z-face terms as well, at 3 blocks per SM
// (the carried values need the registers of a smaller block count); the
// autotuner times it against the plain second stage.
template <int STAGE, bool FUSE, bool CRF, bool C2 = false>
__global__ void __launch_bounds__(RX *TY, (STAGE == 2 && C2) ? 3 : 4)
    k_rk32(const __grid_constant__ CUtensorMap mu, const __grid_constant__ CUtensorMap mv,
           const __grid_constant__ CUtensorMap mw, Geo g, RkConst K,
           const Coef *__restrict__ coef, const StepConst *__restrict__ sc, float bc_u,
           float *ou, float *ov, float *ow, int kchunk, int *err, BulkMean bm) {
  extern __shared__ unsigned char smem_raw[];
  float *slot = reinterpret_cast<float *>(
      (reinterpret_cast<unsigned long long>(smem_raw) + 127ull) & ~127ull);
  Coef *zc = reinterpret_cast<Coef *>(slot + 3 * NSLOT * SLOT);
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(zc + KCHUNK + 2);
  unsigned long long *empty = bar + NSLOT;
  constexpr unsigned kWarps = RX * TY / 32;

  constexpr bool kMean = (STAGE == 2 && FUSE);
  // the first stage carries its z-face terms from plane to plane (about a
  // tenth fewer instructions: RK1 0.554 -> 0.506 ms at 768 x 384 x 256); in the
  // second stage the carried values no longer fit the 64 registers of four
  // blocks per SM (it spilled and took 0.91 against 0.73 ms): there only with C2
  constexpr bool kCarry = (STAGE == 1) || C2;
  float msum[3] = {0.f, 0.f, 0.f};  // kMean: the thread's dz-weighted sums
  const int tid = threadIdx.x;
  const int tx = tid & (RX - 1), ty = tid / RX;
  const int x0 = blockIdx.x * RX, y0 = blockIdx.y * RY;  // halo'd coords of the tile corner
  const int i = x0 + tx + 1, ja = y0 + 2 * ty + 1, jb = ja + 1;
  const bool act_a = (i <= g.nx) && (ja <= g.ny);
  const bool act_b = act_a && (jb <= g.ny);
  const int kb = blockIdx.z * kchunk + 1;
  const int ke = min(kb + kchunk - 1, g.nz);
  const int plast = ke + 1;  // last plane to bring in

  auto issue = [&](int p) {  // thread 0 only
    const int s = (p - (kb - 1)) % NSLOT;
    mbar_expect_tx(&bar[s], PLANE_TX_BYTES);
    tma_load_plane(slot + s * SLOT, &mu, x0, y0, p, &bar[s]);
    tma_load_plane(slot + NSLOT * SLOT + s * SLOT, &mv, x0, y0, p, &bar[s]);
    tma_load_plane(slot + 2 * NSLOT * SLOT + s * SLOT, &mw, x0, y0, p, &bar[s]);
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
  // coefficient rows of the block's planes (and, for the bulk mean, dzf/lz)
  __shared__ float zl[KCHUNK];
  for (int e = tid; e < (ke - kb + 1) * NCOEF; e += blockDim.x)
    reinterpret_cast<float *>(zc)[e] = __ldg(reinterpret_cast<const float *>(coef + kb) + e);
  if (kMean && tid < ke - kb + 1) zl[tid] = float(__ldg(g.dzflzi + kb + tid));
  __syncthreads();

  const float dt = float(sc->dt);
  const long long X = g.X, XY = g.XY;
  long long c = g.at(act_a ? i : 1, act_a ? ja : 1, kb);  // point a; point b is c + X
  // RK2 base values (u, v, w) of plane k at rows a and b, read a plane ahead
  float ba[3] = {0.f, 0.f, 0.f}, bb[3] = {0.f, 0.f, 0.f};
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
  ZFace fa_c{}, fb_c{};  // z-face terms carried from plane k-1 (rows a, b)
  const HaloCol ha = halo_col(g, i, ja), hb = halo_col(g, i, jb);
  const bool xy_edge = (ha.dx | ha.dy | hb.dx | hb.dy) != 0;  // images in x or y
  const int o = (2 * ty + 1) * HX + (tx + 1);  // point a in a slot
  int sm = 0, s0 = 1, sp = 2;                  // slots of planes k-1, k, k+1
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
    float na[3] = {0.f, 0.f, 0.f}, nb[3] = {0.f, 0.f, 0.f};  // base values of plane k+1
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
      const Coef z = zc[k - kb];
      float va[3], vb[3];
      {
        // two rows in scalar FP32
        SmemAcc32 a;
        a.base = slot;
        a.off[0] = sm * SLOT + o;
        a.off[1] = s0 * SLOT + o;
        a.off[2] = sp * SLOT + o;
        SmemAcc32 b = a;
        b.off[0] += HX;
        b.off[1] += HX;
        b.off[2] += HX;
        Rhs3f ra, rb;
        if constexpr (kCarry) {
          if (k == kb) {
            ra = momentum_rhs32c<CRF, true>(K, z, a, fa_c, fa_c);
            rb = momentum_rhs32c<CRF, true>(K, z, b, fb_c, fb_c);
          } else {
            ra = momentum_rhs32c<CRF, false>(K, z, a, fa_c, fa_c);
            rb = momentum_rhs32c<CRF, false>(K, z, b, fb_c, fb_c);
          }
        } else {
          ra = momentum_rhs32<CRF>(K, z, a);
          rb = momentum_rhs32<CRF>(K, z, b);
        }
        const float fa[3] = {ra.u, ra.v, ra.w}, fb[3] = {rb.u, rb.v, rb.w};
        const float qa[3] = {a(0, 0, 0, 0), a(1, 0, 0, 0), a(2, 0, 0, 0)};
        const float qb[3] = {b(0, 0, 0, 0), b(1, 0, 0, 0), b(2, 0, 0, 0)};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          va[d] = fmaf(dt, fa[d], qa[d]);
          vb[d] = fmaf(dt, fb[d], qb[d]);
          if (STAGE == 2) {
            va[d] = (va[d] + ba[d]) * 0.5f;
            vb[d] = (vb[d] + bb[d]) * 0.5f;
          }
        }
      }
      if (kMean) {
        const float dzl = zl[k - kb];
#pragma unroll
        for (int d = 0; d < 3; ++d)
          if (bm.forced[d]) {  // uniform
            // the stored value: w(nz) is the wall value 0
            const bool wall = (d == 2 && k == g.nz);
            const float x = wall ? 0.f : va[d] + (act_b ? vb[d] : 0.f);
            msum[d] = fmaf(x, dzl, msum[d]);
          }
      }
      if (FUSE && (xy_edge || k == 1 || k == g.nz)) {
        store_point(ou, g, ha, c, k, va[0], BC_CENTRED, bc_u);
        store_point(ov, g, ha, c, k, va[1], BC_CENTRED, 0.f);
        store_point(ow, g, ha, c, k, va[2], BC_FACE, 0.f);
        if (act_b) {
          store_point(ou, g, hb, c + X, k, vb[0], BC_CENTRED, bc_u);
          store_point(ov, g, hb, c + X, k, vb[1], BC_CENTRED, 0.f);
          store_point(ow, g, hb, c + X, k, vb[2], BC_FACE, 0.f);
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
  if constexpr (kMean) {
    __shared__ float red[RX * TY / 32][3];
    const int lane = tid & 31, wid = tid >> 5;
#pragma unroll
    for (int d = 0; d < 3; ++d)
      if (bm.forced[d]) {  // uniform: only the forced components are reduced
        float x = msum[d];
        for (int o2 = 16; o2 > 0; o2 >>= 1) x += __shfl_down_sync(0xffffffffu, x, o2);
        if (lane == 0) red[wid][d] = x;
      }
    __syncthreads();
    if (tid < 3) {
      // (a parameter array indexed at run time would be copied to local memory)
      const int forced = tid == 0 ? bm.forced[0] : (tid == 1 ? bm.forced[1] : bm.forced[2]);
      double x = 0.0;
      if (forced)
        for (int w2 = 0; w2 < RX * TY / 32; ++w2) x += double(red[w2][tid]);
      const unsigned nblocks = gridDim.x * gridDim.y * gridDim.z;
      bm.partials[tid * nblocks + blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] =
          x;
    }
  }
}

// The same stage for one block of a batched launch over several channels
// (k_rk32_batch, below): the block's coordinates come from the work list and
// the tensor maps by address.  The single-channel kernel above keeps its own
// copy of these lines: at its limit of 64 registers a shared body changed
// its register allocation (it spilled in RK2, which the copy does not).
template <int STAGE, bool FUSE, bool CRF>
__device__ __forceinline__ void rk32_body(const CUtensorMap *mu, const CUtensorMap *mv,
                                          const CUtensorMap *mw, Geo g, RkConst K,
                                          const Coef *__restrict__ coef,
                                          const StepConst *__restrict__ sc, float bc_u, float *ou,
                                          float *ov, float *ow, int kchunk, int *err,
                                          BulkMean bm, VBlk vb) {
  extern __shared__ unsigned char smem_raw[];
  float *slot = reinterpret_cast<float *>(
      (reinterpret_cast<unsigned long long>(smem_raw) + 127ull) & ~127ull);
  Coef *zc = reinterpret_cast<Coef *>(slot + 3 * NSLOT * SLOT);
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(zc + KCHUNK + 2);
  unsigned long long *empty = bar + NSLOT;
  constexpr unsigned kWarps = RX * TY / 32;

  constexpr bool kMean = (STAGE == 2 && FUSE);
  // the first stage carries its z-face terms from plane to plane (about a
  // tenth fewer instructions: RK1 0.554 -> 0.506 ms at 768 x 384 x 256); in the
  // second stage the carried values no longer fit the 64 registers of four
  // blocks per SM (it spilled and took 0.91 against 0.73 ms)
  constexpr bool kCarry = (STAGE == 1);
  float msum[3] = {0.f, 0.f, 0.f};  // kMean: the thread's dz-weighted sums
  const int tid = threadIdx.x;
  const int tx = tid & (RX - 1), ty = tid / RX;
  const int x0 = vb.x() * RX, y0 = vb.y() * RY;  // halo'd coords of the tile corner
  const int i = x0 + tx + 1, ja = y0 + 2 * ty + 1, jb = ja + 1;
  const bool act_a = (i <= g.nx) && (ja <= g.ny);
  const bool act_b = act_a && (jb <= g.ny);
  const int kb = vb.z() * kchunk + 1;
  const int ke = min(kb + kchunk - 1, g.nz);
  const int plast = ke + 1;  // last plane to bring in

  auto issue = [&](int p) {  // thread 0 only
    const int s = (p - (kb - 1)) % NSLOT;
    mbar_expect_tx(&bar[s], PLANE_TX_BYTES);
    tma_load_plane(slot + s * SLOT, mu, x0, y0, p, &bar[s]);
    tma_load_plane(slot + NSLOT * SLOT + s * SLOT, mv, x0, y0, p, &bar[s]);
    tma_load_plane(slot + 2 * NSLOT * SLOT + s * SLOT, mw, x0, y0, p, &bar[s]);
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
  // coefficient rows of the block's planes (and, for the bulk mean, dzf/lz)
  __shared__ float zl[KCHUNK];
  for (int e = tid; e < (ke - kb + 1) * NCOEF; e += blockDim.x)
    reinterpret_cast<float *>(zc)[e] = __ldg(reinterpret_cast<const float *>(coef + kb) + e);
  if (kMean && tid < ke - kb + 1) zl[tid] = float(__ldg(g.dzflzi + kb + tid));
  __syncthreads();

  const float dt = float(sc->dt);
  const long long X = g.X, XY = g.XY;
  long long c = g.at(act_a ? i : 1, act_a ? ja : 1, kb);  // point a; point b is c + X
  // RK2 base values (u, v, w) of plane k at rows a and b, read a plane ahead
  float ba[3] = {0.f, 0.f, 0.f}, bb[3] = {0.f, 0.f, 0.f};
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
  ZFace fa_c{}, fb_c{};  // z-face terms carried from plane k-1 (rows a, b)
  const HaloCol ha = halo_col(g, i, ja), hb = halo_col(g, i, jb);
  const bool xy_edge = (ha.dx | ha.dy | hb.dx | hb.dy) != 0;  // images in x or y
  // the whole warp takes the image path when one of its lanes has images (in
  // small channels most warps do): no divergence between the two paths
  const bool edge_w = __any_sync(0xffffffffu, xy_edge);
  const int o = (2 * ty + 1) * HX + (tx + 1);  // point a in a slot
  int sm = 0, s0 = 1, sp = 2;                  // slots of planes k-1, k, k+1
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
    float na[3] = {0.f, 0.f, 0.f}, nb[3] = {0.f, 0.f, 0.f};  // base values of plane k+1
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
      const Coef z = zc[k - kb];
      float va[3], vb[3];
      {
        // two rows in scalar FP32
        SmemAcc32 a;
        a.base = slot;
        a.off[0] = sm * SLOT + o;
        a.off[1] = s0 * SLOT + o;
        a.off[2] = sp * SLOT + o;
        SmemAcc32 b = a;
        b.off[0] += HX;
        b.off[1] += HX;
        b.off[2] += HX;
        Rhs3f ra, rb;
        if constexpr (kCarry) {
          if (k == kb) {
            ra = momentum_rhs32c<CRF, true>(K, z, a, fa_c, fa_c);
            rb = momentum_rhs32c<CRF, true>(K, z, b, fb_c, fb_c);
          } else {
            ra = momentum_rhs32c<CRF, false>(K, z, a, fa_c, fa_c);
            rb = momentum_rhs32c<CRF, false>(K, z, b, fb_c, fb_c);
          }
        } else {
          ra = momentum_rhs32<CRF>(K, z, a);
          rb = momentum_rhs32<CRF>(K, z, b);
        }
        const float fa[3] = {ra.u, ra.v, ra.w}, fb[3] = {rb.u, rb.v, rb.w};
        const float qa[3] = {a(0, 0, 0, 0), a(1, 0, 0, 0), a(2, 0, 0, 0)};
        const float qb[3] = {b(0, 0, 0, 0), b(1, 0, 0, 0), b(2, 0, 0, 0)};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          va[d] = fmaf(dt, fa[d], qa[d]);
          vb[d] = fmaf(dt, fb[d], qb[d]);
          if (STAGE == 2) {
            va[d] = (va[d] + ba[d]) * 0.5f;
            vb[d] = (vb[d] + bb[d]) * 0.5f;
          }
        }
      }
      if (kMean) {
        const float dzl = zl[k - kb];
#pragma unroll
        for (int d = 0; d < 3; ++d)
          if (bm.forced[d]) {  // uniform
            // the stored value: w(nz) is the wall value 0
            const bool wall = (d == 2 && k == g.nz);
            const float x = wall ? 0.f : va[d] + (act_b ? vb[d] : 0.f);
            msum[d] = fmaf(x, dzl, msum[d]);
          }
      }
      if (FUSE && (edge_w || k == 1 || k == g.nz)) {
        store_point_inline(ou, g, ha, c, k, va[0], BC_CENTRED, bc_u);
        store_point_inline(ov, g, ha, c, k, va[1], BC_CENTRED, 0.f);
        store_point_inline(ow, g, ha, c, k, va[2], BC_FACE, 0.f);
        if (act_b) {
          store_point_inline(ou, g, hb, c + X, k, vb[0], BC_CENTRED, bc_u);
          store_point_inline(ov, g, hb, c + X, k, vb[1], BC_CENTRED, 0.f);
          store_point_inline(ow, g, hb, c + X, k, vb[2], BC_FACE, 0.f);
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
  if constexpr (kMean) {
    __shared__ float red[RX * TY / 32][3];
    const int lane = tid & 31, wid = tid >> 5;
#pragma unroll
    for (int d = 0; d < 3; ++d)
      if (bm.forced[d]) {  // uniform: only the forced components are reduced
        float x = msum[d];
        for (int o2 = 16; o2 > 0; o2 >>= 1) x += __shfl_down_sync(0xffffffffu, x, o2);
        if (lane == 0) red[wid][d] = x;
      }
    __syncthreads();
    if (tid < 3) {
      // (a parameter array indexed at run time would be copied to local memory)
      const int forced = tid == 0 ? bm.forced[0] : (tid == 1 ? bm.forced[1] : bm.forced[2]);
      double x = 0.0;
      if (forced)
        for (int w2 = 0; w2 < RX * TY / 32; ++w2) x += double(red[w2][tid]);
      const unsigned nblocks = vb.gx() * vb.gy() * vb.gz();
      bm.partials[tid * nblocks + vb.x() + vb.gx() * (vb.y() + vb.gy() * vb.z())] = x;
    }
  }
}

// One RK stage over the channels of an ensemble in one launch: the
// arguments of each channel's k_rk32 launch, tensor maps included, travel in
// the kernel parameters (a TMA copy may name a tensor map there), and block
// b works on tile b - start[m] of channel m.
struct Rk32Member {
  CUtensorMap map[3];
  Geo g;
  RkConst K;
  const Coef *coef;
  const StepConst *sc;
  float bc_u;
  float *ou, *ov, *ow;
  int kchunk;
  int *err;
  BulkMean bm;
  int gx, gy, gz;
};
struct Rk32Batch {
  int n;
  int start[kBatchMax + 1];
  Rk32Member m[kBatchMax];
};
static_assert(sizeof(Rk32Batch) <= 32000, "kernel parameters are limited to 32764 bytes");

// MINB resident blocks per SM: 4 as the single-channel kernel (64 registers:
// the work-list arguments then spill a little in RK2) or 3 (80 registers, no
// spills); the batch autotuner times both.
template <int STAGE, bool FUSE, bool CRF, int MINB>
__global__ void __launch_bounds__(RX *TY, MINB) k_rk32_batch(const __grid_constant__ Rk32Batch b) {
  batch_grid_sync();
  const int q = batch_member(b.start, b.n, (int)blockIdx.x);
  const Rk32Member &a = b.m[q];
  const VBlk vb = VBlk::of((int)blockIdx.x - b.start[q], a.gx, a.gy, a.gz);
  rk32_body<STAGE, FUSE, CRF>(&a.map[0], &a.map[1], &a.map[2], a.g, a.K, a.coef, a.sc, a.bc_u,
                              a.ou, a.ov, a.ow, a.kchunk, a.err, a.bm, vb);
}

// The forcing of the mixed form from the fused RK2's partial sums:
// sc->mean[d] = sum / (nx*ny), sc->force[d] = vel_force[d] - mean
// (forceVel, mod_calcVel.cc:280-301).  One block; the partials are added in a
// fixed order.
__device__ __forceinline__ void bulk_force_body(int nx, int ny, StepConst *sc, BulkMean bm,
                                                int nblocks) {
  __shared__ double red[32][3];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double part[3] = {0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
    for (int d = 0; d < 3; ++d) part[d] += bm.partials[d * nblocks + b];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double x = part[d];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[wid][d] = x;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    const int d = threadIdx.x;
    double tot = 0.0;
    for (int w2 = 0; w2 < (int)(blockDim.x >> 5); ++w2) tot += red[w2][d];
    const double mean = tot / nx / ny;
    sc->mean[d] = bm.forced[d] ? mean : 0.0;
    sc->force[d] = bm.forced[d] ? bm.vel_force[d] - mean : 0.0;
  }
}
__global__ void __launch_bounds__(1024) k_bulk_force(Geo g, StepConst *sc, BulkMean bm,
                                                     int nblocks) {
  bulk_force_body(g.nx, g.ny, sc, bm, nblocks);
}
// the same for the channels of an ensemble: block m reduces channel m's partials
struct BulkMember {
  int nx, ny, nblocks;
  StepConst *sc;
  BulkMean bm;
};
struct BulkBatch {
  int n;
  BulkMember m[kBatchMax];
};
__global__ void __launch_bounds__(1024) k_bulk_force_batch(const __grid_constant__ BulkBatch b) {
  batch_grid_sync();
  const BulkMember &a = b.m[blockIdx.x];
  bulk_force_body(a.nx, a.ny, a.sc, a.bm, a.nblocks);
}

// Tensor map of one FP32 halo'd field: dims (pitch, Y, Z), box = one 36 x 18
// tile of one plane.  The pitch is a multiple of 4 (16 bytes) and the tile's x
// origin 32*bx is 128-byte aligned.
bool field_tensor_map32(CUtensorMap *m, const float *ptr, const Geo &g) {
  auto enc = tensor_map_encoder();
  if (!enc || (reinterpret_cast<unsigned long long>(ptr) & 15ull) || (g.X & 3)) return false;
  cuuint64_t dims[3] = {(cuuint64_t)g.X, (cuuint64_t)g.Y, (cuuint64_t)(g.nz + 2)};
  cuuint64_t strides[2] = {(cuuint64_t)g.X * 4ull, (cuuint64_t)g.XY * 4ull};
  cuuint32_t box[3] = {(cuuint32_t)HX, (cuuint32_t)HY, 1u};
  cuuint32_t estr[3] = {1u, 1u, 1u};
  const CUresult r =
      enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(ptr), dims, strides, box,
          estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <int STAGE, bool FUSE, bool CRF>
cudaError_t launch_rk32_t(const plc_ctx *c, const CUtensorMap (&m)[3], const RkConst &K,
                          float bc_u, float *ou, float *ov, float *ow, cudaStream_t s) {
  const size_t smem = rk32_smem_bytes();
  const int kchunk = rk_chunk(c, KCHUNK);
  dim3 grid((c->nx + RX - 1) / RX, (c->ny + RY - 1) / RY, (c->nz + kchunk - 1) / kchunk);
  BulkMean bm;
  for (int d = 0; d < 3; ++d) {
    bm.forced[d] = c->prm.is_forced[d] ? 1 : 0;
    bm.vel_force[d] = c->prm.vel_force[d];
  }
  bm.partials = c->d_mean_partials;
  bool carried = false;
  if constexpr (STAGE == 2 && FUSE) {
    if (c->rk2_carry) {
      k_rk32<STAGE, FUSE, CRF, true><<<grid, RX * TY, smem, s>>>(
          m[0], m[1], m[2], c->geo(), K, reinterpret_cast<const Coef *>(c->d_coef32), c->d_sc,
          bc_u, ou, ov, ow, kchunk, c->d_err, bm);
      carried = true;
    }
  }
  if (!carried)
    k_rk32<STAGE, FUSE, CRF><<<grid, RX * TY, smem, s>>>(
        m[0], m[1], m[2], c->geo(), K,
        reinterpret_cast<const Coef *>(c->d_coef32), c->d_sc, bc_u, ou, ov, ow, kchunk, c->d_err,
        bm);
  if constexpr (STAGE == 2 && FUSE) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_bulk_force<<<1, 1024, 0, s>>>(c->geo(), c->d_sc, bm, (int)(grid.x * grid.y * grid.z));
  }
  return cudaGetLastError();
}

// FP64 (row length len) -> FP32 (row pitch), rows rows
__global__ void k_to_f32(const double *__restrict__ src, float *__restrict__ dst, long long rows,
                         int len, int pitch) {
  const long long n = rows * len;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const long long r = t / len;
    const int x = (int)(t - r * len);
    dst[r * pitch + x] = (float)src[t];
  }
}

__global__ void k_to_f64(const float *__restrict__ src, double *__restrict__ dst, long long rows,
                         int len, int pitch) {
  const long long n = rows * len;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const long long r = t / len;
    const int x = (int)(t - r * len);
    dst[t] = (double)src[r * pitch + x];
  }
}

unsigned convert_blocks(const plc_ctx *c, long long n) {
  long long b = (n + 255) / 256;
  const long long cap = 16ll * c->num_sms;
  return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

// Blocks of the FP32 RK grid at the smallest z chunk the autotuner may
// choose (the capacity of the bulk-mean partials).
long long rk32_blocks(const plc_ctx *c) {
  const int kchunk = c->nz < kRkChunks[0] ? c->nz : kRkChunks[0];
  return (long long)((c->nx + RX - 1) / RX) * ((c->ny + RY - 1) / RY) *
         ((c->nz + kchunk - 1) / kchunk);
}

// Raises the dynamic shared-memory limit of the FP32 RK kernels (up to ~90 KB)
// on the current device.
cudaError_t rk32_configure() {
  const int bytes = (int)rk32_smem_bytes();
  cudaError_t e = cudaSuccess;
#define PLC_RK32_ATTR(S, F, C)                                                            \
  if (e == cudaSuccess)                                                                   \
    e = cudaFuncSetAttribute(k_rk32<S, F, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                             bytes);
  PLC_RK32_ATTR(1, true, true)
  PLC_RK32_ATTR(1, true, false)
  PLC_RK32_ATTR(1, false, true)
  PLC_RK32_ATTR(1, false, false)
  PLC_RK32_ATTR(2, true, true)
  PLC_RK32_ATTR(2, true, false)
  PLC_RK32_ATTR(2, false, true)
  PLC_RK32_ATTR(2, false, false)
#undef PLC_RK32_ATTR
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_rk32<2, true, true, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_rk32<2, true, false, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
#define PLC_RK32B_ATTR(S, C, M)                                                            \
  if (e == cudaSuccess)                                                                   \
    e = cudaFuncSetAttribute(k_rk32_batch<S, true, C, M>,                                 \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  PLC_RK32B_ATTR(1, true, 3)
  PLC_RK32B_ATTR(1, false, 3)
  PLC_RK32B_ATTR(2, true, 3)
  PLC_RK32B_ATTR(2, false, 3)
  PLC_RK32B_ATTR(1, true, 4)
  PLC_RK32B_ATTR(1, false, 4)
  PLC_RK32B_ATTR(2, true, 4)
  PLC_RK32B_ATTR(2, false, 4)
#undef PLC_RK32B_ATTR
  return e;
}

namespace {
RkConst rk32_const(const plc_ctx *c, double u_crf) {
  RkConst K;
  K.qx = float(0.25 * c->dx_inv);
  K.qy = float(0.25 * c->dy_inv);
  K.rx = float(c->re_inv * c->dx_inv * c->dx_inv);
  K.ry = float(c->re_inv * c->dy_inv * c->dy_inv);
  K.crf = float(0.5 * u_crf * c->dx_inv);
  return K;
}
}  // namespace

cudaError_t launch_rk(const plc_ctx *c, int stage, bool fuse_bc, double u_crf, const float *qu,
                      const float *qv, const float *qw, float *ou, float *ov, float *ow,
                      cudaStream_t s) {
  const Geo g = c->geo();
  // operand tiles (36 x 18) of q
  CUtensorMap m[3];
  if (!field_tensor_map32(&m[0], qu, g) || !field_tensor_map32(&m[1], qv, g) ||
      !field_tensor_map32(&m[2], qw, g))
    return cudaErrorInvalidValue;  // FP32 fields are allocated 16-byte aligned and padded
  const RkConst K = rk32_const(c, u_crf);
  const float bc_u = float(0.0 - u_crf);
  const bool crf = (u_crf != 0.0);
#define PLC_RK32(S, F, C) return launch_rk32_t<S, F, C>(c, m, K, bc_u, ou, ov, ow, s)
  if (stage == 1) {
    if (fuse_bc) {
      if (crf) PLC_RK32(1, true, true);
      PLC_RK32(1, true, false);
    }
    if (crf) PLC_RK32(1, false, true);
    PLC_RK32(1, false, false);
  }
  if (fuse_bc) {
    if (crf) PLC_RK32(2, true, true);
    PLC_RK32(2, true, false);
  }
  if (crf) PLC_RK32(2, false, true);
  PLC_RK32(2, false, false);
#undef PLC_RK32
}

// One fused RK stage (halos written; the second stage also reduces each
// channel's bulk forcing) of n mixed-form channels: one launch for the
// channels at rest in their frame and one for those in a convecting frame,
// each of up to kBatchMax channels.  kchunk > 0: z planes per block of every
// channel whose own choice is not pinned (the bulk-mean partials then round
// differently in FP32 from the channel's own step); 0: each channel's own.
cudaError_t launch_rk_batch(plc_ctx *const *cs, int n, int stage, int kchunk, int minb,
                            cudaStream_t s, bool pdl) {
  const size_t smem = rk32_smem_bytes();
  for (int crf = 0; crf < 2; ++crf) {
    std::vector<int> idx;
    for (int m = 0; m < n; ++m)
      if ((cs[m]->prm.u_crf != 0.0) == (crf == 1)) idx.push_back(m);
    for (size_t q0 = 0; q0 < idx.size(); q0 += kBatchMax) {
      const int cnt = (int)std::min<size_t>(kBatchMax, idx.size() - q0);
      Rk32Batch b;
      BulkBatch bb;
      std::memset(&b, 0, sizeof b);
      std::memset(&bb, 0, sizeof bb);
      b.n = bb.n = cnt;
      int tot = 0;
      for (int q = 0; q < cnt; ++q) {
        const plc_ctx *c = cs[idx[q0 + q]];
        if (!c->mixed) return cudaErrorInvalidValue;
        float *const *f = c->f_field;
        const int iq = stage == 1 ? PLC_U : PLC_U1, io = stage == 1 ? PLC_U1 : PLC_U;
        Rk32Member &a = b.m[q];
        a.g = c->geo();
        for (int d = 0; d < 3; ++d)
          if (!field_tensor_map32(&a.map[d], f[iq + d], a.g)) return cudaErrorInvalidValue;
        a.K = rk32_const(c, c->prm.u_crf);
        a.coef = reinterpret_cast<const Coef *>(c->d_coef32);
        a.sc = c->d_sc;
        a.bc_u = float(0.0 - c->prm.u_crf);
        a.ou = f[io];
        a.ov = f[io + 1];
        a.ow = f[io + 2];
        a.kchunk = (kchunk > 0 && !c->rk_pinned) ? std::min(std::min(kchunk, KCHUNK), c->nz)
                                                 : rk_chunk(c, KCHUNK);
        a.err = c->d_err;
        for (int d = 0; d < 3; ++d) {
          a.bm.forced[d] = c->prm.is_forced[d] ? 1 : 0;
          a.bm.vel_force[d] = c->prm.vel_force[d];
        }
        a.bm.partials = c->d_mean_partials;
        a.gx = (c->nx + RX - 1) / RX;
        a.gy = (c->ny + RY - 1) / RY;
        a.gz = (c->nz + a.kchunk - 1) / a.kchunk;
        b.start[q] = tot;
        tot += a.gx * a.gy * a.gz;
        bb.m[q] = BulkMember{c->nx, c->ny, a.gx * a.gy * a.gz, c->d_sc, a.bm};
      }
      b.start[cnt] = tot;
      auto go = [&](auto SC, auto CC, auto MC) {
        return launch_batched(
            k_rk32_batch<decltype(SC)::value, true, decltype(CC)::value, decltype(MC)::value>,
            (unsigned)tot, dim3(RX * TY), smem, s, b, pdl);
      };
      using I1 = std::integral_constant<int, 1>;
      using I2 = std::integral_constant<int, 2>;
      using B0 = std::integral_constant<bool, false>;
      using B1 = std::integral_constant<bool, true>;
      using M3 = std::integral_constant<int, 3>;
      using M4 = std::integral_constant<int, 4>;
      const bool m4 = minb != 3;
      cudaError_t e;
      if (stage == 1) {
        if (crf) e = m4 ? go(I1{}, B1{}, M4{}) : go(I1{}, B1{}, M3{});
        else e = m4 ? go(I1{}, B0{}, M4{}) : go(I1{}, B0{}, M3{});
      } else {
        if (crf) e = m4 ? go(I2{}, B1{}, M4{}) : go(I2{}, B1{}, M3{});
        else e = m4 ? go(I2{}, B0{}, M4{}) : go(I2{}, B0{}, M3{});
        if (e == cudaSuccess)
          e = launch_batched(k_bulk_force_batch, (unsigned)cnt, dim3(1024), 0, s, bb, pdl);
      }
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

cudaError_t launch_to_f32(const plc_ctx *c, const double *src, float *dst, long long rows, int len,
                          int pitch, cudaStream_t s) {
  const long long n = rows * len;
  k_to_f32<<<convert_blocks(c, n), 256, 0, s>>>(src, dst, rows, len, pitch);
  return cudaGetLastError();
}

cudaError_t launch_to_f64(const plc_ctx *c, const float *src, double *dst, long long rows, int len,
                          int pitch, cudaStream_t s) {
  const long long n = rows * len;
  k_to_f64<<<convert_blocks(c, n), 256, 0, s>>>(src, dst, rows, len, pitch);
  return cudaGetLastError();
}

// Per-plane coefficient rows of the FP32 RK kernels (k = 0 .. nz+1; the rows
// of the ghost planes are not used).
void host_rk32_coef(const plc_ctx *c, std::vector<float> &out) {
  const int nz = c->nz;
  out.assign((size_t)(nz + 2) * NCOEF, 0.f);
  for (int k = 1; k <= nz; ++k) {
    const double dzf_m = c->h_dzf[k - 1], dzf_0 = c->h_dzf[k], dzf_p = c->h_dzf[k + 1];
    const double dzfi_0 = c->h_dzf_inv[k], dzfi_p = c->h_dzf_inv[k + 1];
    const double dzci_m = c->h_dzc_inv[k - 1], dzci_0 = c->h_dzc_inv[k];
    float *r = out.data() + (size_t)k * NCOEF;
    r[0] = float(dzf_p * dzci_0);
    r[1] = float(dzf_0 * dzci_0);
    r[2] = float(dzf_m * dzci_m);
    r[3] = float(dzf_0 * dzci_m);
    r[4] = float(0.25 * dzfi_0);
    r[5] = float(0.25 * dzci_0);
    r[6] = float(c->re_inv * dzfi_0 * dzci_0);
    r[7] = float(c->re_inv * dzfi_0 * dzci_m);
    r[8] = float(c->re_inv * dzci_0 * dzfi_p);
    r[9] = float(c->re_inv * dzci_0 * dzfi_0);
  }
}

int rk32_coef_floats() { return NCOEF; }

}  // namespace plc
