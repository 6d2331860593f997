// C ABI of libplc.so: context management, the module entry points of the
// reference (mod_calcVel, mod_calcRHS, mod_updateBound, mod_poisson_solver,
// mod_fft, mod_utils, mod_initFlow) and the fused, graph-captured time step.

#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <type_traits>
#include <vector>

#include "plc_internal.h"

namespace {
thread_local std::string g_err;  // errors without a context
}

plc::Geo plc_ctx::geo() const {
  plc::Geo g;
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  g.X = pitch;
  g.Y = ny + 2;
  g.XY = (long long)g.X * g.Y;
  g.dx_inv = dx_inv;
  g.dy_inv = dy_inv;
  g.re_inv = re_inv;
  const size_t m = (size_t)nz + 2;
  g.dzf = d_mesh;
  g.dzf_inv = d_mesh + m;
  g.dzc_inv = d_mesh + 2 * m;
  g.dzflzi = d_mesh + 3 * m;
  return g;
}

namespace plc {

int set_error(plc_ctx *ctx, int code, const std::string &msg) {
  if (ctx)
    ctx->err = msg;
  else
    g_err = msg;
  return code;
}

int cuda_status(plc_ctx *ctx, cudaError_t e, const char *what) {
  return set_error(ctx, PLC_ERR_CUDA,
                   std::string("CUDA error '") + cudaGetErrorString(e) + "' in " + what);
}

namespace {

bool fft_length_ok(int n) {
  int r[16], np;
  return n >= 2 && (n % 2 == 0) && host_fft_factor(n, r, &np);
}

int upload_step_consts(plc_ctx *c, double dt) {
  StepConst sc;
  memset(&sc, 0, sizeof sc);
  // the same host arithmetic as the reference: mod_calcVel.cc:36,256-258,
  // mod_calcRHS.cc:11-13
  sc.dt = dt;
  sc.dti = 1.0 / dt;
  sc.dtidxi = sc.dti * c->dx_inv;
  sc.dtidyi = sc.dti * c->dy_inv;
  sc.dtdxi = dt * c->dx_inv;
  sc.dtdyi = dt * c->dy_inv;
  // keep force/mean/cfl fields as they are on the device
  PLC_CUDA(c, cudaMemcpyAsync(c->d_sc, &sc, 6 * sizeof(double), cudaMemcpyHostToDevice,
                              c->stream));
  PLC_CUDA(c, cudaStreamSynchronize(c->stream));
  c->dt_host = dt;
  return PLC_OK;
}

// The same without waiting for the copy (after a check that synchronised the
// stream): the values are staged in pinned scalars 16..21, which only this
// function writes, and the next upload comes after the next check's
// synchronisation.
int upload_step_consts_async(plc_ctx *c, double dt) {
  double *st = c->h_scal + 16;
  st[0] = dt;
  st[1] = 1.0 / dt;
  st[2] = st[1] * c->dx_inv;
  st[3] = st[1] * c->dy_inv;
  st[4] = dt * c->dx_inv;
  st[5] = dt * c->dy_inv;
  PLC_CUDA(c, cudaMemcpyAsync(c->d_sc, st, 6 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  c->dt_host = dt;
  return PLC_OK;
}

void free_poisson(plc_ctx *c) {
  // the captured step holds the solver's tables and tile sizes
  if (c->graph) cudaStreamSynchronize(c->stream);
  drop_graph(c);
  cudaFree(c->d_rpiv);
  cudaFree(c->d_ac);
  cudaFree(c->d_low);
  cudaFree(c->d_rpiv32);
  cudaFree(c->d_ac32);
  cudaFree(c->plan_x.tw);
  cudaFree(c->plan_y.tw);
  cudaFree(c->plan_x.tw32);
  cudaFree(c->plan_y.tw32);
  c->d_rpiv = nullptr;
  c->d_ac = nullptr;
  c->d_low = nullptr;
  c->d_rpiv32 = nullptr;
  c->d_ac32 = nullptr;
  c->plan_x.tw = nullptr;
  c->plan_y.tw = nullptr;
  c->plan_x.tw32 = nullptr;
  c->plan_y.tw32 = nullptr;
  c->poisson_ready = false;
}

int init_poisson(plc_ctx *c, const double *dzf_global) {
  free_poisson(c);
  std::vector<double> rpiv, a, cc;
  host_trid_tables(c->nx, c->ny, c->nz, c->dx, c->dy, dzf_global, rpiv, a, cc);
  if (c->mixed) {
    // The (0,0) system is singular (Neumann in z): its last pivot is zero up
    // to rounding and its right-hand side sums to zero only up to FP32
    // rounding.  The mixed form pins it: the reciprocal of the last pivot is
    // set to 0, so the top value of the (0,0) mode is 0 and the rest follow
    // by back substitution (the pressure is defined up to a constant).
    const size_t plane = (size_t)(c->nx / 2 + 1) * (c->ny / 2 + 1);
    rpiv[(size_t)(c->nz - 1) * plane] = 0.0;
    const size_t nlow = (size_t)c->nz * kLowModes * kLowModes;
    PLC_CUDA(c, cudaMalloc(&c->d_low, nlow * sizeof(double)));
  }
  PLC_CUDA(c, cudaMalloc(&c->d_rpiv, rpiv.size() * sizeof(double)));
  PLC_CUDA(c, cudaMemcpy(c->d_rpiv, rpiv.data(), rpiv.size() * sizeof(double),
                         cudaMemcpyHostToDevice));
  std::vector<double> ac(a);
  ac.insert(ac.end(), cc.begin(), cc.end());
  PLC_CUDA(c, cudaMalloc(&c->d_ac, ac.size() * sizeof(double)));
  PLC_CUDA(c, cudaMemcpy(c->d_ac, ac.data(), ac.size() * sizeof(double), cudaMemcpyHostToDevice));
  if (c->mixed) {
    // FP32 copies for the systems that sweep in FP32
    const std::vector<float> rpiv32(rpiv.begin(), rpiv.end()), ac32(ac.begin(), ac.end());
    PLC_CUDA(c, cudaMalloc(&c->d_rpiv32, rpiv32.size() * sizeof(float)));
    PLC_CUDA(c, cudaMemcpy(c->d_rpiv32, rpiv32.data(), rpiv32.size() * sizeof(float),
                           cudaMemcpyHostToDevice));
    PLC_CUDA(c, cudaMalloc(&c->d_ac32, ac32.size() * sizeof(float)));
    PLC_CUDA(c, cudaMemcpy(c->d_ac32, ac32.data(), ac32.size() * sizeof(float),
                           cudaMemcpyHostToDevice));
  }
  FftPlan *plans[2] = {&c->plan_x, &c->plan_y};
  const int ns[2] = {c->nx, c->ny};
  for (int d = 0; d < 2; ++d) {
    FftPlan &p = *plans[d];
    p.n = ns[d];
    if (!host_fft_factor(p.n, p.radix, &p.npass))
      return set_error(c, PLC_ERR_SIZE, "FFT length is not 2^a*3^b");
    std::vector<double> tw;
    host_twiddles(p.n, tw);
    PLC_CUDA(c, cudaMalloc(&p.tw, tw.size() * sizeof(double)));
    PLC_CUDA(c, cudaMemcpy(p.tw, tw.data(), tw.size() * sizeof(double), cudaMemcpyHostToDevice));
    if (c->mixed) {
      std::vector<float> tw32(tw.begin(), tw.end());
      PLC_CUDA(c, cudaMalloc(&p.tw32, tw32.size() * sizeof(float)));
      PLC_CUDA(c, cudaMemcpy(p.tw32, tw32.data(), tw32.size() * sizeof(float),
                             cudaMemcpyHostToDevice));
    }
  }
  int dev_max = 0;
  PLC_CUDA(c, cudaDeviceGetAttribute(&dev_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
  // the limit is a per-kernel attribute shared by all contexts: raise it to the
  // device maximum so that no context can lower it under another one
  PLC_CUDA(c, fft_configure((size_t)dev_max));
  c->trid_smem_max = (size_t)dev_max;
  if (fft_setup(c, 76 * 1024, (size_t)dev_max) != cudaSuccess)
    return set_error(c, PLC_ERR_SIZE, "FFT line too long for shared memory");
  c->poisson_ready = true;
  return PLC_OK;
}

int check_ptr(plc_ctx *c, const void *p, const char *name) {
  if (!p) return set_error(c, PLC_ERR_ARG, std::string("null pointer: ") + name);
  return PLC_OK;
}

#define PLC_CHECK_CTX(c) \
  if (!(c)) return plc::set_error(nullptr, PLC_ERR_ARG, "null context")
#define PLC_REQ(c, p) \
  if (int _r = check_ptr(c, p, #p)) return _r

// halo'd linear index of the context's layout -> 0-based (i, j, k) with the
// halo, i.e. the reference's 1-based global indices of the interior
void to_ijk(const plc_ctx *c, long long idx, plc_value_index *out, double value) {
  const long long X = c->pitch, XY = X * (c->ny + 2);
  out->value = value;
  out->kg = (int)(idx / XY);
  out->jg = (int)((idx % XY) / X);
  out->ig = (int)(idx % X);
}

// Reads the error word that kernels with bounded device-side waits raise when
// a wait gives up (synchronises the stream).
int device_error(plc_ctx *c) {
  int flag = 0;
  PLC_CUDA(c, cudaMemcpyAsync(&flag, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  PLC_CUDA(c, cudaStreamSynchronize(c->stream));
  if (flag)
    return set_error(c, PLC_ERR_CUDA,
                     "a device-side wait for a tensor copy timed out (kernel left early)");
  return PLC_OK;
}

template <class T>
int run_check(plc_ctx *c, int what, const T *u, const T *v, const T *w) {
  PLC_CUDA(c, launch_check(c, u, v, w, what, c->stream));
  PLC_CUDA(c, cudaMemcpyAsync(c->h_check, c->d_check, sizeof(CheckResult), cudaMemcpyDeviceToHost,
                              c->stream));
  PLC_CUDA(c, cudaStreamSynchronize(c->stream));
  return PLC_OK;
}

// the checks of the context's own u, v, w in either precision form
int run_check_fields(plc_ctx *c, int what) {
  if (c->mixed)
    return run_check(c, what, c->f_field[PLC_U], c->f_field[PLC_V], c->f_field[PLC_W]);
  return run_check(c, what, c->d_field[PLC_U], c->d_field[PLC_V], c->d_field[PLC_W]);
}

// Autotuner of the RK stages' z planes per block: each candidate of
// kRkChunks (at most nz) timed on both fused stages over the context's own
// fields (best of three after a warm-up launch); the chunk changes which
// blocks compute which planes: no result of the FP64 form, and in the mixed
// form only the FP32 rounding of the per-block bulk-mean sums.  Run at
// creation, before
// the fields hold data to keep (the stages overwrite u1..w1 and u..w).
cudaError_t rk_autotune(plc_ctx *c) {
  cudaEvent_t e0, e1;
  cudaError_t e = cudaEventCreate(&e0);
  if (e != cudaSuccess) return e;
  if ((e = cudaEventCreate(&e1)) != cudaSuccess) {
    cudaEventDestroy(e0);
    return e;
  }
  cudaStream_t s = c->stream;
  const double u_crf = c->prm.u_crf;
  auto launch = [&]() -> cudaError_t {
    cudaError_t r;
    if (c->mixed) {
      float *const *f = c->f_field;
      r = launch_rk(c, 1, true, u_crf, f[PLC_U], f[PLC_V], f[PLC_W], f[PLC_U1], f[PLC_V1],
                    f[PLC_W1], s);
      if (r == cudaSuccess)
        r = launch_rk(c, 2, true, u_crf, f[PLC_U1], f[PLC_V1], f[PLC_W1], f[PLC_U], f[PLC_V],
                      f[PLC_W], s);
    } else {
      double *const *f = c->d_field;
      r = launch_rk(c, 1, true, u_crf, f[PLC_U], f[PLC_V], f[PLC_W], f[PLC_U1], f[PLC_V1],
                    f[PLC_W1], s);
      if (r == cudaSuccess)
        r = launch_rk(c, 2, true, u_crf, f[PLC_U1], f[PLC_V1], f[PLC_W1], f[PLC_U], f[PLC_V],
                      f[PLC_W], s);
    }
    return r;
  };
  int best_k = 0;
  bool best_carry = c->rk2_carry;
  float best_t = -1.f;
  // the mixed form's second stage with or without the z-face carry (unless
  // PLC_RK2_CARRY pins it), with every chunk
  const bool tune_carry = c->mixed && !c->rk2_carry_pinned;
  for (int v = 0; v < (tune_carry ? 2 : 1) && e == cudaSuccess; ++v) {
    if (tune_carry) c->rk2_carry = v == 1;
    int last = -1;
    for (int k : kRkChunks) {
      c->rk_kchunk = k;
      const int eff = rk_chunk(c, 32);
      if (eff == last) continue;  // the same chunk once clamped to nz
      last = eff;
      if ((e = launch()) != cudaSuccess) break;
      float best = -1.f;
      for (int r = 0; r < 3 && e == cudaSuccess; ++r) {
        if ((e = cudaEventRecord(e0, s)) != cudaSuccess || (e = launch()) != cudaSuccess ||
            (e = cudaEventRecord(e1, s)) != cudaSuccess ||
            (e = cudaEventSynchronize(e1)) != cudaSuccess)
          break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (best < 0.f || ms < best) best = ms;
      }
      if (e != cudaSuccess) break;
      if (best_t < 0.f || best < best_t) {
        best_t = best;
        best_k = k;
        best_carry = c->rk2_carry;
      }
    }
  }
  c->rk_kchunk = best_k;
  c->rk2_carry = best_carry;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e;
}

const char *const kStepKernelNames[] = {
    "rk1+bound(u1)", "rk2+bound(u)", "calcRHS+fft_x_fwd", "fft_y_fwd", "trid_z",
    "fft_y_bwd",     "fft_x_bwd+bound(p)", "correct+mean", "force+bound(u)"};
constexpr int kStepKernels = 9;
// the mixed form sums the bulk mean in RK2 and forces in the correction
const char *const kStepKernelNamesMixed[] = {
    "rk1+bound(u1)", "rk2+bound(u)+mean", "calcRHS+fft_x_fwd", "fft_y_fwd", "trid_z",
    "fft_y_bwd",     "fft_x_bwd+bound(p)", "correct+force+bound(u)"};
constexpr int kStepKernelsMixed = 8;  // the one-block bulk_force sum is timed with RK2
int step_kernels(const plc_ctx *c) { return c->mixed ? kStepKernelsMixed : kStepKernels; }

// Launches of one fused step (main.cc:116-154) on the context's fields, in
// the context's storage type T.  With ev != nullptr, ev[0] is recorded before
// the first kernel and ev[q+1] after kernel q (per-kernel timing; not used
// inside graph capture).
template <class T>
int enqueue_step_t(plc_ctx *c, T *const *f, cudaStream_t s, cudaEvent_t *ev) {
  T *u = f[PLC_U], *v = f[PLC_V], *w = f[PLC_W];
  T *u1 = f[PLC_U1], *v1 = f[PLC_V1], *w1 = f[PLC_W1];
  T *p = f[PLC_P], *spec = f[PLC_SPEC];
  const double u_crf = c->prm.u_crf;
  int q = 0;
  auto mark = [&]() -> cudaError_t {
    return ev ? cudaEventRecord(ev[q++], s) : cudaSuccess;
  };
  PLC_CUDA(c, mark());
  PLC_CUDA(c, launch_rk(c, 1, true, u_crf, u, v, w, u1, v1, w1, s));     // RK1 + bound(u1)
  PLC_CUDA(c, mark());
  PLC_CUDA(c, launch_rk(c, 2, true, u_crf, u1, v1, w1, u, v, w, s));     // RK2 + bound(u)
  PLC_CUDA(c, mark());
  if constexpr (std::is_same<T, double>::value)
    PLC_CUDA(c, launch_fft_x_fwd(c, nullptr, u, v, w, spec, s));         // calcRHS + x-FFT
  else
    PLC_CUDA(c, launch_fft_x_fwd(c, u, v, w, spec, s));
  PLC_CUDA(c, mark());
  PLC_CUDA(c, launch_fft_y(c, spec, false, s));                          // y-FFT
  PLC_CUDA(c, mark());
  PLC_CUDA(c, launch_trid(c, spec, s));                                  // z solve
  PLC_CUDA(c, mark());
  PLC_CUDA(c, launch_fft_y(c, spec, true, s));                           // y-iFFT
  PLC_CUDA(c, mark());
  PLC_CUDA(c, launch_fft_x_bwd(c, spec, p, true, s));                    // x-iFFT + bound(p)
  PLC_CUDA(c, mark());
  PLC_CUDA(c, launch_correct(c, true, p, u, v, w, s));                   // correct + mean
  PLC_CUDA(c, mark());
  if constexpr (std::is_same<T, double>::value) {
    PLC_CUDA(c, launch_force_apply(c, true, u, v, w, s));                // force + bound(u)
    PLC_CUDA(c, mark());
  }
  return PLC_OK;
}

int enqueue_step(plc_ctx *c, cudaStream_t s, cudaEvent_t *ev = nullptr) {
  if (c->mixed) return enqueue_step_t<float>(c, c->f_field, s, ev);
  return enqueue_step_t<double>(c, c->d_field, s, ev);
}

int build_graph(plc_ctx *c) {
  if (c->graph) return PLC_OK;
  cudaGraph_t g = nullptr;
  PLC_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  int rc = enqueue_step(c, c->stream);
  cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  if (rc != PLC_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return cuda_status(c, e, "cudaStreamEndCapture");
  size_t nodes = 0;
  cudaGraphGetNodes(g, nullptr, &nodes);
  e = cudaGraphInstantiate(&c->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_status(c, e, "cudaGraphInstantiate");
  // the graph's first launch would otherwise carry its upload to the device
  PLC_CUDA(c, cudaGraphUpload(c->graph, c->stream));
  c->graph_kernels = (int)nodes;
  return PLC_OK;
}

// Mean (mod_utils.cc:30-51) of a device field in the context's layout.
template <class T>
int mean_of(plc_ctx *c, int nxg, int nyg, const T *var, double *mean) {
  PLC_CUDA(c, launch_mean(c, 0, nxg, nyg, var, c->stream));
  PLC_CUDA(c, cudaMemcpyAsync(c->h_scal, reinterpret_cast<char *>(c->d_sc) + offsetof(StepConst, mean),
                              sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  PLC_CUDA(c, cudaStreamSynchronize(c->stream));
  *mean = c->h_scal[0];
  return PLC_OK;
}

// initFlow (mod_initFlow.cc:47-118) on the context's u, v, w from the profile
// prof[k], then transform2CRF and the boundary update (main.cc:78-82).  The
// spectral array serves as device scratch for the profile (its nx*ny*nz
// elements hold more than nz+2 doubles).
template <class T>
int init_fields(plc_ctx *c, const std::vector<double> &prof, bool is_mean, T *const *f) {
  const plc_params &P = c->prm;
  T *u = f[PLC_U], *v = f[PLC_V], *w = f[PLC_W];
  double *scratch = reinterpret_cast<double *>(f[PLC_SPEC]);
  PLC_CUDA(c, cudaMemcpyAsync(scratch, prof.data(), prof.size() * sizeof(double),
                              cudaMemcpyHostToDevice, c->stream));
  PLC_CUDA(c, launch_init_flow(c, u, v, w, scratch, c->stream));
  if (is_mean) {
    double meanold = 0.0;
    // the reference passes (nz, ny) as the global sizes here (mod_initFlow.cc:92)
    if (int rc = mean_of(c, c->nz, c->ny, u, &meanold)) return rc;
    if (meanold != 0.0) {
      c->h_scal[0] = 1.0 / (meanold * P.u_ref);
      PLC_CUDA(c, cudaMemcpyAsync(scratch, c->h_scal, sizeof(double), cudaMemcpyHostToDevice,
                                  c->stream));
      PLC_CUDA(c, launch_scale(c, u, scratch, c->stream));
    }
  }
  if (P.init_vortex_amp != 0.0) {
    // face heights zf[0..nz] after the profile in the scratch
    std::vector<double> zf(c->nz + 1, 0.0);
    for (int k = 1; k <= c->nz; ++k) zf[k] = zf[k - 1] + c->h_dzf_global[k];
    double *d_zf = scratch + prof.size();
    PLC_CUDA(c, cudaMemcpyAsync(d_zf, zf.data(), zf.size() * sizeof(double), cudaMemcpyHostToDevice,
                                c->stream));
    PLC_CUDA(c, launch_add_vortices(c, v, w, d_zf, c->stream));
    PLC_CUDA(c, cudaStreamSynchronize(c->stream));  // zf is a host temporary
  }
  // transform2CRF (mod_calcVel.cc:13-25)
  if (P.u_crf != 0.0) {
    PLC_CUDA(c, launch_shift(c, u, P.u_crf, c->stream));
    c->prm.vel_force[0] -= P.u_crf;
  }
  PLC_CUDA(c, launch_bound_vel(c, P.u_crf, u, v, w, c->stream));
  PLC_CUDA(c, launch_bound_p(c, f[PLC_P], c->stream));
  PLC_CUDA(c, cudaStreamSynchronize(c->stream));
  return PLC_OK;
}

}  // namespace

int capture_step(plc_ctx *c, cudaStream_t s) { return enqueue_step(c, s); }

int step_graph(plc_ctx *c, cudaGraphExec_t *g) {
  if (int rc = build_graph(c)) return rc;
  *g = c->graph;
  return PLC_OK;
}

void drop_graph(plc_ctx *c) {
  if (c->graph) {
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
  ++c->graph_epoch;
}

int shift_field(plc_ctx *c, int field, double delta) {
  if (field < PLC_U || field > PLC_P) return set_error(c, PLC_ERR_ARG, "bad field");
  if (c->mixed)
    PLC_CUDA(c, launch_shift(c, c->f_field[field], delta, c->stream));
  else
    PLC_CUDA(c, launch_shift(c, c->d_field[field], delta, c->stream));
  PLC_CUDA(c, cudaStreamSynchronize(c->stream));
  return PLC_OK;
}

}  // namespace plc

using namespace plc;

extern "C" {

int plc_params_default(plc_params *prm) {
  if (!prm) return set_error(nullptr, PLC_ERR_ARG, "null params");
  memset(prm, 0, sizeof *prm);
  // mod_parameters.hh:15-88: globals are zero unless given a default there
  prm->p_row = 1;
  prm->p_col = 1;
  snprintf(prm->fn_prefix_input_inst, sizeof prm->fn_prefix_input_inst, "save");
  snprintf(prm->fn_prefix_input_stat, sizeof prm->fn_prefix_input_stat, "save_stat");
  prm->u0 = 0.0;
  prm->init_with_noise = 0;
  prm->noise_intensity = 0.0;
  prm->smooth_wall_visc = 0;
  prm->u_crf = 0.0;
  prm->sample_interval = 0;
  prm->overwrite_save = 1;
  prm->auto_cleanup = 1;
  prm->num_retained = 0;
  prm->nt_out_moni = 0;
  prm->precision = PLC_FP64;
  prm->cfl_target = 0.0;
  return PLC_OK;
}

int plc_params_read_json(const char *path, plc_params *prm) {
  if (!path || !prm) return set_error(nullptr, PLC_ERR_ARG, "null argument");
  std::string err;
  int rc = host_parse_param_json(path, prm, err);
  if (rc != PLC_OK) return set_error(nullptr, rc, err);
  return PLC_OK;
}

int plc_params_check(const plc_params *prm) {
  if (!prm) return set_error(nullptr, PLC_ERR_ARG, "null params");
  if (prm->p_row * prm->p_col != 1)
    return set_error(nullptr, PLC_ERR_DECOMP,
                     "PowerLLEL.ERROR: only p_row = p_col = 1 (one GPU) is supported");
  // checkMeshAndPara, mod_parameters.cc:174-177
  if (prm->nx <= 0 || prm->ny <= 0 || prm->nz <= 0 || prm->nx % 2 || prm->ny % 2 || prm->nz % 2)
    return set_error(nullptr, PLC_ERR_SIZE,
                     "PowerLLEL.ERROR.checkInputParam: <nx>, <ny>, <nz> should be even integers!");
  if (!fft_length_ok(prm->nx) || !fft_length_ok(prm->ny))
    return set_error(nullptr, PLC_ERR_SIZE, "nx and ny must be of the form 2^a*3^b");
  if (!(prm->dt > 0.0) || !(prm->re > 0.0) || !(prm->lx > 0.0) || !(prm->ly > 0.0) ||
      !(prm->lz > 0.0) || !(prm->u_ref > 0.0) || !(prm->l_ref > 0.0))
    return set_error(nullptr, PLC_ERR_ARG, "dt, re, lx, ly, lz, u_ref and l_ref must be positive");
  if (prm->precision != PLC_FP64 && prm->precision != PLC_MIXED)
    return set_error(nullptr, PLC_ERR_ARG, "unknown precision form");
  // the FP32 transforms stage 16-byte chunks of 4 elements along x and y rows
  if (prm->precision == PLC_MIXED && (prm->nx % 4 || prm->ny % 4))
    return set_error(nullptr, PLC_ERR_SIZE, "the mixed-precision form needs nx and ny divisible by 4");
  return PLC_OK;
}

int plc_create(const plc_params *prm, const double *h_dzf_global, int device, plc_ctx **out) {
  if (!prm || !out) return set_error(nullptr, PLC_ERR_ARG, "null argument");
  *out = nullptr;
  if (int rc = plc_params_check(prm)) return rc;
  if (prm->read_mesh && !h_dzf_global)
    return set_error(nullptr, PLC_ERR_ARG, "read_mesh = 1 needs dzf_global (mesh.in)");
  plc_ctx *c = new (std::nothrow) plc_ctx;
  if (!c) return set_error(nullptr, PLC_ERR_NOMEM, "host allocation failed");
  c->prm = *prm;
  c->device = device;
  c->nx = prm->nx;
  c->ny = prm->ny;
  c->nz = prm->nz;
  // mod_mesh.cc:26-29 and mod_parameters.cc:259
  c->dx = prm->lx / prm->nx;
  c->dy = prm->ly / prm->ny;
  c->dx_inv = 1.0 / c->dx;
  c->dy_inv = 1.0 / c->dy;
  c->re_inv = prm->u_ref * prm->l_ref / prm->re;
  c->mixed = (prm->precision == PLC_MIXED);
  // FP64 fields keep the reference's row length; FP32 rows are padded to 16 bytes
  c->pitch = c->mixed ? ((c->nx + 2 + 3) / 4) * 4 : c->nx + 2;
  c->nfield = (size_t)c->pitch * (c->ny + 2) * (c->nz + 2);
  c->nspec = (size_t)c->nx * c->ny * c->nz;
  auto fail = [&](int rc) {
    std::string msg = c->err;
    plc_destroy(c);
    return set_error(nullptr, rc, msg);
  };
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(cuda_status(c, e, "cudaSetDevice"));
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return fail(cuda_status(c, e, "cudaStreamCreate"));
  // mesh
  const int nz = c->nz;
  const size_t m = (size_t)nz + 2;
  c->h_dzf_global.assign(m, 0.0);
  if (h_dzf_global)
    memcpy(c->h_dzf_global.data(), h_dzf_global, m * sizeof(double));
  else
    host_mesh_by_func(prm->mesh_type, prm->stretch_func, prm->stretch_ratio, nz, prm->lz,
                      c->h_dzf_global.data());
  c->h_dzf.assign(m, 0.0);
  c->h_dzf_inv.assign(m, 0.0);
  c->h_dzc.assign(m, 0.0);
  c->h_dzc_inv.assign(m, 0.0);
  c->h_dzflzi.assign(m, 0.0);
  c->h_zc_global.assign(m, 0.0);
  host_mesh_derived(nz, prm->lz, c->h_dzf_global.data(), c->h_dzf.data(), c->h_dzf_inv.data(),
                    c->h_dzc.data(), c->h_dzc_inv.data(), c->h_dzflzi.data(),
                    c->h_zc_global.data());
  e = cudaMalloc(&c->d_mesh, 4 * m * sizeof(double));
  if (e != cudaSuccess) return fail(set_error(c, PLC_ERR_NOMEM, "cudaMalloc mesh"));
  const std::vector<double> *parts[4] = {&c->h_dzf, &c->h_dzf_inv, &c->h_dzc_inv, &c->h_dzflzi};
  for (int q = 0; q < 4; ++q) {
    e = cudaMemcpy(c->d_mesh + q * m, parts[q]->data(), m * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(cuda_status(c, e, "upload mesh"));
  }
  // fields (mod_variables.cc:4-12) and the spectral array, zero-initialised
  const size_t esize = c->mixed ? sizeof(float) : sizeof(double);
  for (int f = 0; f < 8; ++f) {
    const size_t n = (f == PLC_SPEC) ? c->nspec : c->nfield;
    void *ptr = nullptr;
    e = cudaMalloc(&ptr, n * esize);
    if (e != cudaSuccess) return fail(set_error(c, PLC_ERR_NOMEM, "cudaMalloc field"));
    if (c->mixed)
      c->f_field[f] = static_cast<float *>(ptr);
    else
      c->d_field[f] = static_cast<double *>(ptr);
    e = cudaMemset(ptr, 0, n * esize);
    if (e != cudaSuccess) return fail(cuda_status(c, e, "cudaMemset field"));
  }
  if (!c->mixed && (e = rk_tma_configure()) != cudaSuccess)
    return fail(cuda_status(c, e, "rk_tma_configure"));
  if (c->mixed) {
    if ((e = rk32_configure()) != cudaSuccess) return fail(cuda_status(c, e, "rk32_configure"));
    // one partial per block of the fused RK2
    if ((e = cudaMalloc(&c->d_mean_partials, 3 * (size_t)rk32_blocks(c) * sizeof(double))) !=
        cudaSuccess)
      return fail(set_error(c, PLC_ERR_NOMEM, "cudaMalloc bulk-mean partials"));
    std::vector<float> coef;
    host_rk32_coef(c, coef);
    if ((e = cudaMalloc(&c->d_coef32, coef.size() * sizeof(float))) != cudaSuccess ||
        (e = cudaMemcpy(c->d_coef32, coef.data(), coef.size() * sizeof(float),
                        cudaMemcpyHostToDevice)) != cudaSuccess)
      return fail(cuda_status(c, e, "RK coefficient table"));
  }
  // scalars and scratch
  if ((e = cudaMalloc(&c->d_sc, sizeof(StepConst))) != cudaSuccess ||
      (e = cudaMemset(c->d_sc, 0, sizeof(StepConst))) != cudaSuccess ||
      (e = cudaMalloc(&c->d_partials, 8 * kMaxBlocksReduce * sizeof(double))) != cudaSuccess ||
      (e = cudaMalloc(&c->d_counter, 8 * sizeof(unsigned int))) != cudaSuccess ||
      (e = cudaMemset(c->d_counter, 0, 8 * sizeof(unsigned int))) != cudaSuccess ||
      (e = cudaMalloc(&c->d_check, sizeof(CheckResult))) != cudaSuccess ||
      (e = cudaMallocHost(&c->h_check, sizeof(CheckResult))) != cudaSuccess ||
      (e = cudaMallocHost(&c->h_scal, 32 * sizeof(double))) != cudaSuccess)
    return fail(cuda_status(c, e, "scratch allocation"));
  c->d_err = reinterpret_cast<int *>(c->d_counter + 4);  // zeroed with the counters
  if ((e = cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device)) !=
      cudaSuccess)
    return fail(cuda_status(c, e, "cudaDeviceGetAttribute"));
  c->device_sms = c->num_sms;
  if (int rc = upload_step_consts(c, prm->dt)) return fail(rc);
  if (int rc = init_poisson(c, c->h_dzf_global.data())) return fail(rc);
  // the fields hold zeros: time the transforms' tile sizes on them
  // PLC_FFT_TILES / PLC_FFT_TILES_F32 = "xf,x,y" (line pairs per tile of the
  // forward x, backward x and y transforms) replace the timing of the FP64 /
  // FP32 transforms: a profiler distorts the event times the autotuner
  // compares, so a profiled run pins the tiles an unprofiled run chose.
  // Plane order (high planes first) of the FP64 second RK stage, the y
  // transforms and the backward x transform: a kernel that starts on the
  // planes its predecessor wrote last finds them in L2 (the Thomas sweep
  // starts and ends at the lowest plane).  Measured at 768 x 384 x 256: the
  // backward x transform, FP64 0.454 -> 0.429 ms.
  {
    const unsigned char fp64[SK_ORDERS] = {1, 1, 0, 1};  // RK2, y fwd, y bwd, x bwd
    const unsigned char fp32[SK_ORDERS] = {0, 1, 0, 1};
    for (int q = 0; q < SK_ORDERS; ++q) c->order[q] = c->mixed ? fp32[q] : fp64[q];
  }
  // PLC_FFT_PLANS / PLC_FFT_PLANS_F32 = "x,y" pin the plan families of the x
  // and y transforms (0: radix 16/8/4/2/3 passes, 1: two passes ending in
  // radix 24, 2: warp-line kernels, 3: two passes in registers; 1, 2 and 3
  // only for lengths that have them)
  // the same way; the tiles are then timed under the pinned families.
  // A third value pins the forward x transform's family apart from the
  // backward one's ("x,y,xf").
  if (const char *env = getenv(c->mixed ? "PLC_FFT_PLANS_F32" : "PLC_FFT_PLANS")) {
    int px = -1, py = -1, pxf = -1;
    const int nread = sscanf(env, "%d,%d,%d", &px, &py, &pxf);
    if (nread == 2) pxf = px;
    auto valid_x = [&](int q) {
      return q >= 0 && q <= 3 && (q != 1 || fft_has_two_plans(c->nx)) &&
             (q != 2 || fft_has_warp_plan(c->nx, c->ny)) && (q != 3 || fft_has_x2_plan(c->nx, c->ny));
    };
    if (nread < 2 || !valid_x(px) || !valid_x(pxf) || py < 0 || py > 3 ||
        (py == 1 && !fft_has_two_plans(c->ny)) ||
        (py == 2 && !fft_has_warp_plan(c->ny, c->nx)) ||
        (py == 3 && !fft_has_y2_plan(c->ny, c->nx, c->mixed ? 4 : 8)))
      return fail(set_error(c, PLC_ERR_ARG, std::string("invalid FFT plans in the environment: ") + env));
    c->fft_plan_x = px;
    c->fft_plan_xf = pxf;
    c->fft_plan_y = py;
    c->fft_plans_pinned = true;
    if ((e = fft_set_lines(c, c->fft_lines_xf, c->fft_lines_x, c->fft_lines_y)) != cudaSuccess)
      return fail(cuda_status(c, e, "fft_set_lines"));
  }
  // PLC_TRID = "tile" / "stream" pins the Thomas sweep (columns on chip or
  // streamed through HBM) instead of timing both
  if (const char *env = getenv("PLC_TRID")) {
    if (strcmp(env, "tile") != 0 && strcmp(env, "stream") != 0)
      return fail(set_error(c, PLC_ERR_ARG, std::string("invalid PLC_TRID: ") + env));
    c->trid_tile = strcmp(env, "tile") == 0;
    c->trid_pinned = true;
  }
  bool pinned = false;
  if (const char *env = getenv(c->mixed ? "PLC_FFT_TILES_F32" : "PLC_FFT_TILES")) {
    int xf = 0, xb = 0, y = 0;
    if (sscanf(env, "%d,%d,%d", &xf, &xb, &y) != 3 || xf < 1 || xb < 1 || y < 1 ||
        (c->ny / 2) % xf || (c->ny / 2) % xb || (c->nx / 2) % y || (c->mixed && y % 2) ||
        fft_set_lines(c, xf, xb, y) != cudaSuccess)
      return fail(set_error(c, PLC_ERR_ARG, std::string("invalid FFT tiles in the environment: ") + env));
    pinned = true;
  }
  if (!pinned && (e = fft_autotune(c)) != cudaSuccess) return fail(cuda_status(c, e, "fft_autotune"));
  // PLC_RK2_CARRY = 0 / 1 pins the mixed form's second RK stage without or
  // with the z-face carry instead of timing both
  if (const char *env = getenv("PLC_RK2_CARRY")) {
    if (strcmp(env, "0") != 0 && strcmp(env, "1") != 0)
      return fail(set_error(c, PLC_ERR_ARG, std::string("invalid PLC_RK2_CARRY: ") + env));
    c->rk2_carry = c->mixed && strcmp(env, "1") == 0;
    c->rk2_carry_pinned = true;
  }
  // PLC_RK_KCHUNK pins the RK stages' z planes per block instead of timing
  // the candidates
  if (const char *env = getenv(c->mixed ? "PLC_RK_KCHUNK_F32" : "PLC_RK_KCHUNK")) {
    // at least the smallest candidate: the mixed form's bulk-mean partials
    // hold the blocks of a grid of that chunk (rk32_blocks)
    const int k = atoi(env);
    if (k < kRkChunks[0] || k > 32)
      return fail(set_error(c, PLC_ERR_ARG, std::string("invalid PLC_RK_KCHUNK: ") + env));
    c->rk_kchunk = k;
    c->rk_pinned = true;
  } else if ((e = rk_autotune(c)) != cudaSuccess) {
    return fail(cuda_status(c, e, "rk_autotune"));
  }
  c->tuned_lines[0] = c->fft_lines_xf;
  c->tuned_lines[1] = c->fft_lines_x;
  c->tuned_lines[2] = c->fft_lines_y;
  *out = c;
  return PLC_OK;
}

int plc_destroy(plc_ctx *c) {
  if (!c) return PLC_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  free_poisson(c);  // also releases the captured step
  plc_stat_free(c);
  io_free(c);
  for (auto &f : c->d_field) cudaFree(f);
  for (auto &f : c->f_field) cudaFree(f);
  cudaFree(c->d_coef32);
  cudaFree(c->d_mean_partials);
  cudaFree(c->d_mesh);
  cudaFree(c->d_sc);
  cudaFree(c->d_partials);
  cudaFree(c->d_counter);
  cudaFree(c->d_check);
  if (c->h_check) cudaFreeHost(c->h_check);
  if (c->h_scal) cudaFreeHost(c->h_scal);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return PLC_OK;
}

const char *plc_last_error(const plc_ctx *c) { return c ? c->err.c_str() : g_err.c_str(); }

int plc_sync(plc_ctx *c) {
  PLC_CHECK_CTX(c);
  PLC_CUDA(c, cudaStreamSynchronize(c->stream));
  return device_error(c);
}

int plc_get_mesh(const plc_ctx *c, int which, double *h_out) {
  if (!c || !h_out) return set_error(nullptr, PLC_ERR_ARG, "null argument");
  const std::vector<double> *arr[7] = {&c->h_dzf_global, &c->h_dzf,    &c->h_dzf_inv, &c->h_dzc,
                                       &c->h_dzc_inv,    &c->h_dzflzi, &c->h_zc_global};
  if (which < 0 || which > 6) return set_error(nullptr, PLC_ERR_ARG, "bad mesh array id");
  memcpy(h_out, arr[which]->data(), arr[which]->size() * sizeof(double));
  return PLC_OK;
}

#define PLC_NEED_FP64(c)                                                              \
  if ((c)->mixed)                                                                     \
  return set_error(c, PLC_ERR_STATE,                                                  \
                   "the module entry points take FP64 fields; this context holds the " \
                   "mixed-precision form (use plc_step, plc_upload/plc_download)")

int plc_field_ptr(plc_ctx *c, int field, double **d_ptr, size_t *count) {
  PLC_CHECK_CTX(c);
  PLC_NEED_FP64(c);
  if (field < 0 || field > PLC_SPEC) return set_error(c, PLC_ERR_ARG, "bad field id");
  if (d_ptr) *d_ptr = c->d_field[field];
  if (count) *count = (field == PLC_SPEC) ? c->nspec : c->nfield;
  return PLC_OK;
}

int plc_field_ptr_f32(plc_ctx *c, int field, float **d_ptr, size_t *count, int *pitch) {
  PLC_CHECK_CTX(c);
  if (!c->mixed) return set_error(c, PLC_ERR_STATE, "the context holds FP64 fields");
  if (field < 0 || field > PLC_SPEC) return set_error(c, PLC_ERR_ARG, "bad field id");
  if (d_ptr) *d_ptr = c->f_field[field];
  if (count) *count = (field == PLC_SPEC) ? c->nspec : c->nfield;
  if (pitch) *pitch = (field == PLC_SPEC) ? c->nx : c->pitch;
  return PLC_OK;
}

// rows and row length of a field in the reference's layout
static void ref_shape(const plc_ctx *c, int field, long long *rows, int *len) {
  if (field == PLC_SPEC) {
    *rows = (long long)c->ny * c->nz;
    *len = c->nx;
  } else {
    *rows = (long long)(c->ny + 2) * (c->nz + 2);
    *len = c->nx + 2;
  }
}

int plc_fft_plans(const plc_ctx *c, int *plan_x, int *plan_y) {
  if (!c) return set_error(nullptr, PLC_ERR_ARG, "null context");
  if (plan_x) *plan_x = c->fft_plan_x;
  if (plan_y) *plan_y = c->fft_plan_y;
  return PLC_OK;
}

int plc_rk_kchunk(const plc_ctx *c, int *kchunk) {
  if (!c || !kchunk) return set_error(nullptr, PLC_ERR_ARG, "null argument");
  *kchunk = rk_chunk(c, 32);
  return PLC_OK;
}

int plc_rk2_carry(const plc_ctx *c, int *carry) {
  if (!c || !carry) return set_error(nullptr, PLC_ERR_ARG, "null argument");
  *carry = c->rk2_carry ? 1 : 0;
  return PLC_OK;
}

int plc_fft_plan_x_fwd(const plc_ctx *c, int *plan) {
  if (!c || !plan) return set_error(nullptr, PLC_ERR_ARG, "null argument");
  *plan = c->fft_plan_xf >= 0 ? c->fft_plan_xf : c->fft_plan_x;
  return PLC_OK;
}

int plc_fft_tiles(const plc_ctx *c, int *lines_xf, int *lines_x, int *lines_y) {
  if (!c) return set_error(nullptr, PLC_ERR_ARG, "null context");
  if (lines_xf) *lines_xf = c->fft_lines_xf;
  if (lines_x) *lines_x = c->fft_lines_x;
  if (lines_y) *lines_y = c->fft_lines_y;
  return PLC_OK;
}

int plc_upload(plc_ctx *c, int field, const double *h_src) {
  PLC_CHECK_CTX(c);
  PLC_REQ(c, h_src);
  if (field < 0 || field > PLC_SPEC) return set_error(c, PLC_ERR_ARG, "bad field id");
  if (!c->mixed) {
    const size_t n = (field == PLC_SPEC) ? c->nspec : c->nfield;
    PLC_CUDA(c, cudaMemcpyAsync(c->d_field[field], h_src, n * sizeof(double),
                                cudaMemcpyHostToDevice, c->stream));
    PLC_CUDA(c, cudaStreamSynchronize(c->stream));
    return PLC_OK;
  }
  // mixed form: FP64 host field -> stream-ordered FP64 staging -> FP32 field
  long long rows;
  int len;
  ref_shape(c, field, &rows, &len);
  const size_t n = (size_t)rows * len;
  double *tmp = nullptr;
  PLC_CUDA(c, cudaMallocAsync(&tmp, n * sizeof(double), c->stream));
  cudaError_t e = cudaMemcpyAsync(tmp, h_src, n * sizeof(double), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess)
    e = launch_to_f32(c, tmp, c->f_field[field], rows, len,
                      field == PLC_SPEC ? c->nx : c->pitch, c->stream);
  const cudaError_t ef = cudaFreeAsync(tmp, c->stream);
  if (e == cudaSuccess) e = ef;
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_status(c, e, "plc_upload (FP64 -> FP32)");
  return PLC_OK;
}

int plc_download(plc_ctx *c, int field, double *h_dst) {
  PLC_CHECK_CTX(c);
  PLC_REQ(c, h_dst);
  if (field < 0 || field > PLC_SPEC) return set_error(c, PLC_ERR_ARG, "bad field id");
  if (!c->mixed) {
    const size_t n = (field == PLC_SPEC) ? c->nspec : c->nfield;
    PLC_CUDA(c, cudaMemcpyAsync(h_dst, c->d_field[field], n * sizeof(double),
                                cudaMemcpyDeviceToHost, c->stream));
    PLC_CUDA(c, cudaStreamSynchronize(c->stream));
    return PLC_OK;
  }
  long long rows;
  int len;
  ref_shape(c, field, &rows, &len);
  const size_t n = (size_t)rows * len;
  double *tmp = nullptr;
  PLC_CUDA(c, cudaMallocAsync(&tmp, n * sizeof(double), c->stream));
  cudaError_t e = launch_to_f64(c, c->f_field[field], tmp, rows, len,
                                field == PLC_SPEC ? c->nx : c->pitch, c->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h_dst, tmp, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  const cudaError_t ef = cudaFreeAsync(tmp, c->stream);
  if (e == cudaSuccess) e = ef;
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_status(c, e, "plc_download (FP32 -> FP64)");
  return PLC_OK;
}

int plc_get_dt(plc_ctx *c, double *dt) {
  PLC_CHECK_CTX(c);
  PLC_REQ(c, dt);
  *dt = c->dt_host;
  return PLC_OK;
}

int plc_step_forcing(plc_ctx *c, double *mean3, double *force3) {
  PLC_CHECK_CTX(c);
  PLC_REQ(c, mean3);
  // force[3] and mean[3] are adjacent in the device struct
  static_assert(offsetof(StepConst, mean) == offsetof(StepConst, force) + 3 * sizeof(double),
                "force and mean adjacent");
  PLC_CUDA(c, cudaMemcpyAsync(c->h_scal, reinterpret_cast<char *>(c->d_sc) + offsetof(StepConst, force),
                              6 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  PLC_CUDA(c, cudaStreamSynchronize(c->stream));
  for (int d = 0; d < 3; ++d) {
    mean3[d] = c->h_scal[3 + d];
    if (force3) force3[d] = c->h_scal[d];
  }
  return PLC_OK;
}

int plc_set_dt(plc_ctx *c, double dt) {
  PLC_CHECK_CTX(c);
  if (!(dt > 0.0)) return set_error(c, PLC_ERR_ARG, "dt must be positive");
  c->prm.dt = dt;
  return upload_step_consts(c, dt);
}

// ---- mod_calcVel ----------------------------------------------------------
int plc_transform2crf(plc_ctx *c, double vel_crf, double *d_vel, double *vel_force) {
  PLC_CHECK_CTX(c);
  PLC_NEED_FP64(c);
  PLC_REQ(c, d_vel);
  if (vel_crf != 0) {
    PLC_CUDA(c, launch_shift(c, d_vel, vel_crf, c->stream));
    if (vel_force) *vel_force -= vel_crf;
  }
  return PLC_OK;
}

int plc_time_int_vel_rk1(plc_ctx *c, double u_crf, const double *d_u, const double *d_v,
                         const double *d_w, double *d_u1, double *d_v1, double *d_w1) {
  PLC_CHECK_CTX(c);
  PLC_NEED_FP64(c);
  PLC_REQ(c, d_u);
  PLC_REQ(c, d_v);
  PLC_REQ(c, d_w);
  PLC_REQ(c, d_u1);
  PLC_REQ(c, d_v1);
  PLC_REQ(c, d_w1);
  PLC_CUDA(c, launch_rk(c, 1, false, u_crf, d_u, d_v, d_w, d_u1, d_v1, d_w1, c->stream));
  return PLC_OK;
}

int plc_time_int_vel_rk2(plc_ctx *c, double u_crf, double *d_u, double *d_v, double *d_w,
                         const double *d_u1, const double *d_v1, const double *d_w1) {
  PLC_CHECK_CTX(c);
  PLC_NEED_FP64(c);
  PLC_REQ(c, d_u);
  PLC_REQ(c, d_v);
  PLC_REQ(c, d_w);
  PLC_REQ(c, d_u1);
  PLC_REQ(c, d_v1);
  PLC_REQ(c, d_w1);
  PLC_CUDA(c, launch_rk(c, 2, false, u_crf, d_u1, d_v1, d_w1, d_u, d_v, d_w, c->stream));
  return PLC_OK;
}

int plc_correct_vel(plc_ctx *c, const double *d_p, double *d_u, double *d_v, double *d_w) {
  PLC_CHECK_CTX(c);
  PLC_NEED_FP64(c);
  PLC_REQ(c, d_p);
  PLC_REQ(c, d_u);
  PLC_REQ(c, d_v);
  PLC_REQ(c, d_w);
  PLC_CUDA(c, launch_correct(c, false, d_p, d_u, d_v, d_w, c->stream));
  return PLC_OK;
}

int plc_force_vel(plc_ctx *c, double *d_u, double *d_v, double *d_w, double *force_out) {
  PLC_CHECK_CTX(c);
  PLC_NEED_FP64(c);
  PLC_REQ(c, d_u);
  PLC_REQ(c, d_v);
  PLC_REQ(c, d_w);
  double *q[3] = {d_u, d_v, d_w};
  for (int d = 0; d < 3; ++d)
    if (c->prm.is_forced[d]) PLC_CUDA(c, launch_mean(c, d, c->nx, c->ny, q[d], c->stream));
  PLC_CUDA(c, cudaMemcpyAsync(c->h_scal, c->d_sc, sizeof(StepConst), cudaMemcpyDeviceToHost,
                              c->stream));
  PLC_CUDA(c, cudaStreamSynchronize(c->stream));
  StepConst sc;
  memcpy(&sc, c->h_scal, sizeof sc);
  double force[3] = {0.0, 0.0, 0.0};
  for (int d = 0; d < 3; ++d)
    if (c->prm.is_forced[d]) force[d] = c->prm.vel_force[d] - sc.mean[d];  // mod_calcVel.cc:297
  memcpy(c->h_scal, force, sizeof force);
  PLC_CUDA(c, cudaMemcpyAsync(reinterpret_cast<char *>(c->d_sc) + offsetof(StepConst, force),
                              c->h_scal, sizeof force, cudaMemcpyHostToDevice, c->stream));
  PLC_CUDA(c, launch_force_apply(c, false, d_u, d_v, d_w, c->stream));
  PLC_CUDA(c, cudaStreamSynchronize(c->stream));
  if (force_out) memcpy(force_out, force, sizeof force);
  return PLC_OK;
}

// ---- mod_calcRHS ----------------------------------------------------------
int plc_calc_rhs(plc_ctx *c, const double *d_u, const double *d_v, const double *d_w,
                 double *d_rhs) {
  PLC_CHECK_CTX(c);
  PLC_NEED_FP64(c);
  PLC_REQ(c, d_u);
  PLC_REQ(c, d_v);
  PLC_REQ(c, d_w);
  PLC_REQ(c, d_rhs);
  PLC_CUDA(c, launch_calc_rhs(c, d_u, d_v, d_w, d_rhs, c->stream));
  return PLC_OK;
}

// ---- mod_updateBound ------------------------------------------------------
int plc_update_bound_vel(plc_ctx *c, double u_crf, double *d_u, double *d_v, double *d_w) {
  PLC_CHECK_CTX(c);
  PLC_NEED_FP64(c);
  PLC_REQ(c, d_u);
  PLC_REQ(c, d_v);
  PLC_REQ(c, d_w);
  PLC_CUDA(c, launch_bound_vel(c, u_crf, d_u, d_v, d_w, c->stream));
  return PLC_OK;
}

int plc_impose_bc_vel(plc_ctx *c, double *d_u, double *d_v, double *d_w, double u_crf) {
  return plc_update_bound_vel(c, u_crf, d_u, d_v, d_w);
}

int plc_update_bound_p(plc_ctx *c, double *d_p) {
  PLC_CHECK_CTX(c);
  PLC_NEED_FP64(c);
  PLC_REQ(c, d_p);
  PLC_CUDA(c, launch_bound_p(c, d_p, c->stream));
  return PLC_OK;
}

// ---- mod_poisson_solver ---------------------------------------------------
int plc_init_poisson_solver(plc_ctx *c, const double *h_dzf_global, const char *bctype_x,
                            const char *bctype_y, const char *bctype_z) {
  PLC_CHECK_CTX(c);
  PLC_REQ(c, h_dzf_global);
  if (!bctype_x || !bctype_y || !bctype_z || strcmp(bctype_x, "PP") || strcmp(bctype_y, "PP") ||
      strcmp(bctype_z, "NN"))
    return set_error(c, PLC_ERR_ARG, "only bctype PP, PP, NN is supported (mod_fft.cc:20-26)");
  PLC_CUDA(c, cudaStreamSynchronize(c->stream));
  if (int rc = init_poisson(c, h_dzf_global)) return rc;
  if (c->tuned_lines[0] > 0)
    PLC_CUDA(c, fft_set_lines(c, c->tuned_lines[0], c->tuned_lines[1], c->tuned_lines[2]));
  return PLC_OK;
}

int plc_free_poisson_solver(plc_ctx *c) {
  PLC_CHECK_CTX(c);
  PLC_CUDA(c, cudaStreamSynchronize(c->stream));
  free_poisson(c);
  return PLC_OK;
}

#define PLC_NEED_POISSON(c) \
  if (!(c)->poisson_ready) return set_error(c, PLC_ERR_STATE, "Poisson solver not initialised")

int plc_execute_poisson_solver(plc_ctx *c, double *d_p) {
  PLC_CHECK_CTX(c);
  PLC_NEED_FP64(c);
  PLC_REQ(c, d_p);
  PLC_NEED_POISSON(c);
  double *spec = c->d_field[PLC_SPEC];
  PLC_CUDA(c, launch_fft_x_fwd(c, d_p, nullptr, nullptr, nullptr, spec, c->stream));
  PLC_CUDA(c, launch_fft_y(c, spec, false, c->stream));
  PLC_CUDA(c, launch_trid(c, spec, c->stream));
  PLC_CUDA(c, launch_fft_y(c, spec, true, c->stream));
  PLC_CUDA(c, launch_fft_x_bwd(c, spec, d_p, false, c->stream));
  return PLC_OK;
}

int plc_solve_trid(plc_ctx *c, double *d_var) {
  PLC_CHECK_CTX(c);
  PLC_NEED_FP64(c);
  PLC_REQ(c, d_var);
  PLC_NEED_POISSON(c);
  PLC_CUDA(c, launch_trid(c, d_var, c->stream));
  return PLC_OK;
}

// ---- mod_fft --------------------------------------------------------------
int plc_fft_fwd_xpen(plc_ctx *c, const double *d_p, double *d_var) {
  PLC_CHECK_CTX(c);
  PLC_NEED_FP64(c);
  PLC_REQ(c, d_p);
  PLC_REQ(c, d_var);
  PLC_NEED_POISSON(c);
  PLC_CUDA(c, launch_fft_x_fwd(c, d_p, nullptr, nullptr, nullptr, d_var, c->stream));
  return PLC_OK;
}

int plc_fft_bwd_xpen(plc_ctx *c, const double *d_var, double *d_p) {
  PLC_CHECK_CTX(c);
  PLC_NEED_FP64(c);
  PLC_REQ(c, d_p);
  PLC_REQ(c, d_var);
  PLC_NEED_POISSON(c);
  PLC_CUDA(c, launch_fft_x_bwd(c, d_var, d_p, false, c->stream));
  return PLC_OK;
}

int plc_fft_fwd_ypen(plc_ctx *c, double *d_var) {
  PLC_CHECK_CTX(c);
  PLC_NEED_FP64(c);
  PLC_REQ(c, d_var);
  PLC_NEED_POISSON(c);
  PLC_CUDA(c, launch_fft_y(c, d_var, false, c->stream));
  return PLC_OK;
}

int plc_fft_bwd_ypen(plc_ctx *c, double *d_var) {
  PLC_CHECK_CTX(c);
  PLC_NEED_FP64(c);
  PLC_REQ(c, d_var);
  PLC_NEED_POISSON(c);
  PLC_CUDA(c, launch_fft_y(c, d_var, true, c->stream));
  return PLC_OK;
}

int plc_get_eigen_values(int ist, int isz, int isz_global, const char *bctype, double *h_lambda) {
  if (!bctype || strcmp(bctype, "PP") || !h_lambda || isz_global < 2 || ist < 1 ||
      ist + isz - 1 > isz_global)
    return set_error(nullptr, PLC_ERR_ARG, "bad arguments to get_eigen_values (PP only)");
  host_eigen_values(ist, isz, isz_global, h_lambda);
  return PLC_OK;
}

// ---- mod_utils ------------------------------------------------------------
int plc_mean(plc_ctx *c, int nx_global, int ny_global, const double *d_var, double *mean) {
  PLC_CHECK_CTX(c);
  PLC_NEED_FP64(c);
  PLC_REQ(c, d_var);
  PLC_REQ(c, mean);
  return mean_of(c, nx_global, ny_global, d_var, mean);
}

int plc_check_nan(plc_ctx *c, const double *d_var, int *passed) {
  PLC_CHECK_CTX(c);
  PLC_NEED_FP64(c);
  PLC_REQ(c, d_var);
  PLC_REQ(c, passed);
  if (int rc = run_check(c, 1, d_var, d_var, d_var)) return rc;
  *passed = c->h_check->nan_found ? 0 : 1;
  return PLC_OK;
}

int plc_calc_max_cfl(plc_ctx *c, const double *d_u, const double *d_v, const double *d_w,
                     plc_value_index *cfl_max) {
  PLC_CHECK_CTX(c);
  PLC_NEED_FP64(c);
  PLC_REQ(c, d_u);
  PLC_REQ(c, d_v);
  PLC_REQ(c, d_w);
  PLC_REQ(c, cfl_max);
  if (int rc = run_check(c, 2, d_u, d_v, d_w)) return rc;
  to_ijk(c, c->h_check->cfl_idx, cfl_max, c->h_check->cfl * c->dt_host);  // mod_utils.cc:144
  return PLC_OK;
}

int plc_calc_max_div(plc_ctx *c, const double *d_u, const double *d_v, const double *d_w,
                     plc_value_index *div_max) {
  PLC_CHECK_CTX(c);
  PLC_NEED_FP64(c);
  PLC_REQ(c, d_u);
  PLC_REQ(c, d_v);
  PLC_REQ(c, d_w);
  PLC_REQ(c, div_max);
  if (int rc = run_check(c, 4, d_u, d_v, d_w)) return rc;
  to_ijk(c, c->h_check->div_idx, div_max, c->h_check->div);
  return PLC_OK;
}

int plc_check(plc_ctx *c, int *nan_passed, plc_value_index *cfl_max, plc_value_index *div_max) {
  PLC_CHECK_CTX(c);
  if (int rc = run_check_fields(c, 7)) return rc;
  c->last_nan_passed = c->h_check->nan_found ? 0 : 1;
  to_ijk(c, c->h_check->cfl_idx, &c->last_cfl, c->h_check->cfl * c->dt_host);
  to_ijk(c, c->h_check->div_idx, &c->last_div, c->h_check->div);
  if (nan_passed) *nan_passed = c->last_nan_passed;
  if (cfl_max) *cfl_max = c->last_cfl;
  if (div_max) *div_max = c->last_div;
  return PLC_OK;
}

int plc_last_check(plc_ctx *c, int *nan_passed, plc_value_index *cfl_max,
                   plc_value_index *div_max) {
  PLC_CHECK_CTX(c);
  if (nan_passed) *nan_passed = c->last_nan_passed;
  if (cfl_max) *cfl_max = c->last_cfl;
  if (div_max) *div_max = c->last_div;
  return PLC_OK;
}

// ---- mod_initFlow ---------------------------------------------------------
int plc_init_flow(plc_ctx *c) {
  PLC_CHECK_CTX(c);
  const plc_params &P = c->prm;
  const int nz = c->nz;
  std::vector<double> prof(nz + 2, 0.0);
  bool is_mean = false;
  if (P.initial_field == PLC_INIT_UNI) {
    for (int k = 1; k <= nz; ++k) prof[k] = P.u0;
  } else if (P.initial_field == PLC_INIT_POI) {  // mod_initFlow.cc:16-21
    for (int k = 1; k <= nz; ++k) {
      const double z = c->h_zc_global[k] / P.lz;
      prof[k] = 6.0 * (1.0 - z) * z * P.u_ref;
    }
    is_mean = true;
  } else if (P.initial_field == PLC_INIT_LOG) {  // mod_initFlow.cc:23-30
    const double retau = 0.09 * pow(P.re, 0.88);
    for (int k = 1; k <= nz; ++k) {
      const double zn = c->h_zc_global[k] / P.lz;
      const double z = fmin(zn, 1.0 - zn) * 2.0 * retau;
      prof[k] = (z <= 11.6 ? z : 2.5 * log(z) + 5.5);
    }
    is_mean = true;
  } else if (P.initial_field == PLC_INIT_MPI) {
    for (int k = 1; k <= nz; ++k) prof[k] = 0.0;  // rank 0
  } else {
    return set_error(c, PLC_ERR_ARG, "unknown initial_field");
  }
  const int rc = c->mixed ? init_fields(c, prof, is_mean, c->f_field)
                          : init_fields(c, prof, is_mean, c->d_field);
  if (rc != PLC_OK) return rc;
  // the graph bakes the forcing configuration in: rebuild it on the next step
  drop_graph(c);
  return PLC_OK;
}

// main.cc:77-82 after fields were uploaded (inputData on restart): u -= u_crf
// with vel_force[0] shifted likewise, then the velocity and pressure boundary
// update, in either form.
int plc_finish_input(plc_ctx *c) {
  PLC_CHECK_CTX(c);
  const plc_params &P = c->prm;
  if (P.u_crf != 0.0) {
    if (int rc = shift_field(c, PLC_U, P.u_crf)) return rc;
    c->prm.vel_force[0] -= P.u_crf;
  }
  if (c->mixed) {
    PLC_CUDA(c, launch_bound_vel(c, P.u_crf, c->f_field[PLC_U], c->f_field[PLC_V],
                                 c->f_field[PLC_W], c->stream));
    PLC_CUDA(c, launch_bound_p(c, c->f_field[PLC_P], c->stream));
  } else {
    PLC_CUDA(c, launch_bound_vel(c, P.u_crf, c->d_field[PLC_U], c->d_field[PLC_V],
                                 c->d_field[PLC_W], c->stream));
    PLC_CUDA(c, launch_bound_p(c, c->d_field[PLC_P], c->stream));
  }
  PLC_CUDA(c, cudaStreamSynchronize(c->stream));
  drop_graph(c);  // the graph bakes vel_force in
  return PLC_OK;
}

// ---- fused time step ------------------------------------------------------
}  // extern "C"

namespace plc {

// The solver's projection on the context's u, v, w (a proposed or uploaded
// field): the velocity halos, p = div(u)/dt (calcRHS), the Poisson solve
// with the pressure halos, u -= dt grad p (correctVel), the velocity halos
// again.  Either form.
template <class T>
int project_t(plc_ctx *c, T *const *f) {
  T *u = f[PLC_U], *v = f[PLC_V], *w = f[PLC_W], *p = f[PLC_P], *spec = f[PLC_SPEC];
  cudaStream_t s = c->stream;
  // the divergence reads the halos and the wall faces: impose them first
  PLC_CUDA(c, launch_bound_vel(c, c->prm.u_crf, u, v, w, s));
  if constexpr (std::is_same<T, double>::value)
    PLC_CUDA(c, launch_fft_x_fwd(c, nullptr, u, v, w, spec, s));
  else
    PLC_CUDA(c, launch_fft_x_fwd(c, u, v, w, spec, s));
  PLC_CUDA(c, launch_fft_y(c, spec, false, s));
  PLC_CUDA(c, launch_trid(c, spec, s));
  PLC_CUDA(c, launch_fft_y(c, spec, true, s));
  PLC_CUDA(c, launch_fft_x_bwd(c, spec, p, true, s));
  PLC_CUDA(c, launch_correct(c, false, p, u, v, w, s));
  PLC_CUDA(c, launch_bound_vel(c, c->prm.u_crf, u, v, w, s));
  PLC_CUDA(c, cudaStreamSynchronize(s));
  return PLC_OK;
}

int pre_steps(plc_ctx *c) {
  const plc_params &P = c->prm;
  if (P.cfl_target > 0.0 && c->nstep == 0) {
    int passed;
    plc_value_index cm, dm;
    if (int rc = plc_check(c, &passed, &cm, &dm)) return rc;
    if (c->h_check->cfl > 0.0)
      if (int rc = upload_step_consts(c, P.cfl_target / c->h_check->cfl)) return rc;
  }
  return PLC_OK;
}

bool step_needs_host(const plc_ctx *c) {
  const plc_params &P = c->prm;
  const long long n = c->nstep + 1;
  if (P.cfl_target > 0.0 && n < P.nt_check && (n & (n - 1)) == 0) return true;
  return P.nt_check > 0 && n % P.nt_check == 0;
}

// post_step in two halves: post_step_begin queues the step's checks (when
// the step needs them) on the context's stream and their result's copy to
// the host; post_step_end waits for them and acts on the result.  Several
// contexts (an ensemble's members) thus share one wait.
int post_step_begin(plc_ctx *c) {
  const plc_params &P = c->prm;
  ++c->nstep;
  c->pending_check = 0;
  // Under CFL control the first steps also re-evaluate dt (steps 1, 2, 4,
  // ... below nt_check), without the limit checks: the first forcing step
  // moves the bulk velocity from that of the initial field (the reference's
  // rescale divides by nz*ny, mod_initFlow.cc:92) to vel_force, which changes
  // the CFL rate by up to nx/nz.
  if (P.cfl_target > 0.0 && c->nstep < P.nt_check && (c->nstep & (c->nstep - 1)) == 0)
    c->pending_check = 2;
  else if (P.nt_check > 0 && c->nstep % P.nt_check == 0)
    c->pending_check = 7;  // main.cc:156-178
  if (!c->pending_check) return PLC_OK;
  if (c->mixed)
    PLC_CUDA(c, launch_check(c, c->f_field[PLC_U], c->f_field[PLC_V], c->f_field[PLC_W],
                             c->pending_check, c->stream));
  else
    PLC_CUDA(c, launch_check(c, c->d_field[PLC_U], c->d_field[PLC_V], c->d_field[PLC_W],
                             c->pending_check, c->stream));
  PLC_CUDA(c, cudaMemcpyAsync(c->h_check, c->d_check, sizeof(CheckResult), cudaMemcpyDeviceToHost,
                              c->stream));
  return PLC_OK;
}

// Acts on a full check's result in c->h_check (main.cc:156-178): the NaN,
// CFL and divergence limits, then the new dt under CFL control -- copied to
// the device here, or (device_dt) already set there by the check's own
// k_cfl_dt, of which the host keeps the same value.
int check_result(plc_ctx *c, bool device_dt) {
  const plc_params &P = c->prm;
  c->last_nan_passed = c->h_check->nan_found ? 0 : 1;
  to_ijk(c, c->h_check->cfl_idx, &c->last_cfl, c->h_check->cfl * c->dt_host);
  to_ijk(c, c->h_check->div_idx, &c->last_div, c->h_check->div);
  const int passed = c->last_nan_passed;
  const plc_value_index cm = c->last_cfl, dm = c->last_div;
  bool ok = passed != 0;
  std::string msg;
  if (!passed) msg += "PowerLLEL.ERROR.checkNaN: NaN has been detected in <u>!\n";
  if (cm.value > P.cfl_limit || std::isnan(cm.value)) {
    ok = false;
    msg += "PowerLLEL.ERROR.checkCFL: Maximum CFL number exceeds the threshold specified by the user!\n";
  }
  // The mixed form's divergence is at FP32 rounding level: its limit is
  // div_limit scaled by the ratio of the unit round-offs, 2^-24 / 2^-53.
  const double div_limit = c->mixed ? P.div_limit * 536870912.0 : P.div_limit;
  if (dm.value > div_limit || std::isnan(dm.value)) {
    ok = false;
    msg += "PowerLLEL.ERROR.checkDiv: Maximum divergence exceeds the threshold specified by the user!\n";
  }
  if (!ok) {
    char buf[256];
    snprintf(buf, sizeof buf,
             "PowerLLEL.ERROR: nt = %9lld, cfl_max = %10.3e at (%5d,%5d,%5d), div_max = %10.3e at (%5d,%5d,%5d)",
             c->nstep, cm.value, cm.ig, cm.jg, cm.kg, dm.value, dm.ig, dm.jg, dm.kg);
    return set_error(c, PLC_ERR_CHECK, msg + buf);
  }
  if (P.cfl_target > 0.0 && c->h_check->cfl > 0.0) {
    if (device_dt)
      c->dt_host = P.cfl_target / c->h_check->cfl;
    else if (int rc = upload_step_consts_async(c, P.cfl_target / c->h_check->cfl))
      return rc;
  }
  return PLC_OK;
}

int post_step_end(plc_ctx *c) {
  const plc_params &P = c->prm;
  const int what = c->pending_check;
  c->pending_check = 0;
  if (!what) return PLC_OK;
  PLC_CUDA(c, cudaStreamSynchronize(c->stream));
  if (what == 2) {
    if (c->h_check->cfl > 0.0)
      if (int rc = upload_step_consts_async(c, P.cfl_target / c->h_check->cfl)) return rc;
    return PLC_OK;
  }
  return check_result(c, false);
}

int post_step(plc_ctx *c) {
  if (int rc = post_step_begin(c)) return rc;
  return post_step_end(c);
}

namespace {
// CFL control on the device after a full check (the host's arithmetic of
// upload_step_consts: one division for dt, the derived factors from it).
__global__ void k_cfl_dt(const CheckResult *__restrict__ res, StepConst *sc, double cfl_target,
                         double dx_inv, double dy_inv) {
  const double rate = res->cfl;
  if (rate > 0.0) {
    const double dt = cfl_target / rate;
    const double dti = 1.0 / dt;
    sc->dt = dt;
    sc->dti = dti;
    sc->dtidxi = dti * dx_inv;
    sc->dtidyi = dti * dy_inv;
    sc->dtdxi = dt * dx_inv;
    sc->dtdyi = dt * dy_inv;
  }
}
}  // namespace

int enqueue_check_tail(plc_ctx *c, cudaStream_t s) {
  if (c->mixed)
    PLC_CUDA(c, launch_check(c, c->f_field[PLC_U], c->f_field[PLC_V], c->f_field[PLC_W], 7, s));
  else
    PLC_CUDA(c, launch_check(c, c->d_field[PLC_U], c->d_field[PLC_V], c->d_field[PLC_W], 7, s));
  if (c->prm.cfl_target > 0.0) {
    k_cfl_dt<<<1, 1, 0, s>>>(c->d_check, c->d_sc, c->prm.cfl_target, c->dx_inv, c->dy_inv);
    PLC_CUDA(c, cudaGetLastError());
  }
  PLC_CUDA(c, cudaMemcpyAsync(c->h_check, c->d_check, sizeof(CheckResult), cudaMemcpyDeviceToHost, s));
  return PLC_OK;
}

bool device_check_due(const plc_ctx *c, int steps) {
  const plc_params &P = c->prm;
  return P.nt_check > 0 && P.nt_check % steps == 0 && (c->nstep + steps) % P.nt_check == 0;
}

int post_steps_device_check(plc_ctx *c, int steps) {
  c->nstep += steps;
  return check_result(c, true);
}

}  // namespace plc

extern "C" {

int plc_project(plc_ctx *c) {
  PLC_CHECK_CTX(c);
  PLC_NEED_POISSON(c);
  return c->mixed ? project_t<float>(c, c->f_field) : project_t<double>(c, c->d_field);
}


// nsteps graph launches with the checks of main.cc:156-178 every nt_check
// steps; the device error word is not read here.
static int step_launches(plc_ctx *c, int nsteps) {
  PLC_CHECK_CTX(c);
  if (nsteps < 0) return set_error(c, PLC_ERR_ARG, "nsteps < 0");
  PLC_NEED_POISSON(c);
  if (int rc = build_graph(c)) return rc;
  if (int rc = pre_steps(c)) return rc;
  for (int s = 0; s < nsteps; ++s) {
    PLC_CUDA(c, cudaGraphLaunch(c->graph, c->stream));
    if (int rc = post_step(c)) return rc;
  }
  return PLC_OK;
}

int plc_step(plc_ctx *c, int nsteps) {
  if (int rc = step_launches(c, nsteps)) return rc;
  return device_error(c);
}

int plc_step_count(plc_ctx *c, long long *count) {
  PLC_CHECK_CTX(c);
  PLC_REQ(c, count);
  *count = c->nstep;
  return PLC_OK;
}

int plc_set_step_count(plc_ctx *c, long long count) {
  PLC_CHECK_CTX(c);
  if (count < 0) return set_error(c, PLC_ERR_ARG, "negative step count");
  c->nstep = count;
  return PLC_OK;
}

int plc_set_sm_budget(plc_ctx *c, int sms) {
  PLC_CHECK_CTX(c);
  if (sms < 1) return set_error(c, PLC_ERR_ARG, "SM budget < 1");
  c->num_sms = sms < c->device_sms ? sms : c->device_sms;
  if (c->poisson_ready) PLC_CUDA(c, fft_set_lines(c, c->fft_lines_xf, c->fft_lines_x, c->fft_lines_y));
  drop_graph(c);
  return PLC_OK;
}

int plc_get_sm_budget(const plc_ctx *c, int *sms) {
  if (!c || !sms) return set_error(nullptr, PLC_ERR_ARG, "null argument");
  *sms = c->num_sms;
  return PLC_OK;
}

int plc_step_timed(plc_ctx *c, int nsteps, double *ms) {
  PLC_CHECK_CTX(c);
  PLC_REQ(c, ms);
  PLC_NEED_POISSON(c);
  if (int rc = build_graph(c)) return rc;
  cudaEvent_t e0, e1;
  PLC_CUDA(c, cudaEventCreate(&e0));
  PLC_CUDA(c, cudaEventCreate(&e1));
  int rc = PLC_OK;
  cudaError_t e = cudaEventRecord(e0, c->stream);
  if (e == cudaSuccess) {
    rc = step_launches(c, nsteps);
    e = cudaEventRecord(e1, c->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float f = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&f, e0, e1);
    *ms = f;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != PLC_OK) return rc;
  if (e != cudaSuccess) return cuda_status(c, e, "step timing events");
  return device_error(c);
}

int plc_get_stream(plc_ctx *c, void **stream) {
  PLC_CHECK_CTX(c);
  PLC_REQ(c, stream);
  *stream = (void *)c->stream;
  return PLC_OK;
}

int plc_profile_step(plc_ctx *c, int nsteps, float *ms_per_kernel, int *count) {
  PLC_CHECK_CTX(c);
  PLC_REQ(c, ms_per_kernel);
  PLC_NEED_POISSON(c);
  const int nk = step_kernels(c);
  cudaEvent_t ev[kStepKernels + 1];
  for (auto &e : ev) PLC_CUDA(c, cudaEventCreate(&e));
  int rc = PLC_OK;
  for (int s = 0; s < nsteps && rc == PLC_OK; ++s) {
    rc = enqueue_step(c, c->stream, ev);
    if (rc != PLC_OK) break;
    cudaError_t e = cudaEventSynchronize(ev[nk]);
    if (e != cudaSuccess) {
      rc = cuda_status(c, e, "cudaEventSynchronize");
      break;
    }
    for (int q = 0; q < nk; ++q) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[q], ev[q + 1]);
      ms_per_kernel[q] += ms;
    }
    ++c->nstep;
  }
  for (auto &e : ev) cudaEventDestroy(e);
  if (count) *count = nk;
  return rc;
}

const char *plc_step_kernel_name(int i) {
  return (i >= 0 && i < kStepKernels) ? kStepKernelNames[i] : "";
}

const char *plc_step_kernel_name_ctx(const plc_ctx *c, int i) {
  if (!c || !c->mixed) return plc_step_kernel_name(i);
  return (i >= 0 && i < kStepKernelsMixed) ? kStepKernelNamesMixed[i] : "";
}

int plc_mesh_by_func(int mesh_type, int stretch_func, double stretch_ratio, int nz, double lz,
                     double *h_dzf_global) {
  if (!h_dzf_global || nz < 1 || !(lz > 0.0))
    return set_error(nullptr, PLC_ERR_ARG, "bad arguments to plc_mesh_by_func");
  host_mesh_by_func(mesh_type, stretch_func, stretch_ratio, nz, lz, h_dzf_global);
  return PLC_OK;
}

int plc_trid_tables(int nx, int ny, int nz, double lx, double ly, const double *h_dzf_global,
                    double *h_rpiv, double *h_a, double *h_c) {
  if (!h_dzf_global || !h_rpiv || nx < 2 || ny < 2 || nz < 2 || nx % 2 || ny % 2)
    return set_error(nullptr, PLC_ERR_ARG, "bad arguments to plc_trid_tables");
  std::vector<double> rpiv, a, cc;
  host_trid_tables(nx, ny, nz, lx / nx, ly / ny, h_dzf_global, rpiv, a, cc);
  memcpy(h_rpiv, rpiv.data(), rpiv.size() * sizeof(double));
  if (h_a) memcpy(h_a, a.data(), a.size() * sizeof(double));
  if (h_c) memcpy(h_c, cc.data(), cc.size() * sizeof(double));
  return PLC_OK;
}

int plc_host_alloc(size_t bytes, void **ptr) {
  if (!ptr) return set_error(nullptr, PLC_ERR_ARG, "null pointer");
  cudaError_t e = cudaMallocHost(ptr, bytes);
  if (e != cudaSuccess) return cuda_status(nullptr, e, "cudaMallocHost");
  return PLC_OK;
}

int plc_host_free(void *ptr) {
  if (ptr) {
    cudaError_t e = cudaFreeHost(ptr);
    if (e != cudaSuccess) return cuda_status(nullptr, e, "cudaFreeHost");
  }
  return PLC_OK;
}

int plc_kernels_per_step(plc_ctx *c, int *count) {
  PLC_CHECK_CTX(c);
  PLC_REQ(c, count);
  if (int rc = build_graph(c)) return rc;
  *count = c->graph_kernels;
  return PLC_OK;
}

}  // extern "C"
