// Internal declarations shared by the translation units of libplc.so.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "plc.h"

namespace plc {

// indices into plc_ctx::order: the step kernels whose plane order is a choice
enum StepKernel { SK_RK2, SK_YF, SK_YB, SK_XB, SK_ORDERS };

// ---------------------------------------------------------------------------
// Geometry passed by value to every kernel.
// ---------------------------------------------------------------------------

struct Geo {
  int nx, ny, nz;
  int X, Y;           // halo'd x and y lengths (nx+2, ny+2)
  long long XY;       // X*Y
  double dx_inv, dy_inv, re_inv;
  const double *dzf, *dzf_inv, *dzc_inv, *dzflzi;  // device, nz+2 each
  __host__ __device__ long long at(int i, int j, int k) const {
    return (long long)i + (long long)X * j + XY * k;
  }
};

// Per-step scalars that may change on the device (CFL-controlled dt, the
// bulk forcing of the step).  Kernels read them through a device pointer so
// that a captured graph stays valid when they change.
struct StepConst {
  double dt, dti, dtidxi, dtidyi, dtdxi, dtdyi;
  double force[3];   // vel_force - mean of the last forcing
  double mean[3];
  double cfl_rate;   // max |u|/dx + |v|/dy + |w|/dz of the last check (no dt)
};

// Result of the device-side NaN/CFL/divergence check.
struct CheckResult {
  int nan_found;
  int pad;
  double cfl;        // max CFL rate (without dt)
  long long cfl_idx; // halo'd linear index, -1 if none
  double div;
  long long div_idx;
};

// Complex FFT plan for a line length n = 2^a 3^b.
struct FftPlan {
  int n = 0;
  int npass = 0;
  int radix[16] = {0};
  double2 *tw = nullptr;   // device, n entries: exp(-2 pi i t / n)
  float2 *tw32 = nullptr;  // the same rounded to FP32 (mixed form)
};

// capacity (blocks) of each plane of the reduction partials array
constexpr int kMaxBlocksReduce = 4096;

// running statistics of mod_statistics (src/mod_statistics.hh:13): u, v, w,
// u*u, v*v, w*w, u*v, u*w, v*w, p, p*p
constexpr int kStatVars = 11;

// Mixed form: Thomas systems whose packed x and y indices are both below
// kLowModes (wavenumbers |m| < kLowModes/2, the Nyquist line of each axis
// included) sweep in FP64; the others in FP32.
constexpr int kLowModes = 16;

// output files and monitor state of the data-I/O entry points (plc_io.cc)
struct IoState;

}  // namespace plc

struct plc_ctx {
  plc_params prm;
  int device = 0;
  bool mixed = false;  // PLC_MIXED: FP32 fields in f_field, d_field unused
  int nx = 0, ny = 0, nz = 0;
  int pitch = 0;       // x stride of the halo'd fields: nx+2 (FP64), a multiple of 4 (FP32)
  double dx = 0, dy = 0, dx_inv = 0, dy_inv = 0, re_inv = 0;
  size_t nfield = 0;  // pitch*(ny+2)*(nz+2)
  size_t nspec = 0;   // nx*ny*nz
  // host copies of the mesh (nz+2 each)
  std::vector<double> h_dzf_global, h_dzf, h_dzf_inv, h_dzc, h_dzc_inv, h_dzflzi,
      h_zc_global;
  double *d_mesh = nullptr;  // dzf | dzf_inv | dzc_inv | dzflzi
  double *d_field[8] = {nullptr};
  float *f_field[8] = {nullptr};  // mixed form: the same fields in FP32
  // Poisson solver state
  bool poisson_ready = false;
  double *d_rpiv = nullptr;   // 1/b, (nz, ny/2+1, nx/2+1)
  double *d_ac = nullptr;     // a[nz] | c[nz]
  double *d_low = nullptr;    // mixed form: FP64 sweep values of the low modes
  float *d_rpiv32 = nullptr;  // mixed form: the pivot table in FP32
  float *d_ac32 = nullptr;    // mixed form: a[nz] | c[nz] in FP32
  float *d_coef32 = nullptr;  // mixed form: per-plane RK coefficients
  double *d_mean_partials = nullptr;  // mixed form: bulk-mean partials, 3 * RK blocks
  plc::FftPlan plan_x, plan_y;
  int fft_lines_x = 1, fft_lines_xf = 1, fft_lines_y = 1;  // line pairs per tile
  int grid_xf = 1, grid_xb = 1, grid_y = 1;                 // persistent grids
  int tuned_lines[3] = {0, 0, 0};  // autotuned (xf, x, y) line pairs, 0 = not tuned
  // radix plan family of the x and y transforms (0: 16/8/4/2/3 passes; 1: two
  // passes ending in radix 24, lengths 24 .. 384 with one factor 3); autotuned
  // with the tiles unless the environment pins them
  int fft_plan_x = 0, fft_plan_y = 0;
  // family of the forward x transform (-1: that of the backward one)
  int fft_plan_xf = -1;
  // Thomas sweep with the columns on chip (else the streaming sweep), chosen
  // by the autotuner; the device's shared-memory limit per block
  bool trid_tile = true;
  bool trid_pinned = false;  // PLC_TRID = "tile" or "stream"
  // z planes per block of the RK stages (0: the kernels' maximum), chosen by
  // the autotuner among kRkChunks; PLC_RK_KCHUNK pins it
  int rk_kchunk = 0;
  bool rk_pinned = false;  // PLC_RK_KCHUNK(_F32) set
  // mixed form: the second RK stage carries its z-face terms (at 3 blocks
  // per SM), chosen by the autotuner; PLC_RK2_CARRY pins it
  bool rk2_carry = false;
  bool rk2_carry_pinned = false;
  int pending_check = 0;   // checks queued by post_step_begin (0: none)
  size_t trid_smem_max = 0;
  bool fft_plans_pinned = false;
  // Plane order of the step kernels (0: low planes first, 1: high planes
  // first), set per form at creation from measurements; only the speed
  // depends on it.
  unsigned char order[plc::SK_ORDERS] = {0, 0, 0, 0};
  // scalars and scratch
  plc::StepConst *d_sc = nullptr;
  double *d_partials = nullptr;        // 8 * kMaxBlocksReduce
  unsigned int *d_counter = nullptr;   // last-block counters
  int *d_err = nullptr;                // set by a kernel whose bounded wait gave up
  int num_sms = 148;      // SM budget of the persistent grids (plc_set_sm_budget)
  int device_sms = 148;   // SMs of the device
  plc::CheckResult *d_check = nullptr;
  plc::CheckResult *h_check = nullptr;  // pinned
  double *h_scal = nullptr;             // pinned scalars
  double dt_host = 0;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  unsigned graph_epoch = 0;  // bumped whenever a captured step becomes stale
  int graph_kernels = 0;
  long long nstep = 0;
  // statistics (plc_stat_init): running sums, nx*ny*nz doubles each
  double *d_stat[plc::kStatVars] = {nullptr};
  int stat_nts = 0, stat_nte = 0, stat_nspl = 0;
  bool stat_ready = false;
  plc::IoState *io = nullptr;  // plc_output_init / plc_set_output_dir
  int last_nan_passed = 1;
  plc_value_index last_cfl{0, 1, 1, 1}, last_div{0, 1, 1, 1};
  std::string err;
  plc::Geo geo() const;
};

namespace plc {

// error helpers ---------------------------------------------------------------
int set_error(plc_ctx *ctx, int code, const std::string &msg);
int cuda_status(plc_ctx *ctx, cudaError_t e, const char *what);
#define PLC_CUDA(ctx, call)                                     \
  do {                                                          \
    cudaError_t _e = (call);                                    \
    if (_e != cudaSuccess) return plc::cuda_status(ctx, _e, #call); \
  } while (0)
#define PLC_LAUNCH(ctx, what)                                   \
  do {                                                          \
    cudaError_t _e = cudaGetLastError();                        \
    if (_e != cudaSuccess) return plc::cuda_status(ctx, _e, what); \
  } while (0)

// host-side mesh and solver set-up (plc_host.cc, compiled without FMA
// contraction so that the arithmetic follows the reference's host loops)
void host_mesh_by_func(int mesh_type, int stretch_func, double stretch_ratio,
                       int nz, double lz, double *dzf_global);
void host_mesh_derived(int nz, double lz, const double *dzf_global, double *dzf,
                       double *dzf_inv, double *dzc, double *dzc_inv,
                       double *dzflzi, double *zc_global);
void host_eigen_values(int ist, int isz, int isz_global, double *lambda);
// Reciprocal pre-factored pivots 1/b (0 where b == 0), table layout
// (nz, ny/2+1, nx/2+1), plus a[nz] and c[nz].
void host_trid_tables(int nx, int ny, int nz, double dx, double dy,
                      const double *dzf_global, std::vector<double> &rpiv,
                      std::vector<double> &a, std::vector<double> &c);
void host_twiddles(int n, std::vector<double> &re_im);
bool host_fft_factor(int n, int *radix, int *npass);
int host_parse_param_json(const char *path, plc_params *prm, std::string &err);

// kernel launchers (return cudaError_t of the launch) ---------------------------
// RK z-chunk candidates and the chunk a launch uses (at most kmax and nz)
constexpr int kRkChunks[4] = {8, 16, 24, 32};
inline int rk_chunk(const plc_ctx *c, int kmax);
cudaError_t launch_rk(const plc_ctx *c, int stage, bool fuse_bc, double u_crf,
                      const double *qu, const double *qv, const double *qw,
                      double *ou, double *ov, double *ow, cudaStream_t s);
// mixed form (plc_mixed.cu): FP32 operands, FP32 arithmetic
cudaError_t launch_rk(const plc_ctx *c, int stage, bool fuse_bc, double u_crf,
                      const float *qu, const float *qv, const float *qw,
                      float *ou, float *ov, float *ow, cudaStream_t s);
// FP64 rows of `len` elements (the reference's layout) <-> FP32 rows of
// stride `pitch` (the context's layout)
cudaError_t launch_to_f32(const plc_ctx *c, const double *src, float *dst, long long rows, int len,
                          int pitch, cudaStream_t s);
cudaError_t launch_to_f64(const plc_ctx *c, const float *src, double *dst, long long rows, int len,
                          int pitch, cudaStream_t s);
// shared-memory limit of the FP32 RK kernels on the current device
cudaError_t rk32_configure();
cudaError_t rk_tma_configure();
// blocks of the FP32 RK grid
long long rk32_blocks(const plc_ctx *c);
// per-plane coefficient rows of the FP32 RK kernels, rk32_coef_floats() per plane
void host_rk32_coef(const plc_ctx *c, std::vector<float> &out);
int rk32_coef_floats();
cudaError_t launch_calc_rhs(const plc_ctx *c, const double *u, const double *v,
                            const double *w, double *rhs, cudaStream_t s);
cudaError_t launch_correct(const plc_ctx *c, bool fused, const double *p,
                           double *u, double *v, double *w, cudaStream_t s);
cudaError_t launch_correct(const plc_ctx *c, bool fused, const float *p,
                           float *u, float *v, float *w, cudaStream_t s);
cudaError_t launch_force_apply(const plc_ctx *c, bool fuse_bc, double *u,
                               double *v, double *w, cudaStream_t s);
cudaError_t launch_force_apply(const plc_ctx *c, bool fuse_bc, float *u,
                               float *v, float *w, cudaStream_t s);
cudaError_t launch_mean(const plc_ctx *c, int comp, int nxg, int nyg,
                        const double *var, cudaStream_t s);
cudaError_t launch_mean(const plc_ctx *c, int comp, int nxg, int nyg,
                        const float *var, cudaStream_t s);
cudaError_t launch_bound_vel(const plc_ctx *c, double u_crf, double *u,
                             double *v, double *w, cudaStream_t s);
cudaError_t launch_bound_vel(const plc_ctx *c, double u_crf, float *u,
                             float *v, float *w, cudaStream_t s);
cudaError_t launch_bound_p(const plc_ctx *c, double *p, cudaStream_t s);
cudaError_t launch_bound_p(const plc_ctx *c, float *p, cudaStream_t s);
cudaError_t launch_shift(const plc_ctx *c, double *var, double delta,
                         cudaStream_t s);
cudaError_t launch_shift(const plc_ctx *c, float *var, double delta,
                         cudaStream_t s);
cudaError_t launch_fft_x_fwd(const plc_ctx *c, const double *p, const double *u,
                             const double *v, const double *w, double *var,
                             cudaStream_t s);
// mixed form: calcRHS fused with the forward x transform only
cudaError_t launch_fft_x_fwd(const plc_ctx *c, const float *u, const float *v,
                             const float *w, float *var, cudaStream_t s);
cudaError_t launch_fft_x_bwd(const plc_ctx *c, const double *var, double *p,
                             bool fuse_bc, cudaStream_t s);
cudaError_t launch_fft_x_bwd(const plc_ctx *c, const float *var, float *p,
                             bool fuse_bc, cudaStream_t s);
cudaError_t launch_fft_y(const plc_ctx *c, double *var, bool inverse,
                         cudaStream_t s);
cudaError_t launch_fft_y(const plc_ctx *c, float *var, bool inverse,
                         cudaStream_t s);
cudaError_t launch_trid(const plc_ctx *c, double *var, cudaStream_t s);
cudaError_t launch_trid(const plc_ctx *c, float *var, cudaStream_t s);
cudaError_t launch_check(const plc_ctx *c, const double *u, const double *v,
                         const double *w, int what, cudaStream_t s);
cudaError_t launch_check(const plc_ctx *c, const float *u, const float *v,
                         const float *w, int what, cudaStream_t s);
cudaError_t launch_init_flow(const plc_ctx *c, double *u, double *v, double *w,
                             const double *d_prof, cudaStream_t s);
cudaError_t launch_init_flow(const plc_ctx *c, float *u, float *v, float *w,
                             const double *d_prof, cudaStream_t s);
cudaError_t launch_scale(const plc_ctx *c, double *var, const double *d_mult,
                         cudaStream_t s);
cudaError_t launch_scale(const plc_ctx *c, float *var, const double *d_mult,
                         cudaStream_t s);
// streamwise vortices of plc_init_flow (zf: nz+1 face heights, zf[0] = 0)
cudaError_t launch_add_vortices(const plc_ctx *c, double *v, double *w, const double *d_zf,
                                cudaStream_t s);
cudaError_t launch_add_vortices(const plc_ctx *c, float *v, float *w, const double *d_zf,
                                cudaStream_t s);
size_t fft_smem_bytes(int n, int lines);
cudaError_t fft_configure(size_t max_bytes);
cudaError_t fft_setup(plc_ctx *c, size_t smem_cap_per_block, size_t dev_max);
// times the feasible tile sizes of each transform on the context's buffers
// and keeps the fastest (overwrites the spectral array and p)
cudaError_t fft_autotune(plc_ctx *c);
// whether a line length has the radix-24 plan family as well
bool fft_has_two_plans(int n);
// a warp-line plan (family 2) for length n with `lines_axis` real lines
bool fft_has_warp_plan(int n, int lines_axis);
// a two-pass y plan (family 3) for y lines of length ny over nx columns
bool fft_has_y2_plan(int ny, int nx, int elem);
// a two-pass x plan (family 3) for x lines of length nx over ny rows
bool fft_has_x2_plan(int nx, int ny);
cudaError_t fft_set_lines(plc_ctx *c, int lines_xf, int lines_x, int lines_y);

// Batched launches over the mixed-form channels of an ensemble: one launch
// per step stage covers all the channels (the stages whose code depends on a
// line length: one launch per length, on the streams ss[0..ns) in turn, which
// the caller forks from and joins to its own), each block working on a tile
// of one channel.  The arguments of up to kBatchMax channels travel in the
// kernel parameters; more channels take more launches.  Each channel's
// results are those of its own step with the same transform families.
constexpr int kBatchMax = 32;
// Choices of the batched launches, made by the ensemble's batch autotuner:
// per transform (forward x, backward x, y) and line-length group (len_key:
// the compiled length, 0 for the runtime plan) the plan family and the line
// pairs per tile; the RK stages' z planes per block (0: each channel's own).
// Without a choice for a group, the family of the group's largest channel
// and the largest tile all its channels admit are used.
struct BatchPlan {
  struct Group {
    int len_key, pl, nl;
  };
  std::vector<Group> dir[3];  // BATCH_XF, BATCH_XB, BATCH_Y
  int rk_kchunk = 0;
  int rk_minb = 4;  // resident blocks per SM the RK kernels are compiled for (3 or 4)
  bool trid_tile = false;  // the Thomas sweep with its columns on chip
  // programmatic dependent launch: each batched kernel launched with
  // programmatic stream serialisation, so that its blocks become resident
  // while the kernels it depends on drain
  bool pdl = false;
};
enum BatchDir { BATCH_XF = 0, BATCH_XB = 1, BATCH_Y = 2 };
// Launches a batched kernel k(p) (one parameter struct) on stream s; with
// pdl, with programmatic stream serialisation: allowed only for kernels
// whose every block calls batch_grid_sync() first.  In a stream capture the
// edges from the kernels it depends on become programmatic edges.
template <class P>
cudaError_t launch_batched(void (*k)(P), unsigned grid, dim3 block, size_t smem, cudaStream_t s,
                           const P &p, bool pdl) {
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = pdl ? at : nullptr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k, p);
}
cudaError_t launch_rk_batch(plc_ctx *const *cs, int n, int stage, int kchunk, int minb,
                            cudaStream_t s, bool pdl = false);
cudaError_t launch_fft_x_fwd_batch(plc_ctx *const *cs, int n, const BatchPlan *bp,
                                   const cudaStream_t *ss, int ns);
cudaError_t launch_fft_y_batch(plc_ctx *const *cs, int n, bool inverse, const BatchPlan *bp,
                               const cudaStream_t *ss, int ns);
cudaError_t launch_trid_batch(plc_ctx *const *cs, int n, bool tile, cudaStream_t s,
                              bool pdl = false);
// whether every channel admits the batched on-chip Thomas sweep
bool trid_tile_batch_ok(plc_ctx *const *cs, int n);
cudaError_t launch_fft_x_bwd_batch(plc_ctx *const *cs, int n, const BatchPlan *bp,
                                   const cudaStream_t *ss, int ns);
cudaError_t launch_correct_batch(plc_ctx *const *cs, int n, cudaStream_t s, bool pdl = false);
// the full checks of the mixed-form channels at a graph's check step: results
// on the device and in each channel's pinned host copy, the new dt under CFL
// control set on the device
cudaError_t launch_check_batch(plc_ctx *const *cs, int n, cudaStream_t s, bool pdl = false);
// the number of launches (line-length groups) of the batched x and y stages
int fft_batch_groups(plc_ctx *const *cs, int n, bool ydir);
// times the candidate families and tiles of every group of the batched
// transforms on stream s (overwrites the channels' spectral arrays and p)
// and the RK stages' z chunks (overwrites u1, v1, w1, u, v, w), keeping the
// fastest in *bp
cudaError_t batch_autotune(plc_ctx *const *cs, int n, cudaStream_t s, BatchPlan *bp);

// var -= delta on the interior of the context's field (either form), synchronous
int shift_field(plc_ctx *c, int field, double delta);
// the launches of one fused step on stream s (for capture into a caller's graph)
int capture_step(plc_ctx *c, cudaStream_t s);
// the context's captured step, built if needed
int step_graph(plc_ctx *c, cudaGraphExec_t *g);
// releases the context's captured step (it is rebuilt on the next step)
void drop_graph(plc_ctx *c);
// host work around graph-launched steps: before the first step (CFL-controlled
// dt) and after each step (step counter, early dt re-evaluation, the checks
// every nt_check steps); post_step expects the step's work to be ordered
// before the context's stream
int pre_steps(plc_ctx *c);
int post_step(plc_ctx *c);
// post_step in two halves (queue the checks; wait and act on them), so that
// several contexts share one wait
int post_step_begin(plc_ctx *c);
int post_step_end(plc_ctx *c);
// Checks inside a captured graph: after the last of `steps` steps that ends
// on a check step, enqueue_check_tail queues the full check (main.cc:156-178)
// on stream s, the new dt under CFL control set on the device, and the
// result's copy to the host; device_check_due says whether the next `steps`
// steps end on a check step (steps a divisor of nt_check) and
// post_steps_device_check advances the step counter and acts on the copied
// result once the graph has finished.
int enqueue_check_tail(plc_ctx *c, cudaStream_t s);
bool device_check_due(const plc_ctx *c, int steps);
int post_steps_device_check(plc_ctx *c, int steps);
// true when post_step will do host work after the next step
bool step_needs_host(const plc_ctx *c);
// closes the monitor files and releases the I/O state (plc_io.cc)
void io_free(plc_ctx *c);

inline int rk_chunk(const plc_ctx *c, int kmax) {
  int k = c->rk_kchunk > 0 ? c->rk_kchunk : kmax;
  if (k > kmax) k = kmax;
  return k < c->nz ? k : c->nz;
}

}  // namespace plc
