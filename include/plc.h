/*
 * plc.h -- C ABI of the B200 (sm_100a) PowerLLEL_Channel DNS time step.
 *
 * This is the drop-in boundary for the hot path of xiejb6/PowerLLEL_Channel_SYCL
 * at p_row = p_col = 1: one entry point per module function of the reference
 * (src/mod_calcVel.hh, mod_calcRHS.hh, mod_updateBound.hh,
 * mod_poisson_solver.hh, mod_fft.hh, mod_utils.hh) plus a fused, CUDA-graph
 * captured time step.  Every function returns PLC_OK (0) or a negative status;
 * plc_last_error(ctx) gives the message (plc_last_error(NULL) for failures of
 * plc_create and of the context-free helpers).
 *
 * Field layout (same as the reference's _Array3D with one halo cell per side,
 * src/mod_type.hh:81-306): interior nx*ny*nz, stored as (nx+2)*(ny+2)*(nz+2)
 * doubles, x fastest; the reference index (i,j,k), 0 <= i <= nx+1, maps to
 * i + (nx+2)*(j + (ny+2)*k).  The spectral work array of the Poisson solver
 * (var_xpen of src/mod_poisson_solver.cc:196-198) is nx*ny*nz doubles, x
 * fastest, no halos, in the reference's packed real-spectrum order.
 *
 * Pointers named d_* are DEVICE pointers on the context's GPU; h_* are host
 * pointers.  Calls are ordered on the context's CUDA stream; functions that
 * return host values (plc_mean, plc_check, downloads) synchronise it.
 * A context is not safe for concurrent use by several host threads.
 */
#ifndef PLC_H
#define PLC_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define PLC_OK 0
#define PLC_ERR_ARG (-1)        /* bad argument or unsupported configuration */
#define PLC_ERR_SIZE (-2)       /* grid size unsupported (odd, or FFT length not 2^a*3^b) */
#define PLC_ERR_DECOMP (-3)     /* p_row*p_col != 1 */
#define PLC_ERR_CUDA (-4)       /* CUDA runtime error */
#define PLC_ERR_CHECK (-5)      /* NaN / CFL / divergence check failed */
#define PLC_ERR_IO (-6)         /* file could not be read or parsed */
#define PLC_ERR_NOMEM (-7)      /* device allocation failed */
#define PLC_ERR_STATE (-8)      /* call not valid in the context's state */

/* ---- field identifiers (mod_variables.hh:7-9) ---- */
#define PLC_U 0
#define PLC_V 1
#define PLC_W 2
#define PLC_U1 3
#define PLC_V1 4
#define PLC_W1 5
#define PLC_P 6
#define PLC_SPEC 7 /* nx*ny*nz spectral work array (var_xpen) */

/* ---- precision forms ---- */
#define PLC_FP64 0  /* plain FP64, parity with the reference */
/* No counterpart in the reference.  FP32 fields, FP32 stencils and FFTs; FP64
 * time step, forcing sum, NaN/CFL/divergence checks and tridiagonal sweep
 * (with FP64 intermediates for the lowest wavenumbers and the singular (0,0)
 * mode pinned).  nx and ny must be divisible by 4.  A mixed context runs
 * through plc_step / plc_step_timed / plc_profile_step, plc_init_flow,
 * plc_check, plc_upload / plc_download (FP64 host arrays in the reference
 * layout, converted on the device) and plc_field_ptr_f32; the FP64 module
 * entry points return PLC_ERR_STATE.  Its divergence check uses
 * div_limit * 2^29 (the FP32/FP64 unit round-off ratio). */
#define PLC_MIXED 1

/* ---- initial fields (mod_initFlow.cc:47-102) ---- */
#define PLC_INIT_UNI 0
#define PLC_INIT_POI 1
#define PLC_INIT_LOG 2
#define PLC_INIT_MPI 3

/*
 * Every key of the reference's param.json (src/mod_parameters.hh:15-88,
 * read by src/mod_parameters.cc:48-168), with the reference's defaults.
 */
typedef struct plc_params {
  /* PARA */
  int p_row, p_col;
  /* MESH */
  int read_mesh, mesh_type, stretch_func;
  double stretch_ratio;
  int nx, ny, nz;
  double lx, ly, lz;
  /* TIME */
  int nt_end, nt_check;
  double dt, cfl_limit, div_limit;
  /* RESTART */
  int is_restart;
  char fn_prefix_input_inst[128];
  char fn_prefix_input_stat[128];
  /* PHYSICAL */
  double re, u_ref, l_ref;
  int initial_field; /* PLC_INIT_* */
  double u0;
  int init_with_noise;
  double noise_intensity;
  int smooth_wall_visc;
  double u_crf;
  /* FORCE */
  int is_forced[3];
  double vel_force[3];
  /* STATISTICS */
  int nt_init_stat, sample_interval;
  int stat_which_var[11];
  /* OUTPUT */
  int nt_out_scrn, nt_out_inst, nt_out_stat, nt_out_save;
  int overwrite_save, auto_cleanup, num_retained, nt_out_moni;
  /* MONITOR */
  int out_forcing, out_probe_point;
  int probe_ijk[3];
  int out_skf_z[2];
  int out_region, nt_out_region;
  int region_ijk[6];
  /* B200 build options (not in the reference's param.json) */
  int precision; /* PLC_FP64 (default) or PLC_MIXED */
  double cfl_target; /* > 0: dt = cfl_target / max CFL rate, evaluated every nt_check steps */
  double init_vortex_amp; /* != 0: plc_init_flow adds divergence-free streamwise vortices */
} plc_params;

typedef struct plc_value_index {
  /* mod_utils::value_index_pair_t (src/mod_utils.hh:7-12), global 1-based */
  double value;
  int ig, jg, kg;
} plc_value_index;

typedef struct plc_ctx plc_ctx;

/* ---- configuration: replaces readInputParam (src/mod_parameters.cc:220-260) ---- */
/* Fills the reference defaults (keys missing from param.json keep them). */
int plc_params_default(plc_params *prm);
/* Parses a param.json file; sections missing -> PLC_ERR_IO, like the reference's throw. */
int plc_params_read_json(const char *path, plc_params *prm);
/* checkMeshAndPara (src/mod_parameters.cc:170-211) plus the B200 limits. */
int plc_params_check(const plc_params *prm);

/* ---- context: owns the mesh, fields, Poisson state and CUDA stream ---- */
/* The FFT tile sizes are timed per context at creation (plc_fft_tiles);
 * the environment variables PLC_FFT_TILES (FP64 form) and PLC_FFT_TILES_F32
 * (mixed form), "xf,x,y" line pairs per tile, pin them instead (a profiler
 * distorts the event timings the autotuner compares). */
/* initMesh (src/mod_mesh.cc:13-76) + allocVariables (mod_variables.cc:4-12)
 * + init_poisson_solver (mod_poisson_solver.cc:180-315).  dzf_global (nz+2
 * entries, k = 0..nz+1) may be NULL, in which case the mesh is generated
 * from mesh_type/stretch_func/stretch_ratio (read_mesh = 1 requires it). */
int plc_create(const plc_params *prm, const double *h_dzf_global, int device,
               plc_ctx **out);
int plc_destroy(plc_ctx *ctx);
const char *plc_last_error(const plc_ctx *ctx);
int plc_sync(plc_ctx *ctx);

/* Mesh arrays as the reference holds them (nz+2 entries each, k = 0..nz+1):
 * which = 0 dzf_global, 1 dzf, 2 dzf_inv, 3 dzc, 4 dzc_inv, 5 dzflzi,
 * 6 zc_global. */
int plc_get_mesh(const plc_ctx *ctx, int which, double *h_out);
/* Device pointer and element count of a context-owned array (PLC_U..PLC_SPEC). */
int plc_field_ptr(plc_ctx *ctx, int field, double **d_ptr, size_t *count);
/* The same for a PLC_MIXED context: FP32 arrays; halo'd fields have rows of
 * *pitch elements (nx+2 rounded up to a multiple of 4), the spectral array
 * rows of nx.  No counterpart in the reference. */
int plc_field_ptr_f32(plc_ctx *ctx, int field, float **d_ptr, size_t *count, int *pitch);
/* Line pairs per tile of the forward x (fused with calcRHS), backward x and
 * y transforms, as the autotuner of plc_create chose them by timing every
 * feasible size on the device (the choice changes speed, never results).
 * No counterpart in the reference. */
int plc_fft_tiles(const plc_ctx *ctx, int *lines_xf, int *lines_x, int *lines_y);
/* The plan family of the (backward) x and the y transforms, timed per
 * context with the tiles where a length has more than one (0: radix 16, one
 * 8/4/2, then 3s; 1: for lengths 3 * 2^a with 3 <= a <= 7, two passes
 * ending in a radix-24 butterfly; 2: warp-line kernels, groups of four
 * warps transforming their own lines with no block barrier, for lengths
 * 32, 48, 64, 96, 128, 192, 256, 384, 512, 768; 3, y lines only: two passes
 * held in registers with one shared-memory exchange, for lengths 32, 48,
 * 64, 96, 128, 192, 256, 384 over whole blocks of 32 (FP32) or 16 (FP64)
 * columns).  PLC_FFT_PLANS (FP64) and
 * PLC_FFT_PLANS_F32 (mixed), "x,y" or "x,y,xf", pin them (x for both x
 * transforms unless xf gives the forward one's).  No counterpart in the
 * reference. */
int plc_fft_plans(const plc_ctx *ctx, int *plan_x, int *plan_y);
/* The family of the forward x transform (fused with calcRHS in the step),
 * timed separately from the backward one.  No counterpart in the reference. */
int plc_fft_plan_x_fwd(const plc_ctx *ctx, int *plan);
/* z planes per block of the two RK stages, timed per context at creation
 * among 8, 16, 24 and 32 (at most nz) on both fused stages; PLC_RK_KCHUNK
 * (FP64 form) and PLC_RK_KCHUNK_F32 (mixed form) pin it.  The choice changes speed; results only in the mixed form, whose
 * RK2 sums the bulk mean per block in FP32 (by FP32 rounding).  No
 * counterpart in the reference. */
int plc_rk_kchunk(const plc_ctx *ctx, int *kchunk);
/* Whether the mixed form's second RK stage carries its z-face terms from
 * plane to plane (at 3 resident blocks per SM instead of 4), as the
 * autotuner chose (PLC_RK2_CARRY = 0 or 1 pins it).  Changes the mixed
 * results by FP32 rounding only; always 0 in the FP64 form. */
int plc_rk2_carry(const plc_ctx *ctx, int *carry);
/* Copy a whole halo'd field (or the spectral array) between host and device. */
int plc_upload(plc_ctx *ctx, int field, const double *h_src);
int plc_download(plc_ctx *ctx, int field, double *h_dst);
/* Current time step (device-resident; changes under CFL control). */
int plc_get_dt(plc_ctx *ctx, double *dt);
int plc_set_dt(plc_ctx *ctx, double dt);
/* The bulk forcing of the last step, as the step computed it on the device:
 * mean3 = the plane-weighted mean of each forced velocity component before
 * the forcing (0 for unforced ones; the `Mean` of forceVel,
 * mod_calcVel.cc:280-301), force3 (may be NULL) = vel_force - mean3, the
 * uniform shift the step applied.  A 48-byte device-to-host read: the
 * per-step result a caller can fetch without a reduction. */
int plc_step_forcing(plc_ctx *ctx, double *mean3, double *force3);

/* ---- mod_calcVel (src/mod_calcVel.hh:6-14) ---- */
/* transform2CRF (mod_calcVel.cc:13-25); vel_force is updated in place on the host. */
int plc_transform2crf(plc_ctx *ctx, double vel_crf, double *d_vel, double *vel_force);
/* timeIntVelRK1 (mod_calcVel.cc:27-138): u1 = u + dt*(visc - conv), interior only. */
int plc_time_int_vel_rk1(plc_ctx *ctx, double u_crf, const double *d_u,
                         const double *d_v, const double *d_w, double *d_u1,
                         double *d_v1, double *d_w1);
/* timeIntVelRK2 (mod_calcVel.cc:140-251): u = (u1 + dt*(visc - conv)(u1) + u)/2. */
int plc_time_int_vel_rk2(plc_ctx *ctx, double u_crf, double *d_u, double *d_v,
                         double *d_w, const double *d_u1, const double *d_v1,
                         const double *d_w1);
/* correctVel (mod_calcVel.cc:253-278): u -= dt*grad(p), interior only. */
int plc_correct_vel(plc_ctx *ctx, const double *d_p, double *d_u, double *d_v,
                    double *d_w);
/* forceVel (mod_calcVel.cc:280-320): bulk mean per forced component, then a
 * uniform shift of the interior.  force_out (3 doubles, host, may be NULL)
 * receives vel_force - mean. */
int plc_force_vel(plc_ctx *ctx, double *d_u, double *d_v, double *d_w,
                  double *force_out);

/* ---- mod_calcRHS (src/mod_calcRHS.hh:6-7) ---- */
/* calcRHS (mod_calcRHS.cc:7-33): rhs = div(u)/dt on the interior. */
int plc_calc_rhs(plc_ctx *ctx, const double *d_u, const double *d_v,
                 const double *d_w, double *d_rhs);

/* ---- mod_updateBound (src/mod_updateBound.hh:6-8) ---- */
/* updateBoundVel (mod_updateBound.cc:263-285): periodic x/y halos, no-slip z walls. */
int plc_update_bound_vel(plc_ctx *ctx, double u_crf, double *d_u, double *d_v,
                         double *d_w);
/* imposeBCVel (mod_updateBound.cc:217-261); at p_row = p_col = 1 it is the
 * same as plc_update_bound_vel because the y halo is a self-exchange. */
int plc_impose_bc_vel(plc_ctx *ctx, double *d_u, double *d_v, double *d_w,
                      double u_crf);
/* updateBoundP (mod_updateBound.cc:287-330): periodic x/y, zero gradient in z. */
int plc_update_bound_p(plc_ctx *ctx, double *d_p);

/* ---- mod_poisson_solver (src/mod_poisson_solver.hh:5-10) ---- */
/* init_poisson_solver (mod_poisson_solver.cc:180-315).  Called by plc_create
 * with ("PP","PP","NN"); calling it again rebuilds the solver for a new
 * dzf_global.  Only "PP","PP","NN" is supported, as in the reference. */
int plc_init_poisson_solver(plc_ctx *ctx, const double *h_dzf_global,
                            const char *bctype_x, const char *bctype_y,
                            const char *bctype_z);
/* execute_poisson_solver (mod_poisson_solver.cc:454-510): in place, rhs -> phi. */
int plc_execute_poisson_solver(plc_ctx *ctx, double *d_p);
/* free_poisson_solver (mod_poisson_solver.cc:512-537). */
int plc_free_poisson_solver(plc_ctx *ctx);
/* ssolve_trid (mod_poisson_solver.cc:317-357) on the spectral array. */
int plc_solve_trid(plc_ctx *ctx, double *d_var);

/* ---- mod_fft (src/mod_fft.hh:4-11) ---- */
/* execute_fft_fwd_xpen (mod_fft.cc:60-88): p interior -> packed x spectrum. */
int plc_fft_fwd_xpen(plc_ctx *ctx, const double *d_p, double *d_var);
/* execute_fft_bwd_xpen (mod_fft.cc:90-120): packed x spectrum -> p interior, scaled by 1/(nx*ny). */
int plc_fft_bwd_xpen(plc_ctx *ctx, const double *d_var, double *d_p);
/* execute_fft_fwd_ypen / bwd_ypen (mod_fft.cc:122-187): in place along y. */
int plc_fft_fwd_ypen(plc_ctx *ctx, double *d_var);
int plc_fft_bwd_ypen(plc_ctx *ctx, double *d_var);
/* get_eigen_values (mod_fft.cc:196-222), host only, "PP". */
int plc_get_eigen_values(int ist, int isz, int isz_global, const char *bctype,
                         double *h_lambda);

/* ---- mod_utils (src/mod_utils.hh:14-27) ---- */
/* Mean (mod_utils.cc:30-51): sum(var*dzflzi)/nx_global/ny_global over the interior. */
int plc_mean(plc_ctx *ctx, int nx_global, int ny_global, const double *d_var,
             double *mean);
/* checkNaN (mod_utils.cc:77-106): *passed = 1 if no NaN (halos included). */
int plc_check_nan(plc_ctx *ctx, const double *d_var, int *passed);
/* calcMaxCFL (mod_utils.cc:108-150) and calcMaxDiv (:164-205). */
int plc_calc_max_cfl(plc_ctx *ctx, const double *d_u, const double *d_v,
                     const double *d_w, plc_value_index *cfl_max);
int plc_calc_max_div(plc_ctx *ctx, const double *d_u, const double *d_v,
                     const double *d_w, plc_value_index *div_max);

/* ---- mod_statistics (src/mod_statistics.hh:8-16) on the context's fields ---- */
/* Statistic ids of the running sums: cell-centred u (+ u_crf), v, w and their
 * products, p, p*p; sampled when plc_params.stat_which_var[id] is set. */
#define PLC_STAT_U 0
#define PLC_STAT_V 1
#define PLC_STAT_W 2
#define PLC_STAT_UU 3
#define PLC_STAT_VV 4
#define PLC_STAT_WW 5
#define PLC_STAT_UV 6
#define PLC_STAT_UW 7
#define PLC_STAT_VW 8
#define PLC_STAT_P 9
#define PLC_STAT_PP 10
/* allocStat + initStat (mod_statistics.cc:7-28): zeroed device sums of the
 * enabled statistics; nts = nt_init_stat+1, nte = nt_init_stat, nspl = 0. */
int plc_stat_init(plc_ctx *ctx);
/* freeStat (mod_statistics.cc:15-21). */
int plc_stat_free(plc_ctx *ctx);
/* calcStat (mod_statistics.cc:30-106): when (nt - nt_init_stat) is a multiple
 * of sample_interval, adds one sample of the context's u, v, w, p to the sums
 * (nte += sample_interval, nspl += 1).  The sums are FP64 in either form. */
int plc_calc_stat(plc_ctx *ctx, int nt);
/* stat_info (mod_statistics.hh:8-12). */
int plc_stat_info(const plc_ctx *ctx, int *nts, int *nte, int *nspl);
/* A running sum (nx*ny*nz doubles, x fastest, no halos) to / from the host;
 * the upload also restores the counters (inputStatData, mod_dataIO.cc:232-252). */
int plc_stat_download(plc_ctx *ctx, int which, double *h_dst);
int plc_stat_upload(plc_ctx *ctx, int which, const double *h_src, int nts, int nte, int nspl);
/* Plane averages of every statistic divided by the samples: h_prof[id*nz + k-1]
 * (0 for statistics not sampled), the mean and second-moment profiles from
 * which RMS profiles follow.  No counterpart in the reference (its profiles
 * are post-processed from the stat files). */
int plc_stat_profiles(plc_ctx *ctx, double *h_prof);

/* Instantaneous plane means of u + u_crf, h_prof[k-1] for k = 1..nz (no
 * counterpart in the reference; the spin-up judge of the learned
 * initialiser). */
int plc_mean_profile(plc_ctx *ctx, double *h_prof);

/* ---- mod_monitor (src/mod_monitor.cc:57-205) on the context's fields ---- */
/* calcAndWriteForcing (:57-75): Mean of each forced component (u + u_crf), 0 else. */
int plc_monitor_forcing(plc_ctx *ctx, double *vel_mean3);
/* extractAndWriteProbePoint (:77-91): u + u_crf, v, w, p at the 1-based point. */
int plc_monitor_probe(plc_ctx *ctx, int ig, int jg, int kg, double *out4);
/* calcAndWriteSkf (:93-113) at the bottom (wall 0, k = 1) or top (wall 1,
 * k = nz) wall: tau_w = mean of re_inv*(u + u_crf)/(dzf/2) over the plane
 * (double-double sum), u_tau = sqrt(tau_w), cf = tau_w/(u_ref^2/2).  With
 * l_ref = 1 (the half height) Re_tau = u_tau / re_inv. */
int plc_monitor_skf(plc_ctx *ctx, int wall, double *u_tau, double *cf);
/* extractRegion (:117-158, :160-205): the box region_ijk = {i0,i1,j0,j1,k0,k1}
 * (1-based, inclusive, clipped to the domain as initMonitor does) of u, v, w
 * (centred along their own direction, u + u_crf) or p, into h_dst (x fastest). */
int plc_extract_region(plc_ctx *ctx, const int *region_ijk, int field, double *h_dst);

/* The solver's projection of the context's u, v, w onto divergence-free
 * fields: p = div(u)/dt (calcRHS), the Poisson solve, correctVel and the
 * boundary updates, without time integration.  Either form. */
int plc_project(plc_ctx *ctx);

/* ---- initial field (mod_initFlow.cc:47-102) on the context's u, v, w ---- */
/* Followed by transform2CRF and the boundary update, as main.cc:73-82.
 * With init_vortex_amp = A != 0 (no counterpart in the reference, whose
 * laminar + noise field relaminarises on fine grids) the profile and noise
 * are followed by streamwise vortices: v, w from the streamfunction
 * psi = A sin(2 pi n_y y / ly) (1 - zeta^2)^2 (zeta = 2 z / lz - 1) on the
 * cell edges, times 1 + cos(2 pi n_x x / lx) / 2, with n_y = 3 pairs per 2 pi
 * of span and n_x = 2 per 4 pi of length; discretely divergence-free. */
int plc_init_flow(plc_ctx *ctx);
/* main.cc:77-82 for fields uploaded by the caller (inputData on restart):
 * u -= u_crf on the interior with vel_force[0] shifted likewise
 * (transform2CRF, mod_calcVel.cc:13-25), then the velocity and pressure
 * boundary update.  Either form. */
int plc_finish_input(plc_ctx *ctx);

/* ---- fused time step: main.cc:116-154 on the context's fields ---- */
/* Runs nsteps steps of the plain sequence RK1, RK2, RHS, Poisson, correction,
 * forcing and boundary updates with fused kernels replayed from one captured
 * CUDA graph.  Every nt_check steps (counted from the context's step counter)
 * the NaN/CFL/divergence checks of main.cc:156-178 run on the device; a
 * failure returns PLC_ERR_CHECK with the values in plc_last_error and in
 * plc_last_check. */
int plc_step(plc_ctx *ctx, int nsteps);
/* Values of the last NaN/CFL/divergence check run by plc_step or plc_check. */
int plc_last_check(plc_ctx *ctx, int *nan_passed, plc_value_index *cfl_max,
                   plc_value_index *div_max);
/* The checks of main.cc:156-178 on the context's u, v, w right now. */
int plc_check(plc_ctx *ctx, int *nan_passed, plc_value_index *cfl_max,
              plc_value_index *div_max);
/* Number of steps taken by plc_step so far. */
int plc_step_count(plc_ctx *ctx, long long *count);
/* Sets the step counter (the nt of the last completed step), so that the
 * checks of a restarted run fall on the multiples of nt_check of nt. */
int plc_set_step_count(plc_ctx *ctx, long long count);
/* Number of kernel launches one plc_step step issues (graph nodes). */
int plc_kernels_per_step(plc_ctx *ctx, int *count);
/* plc_step(ctx, nsteps) bracketed by CUDA events on the context's stream;
 * *ms receives the device time between the events (checks included). */
int plc_step_timed(plc_ctx *ctx, int nsteps, double *ms);
/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work or timing events after the library's. */
int plc_get_stream(plc_ctx *ctx, void **stream);
/* Runs nsteps plain steps launching the kernels of the fused step one by one
 * with CUDA events between them and adds each kernel's device time (ms) to
 * ms_per_kernel[0..count-1]; *count receives the number of kernels per step
 * (at most 16).  Used for per-kernel roofline figures; advances the state. */
int plc_profile_step(plc_ctx *ctx, int nsteps, float *ms_per_kernel, int *count);
/* Name of kernel i of the fused step of the FP64 form (static string). */
const char *plc_step_kernel_name(int i);
/* Name of kernel i of the context's fused step (either form). */
const char *plc_step_kernel_name_ctx(const plc_ctx *ctx, int i);

/* ---- host-only helpers (no GPU needed) ---- */
/* initMeshByFunc (src/mod_mesh.cc:95-125): dzf_global[0..nz+1]. */
int plc_mesh_by_func(int mesh_type, int stretch_func, double stretch_ratio, int nz,
                     double lz, double *h_dzf_global);
/* The Poisson solver's tridiagonal tables (mod_poisson_solver.cc:35-98,
 * 231-282): reciprocal pre-factored pivots 1/b, laid out (nz, ny/2+1,
 * nx/2+1) over the distinct wavenumber pairs, 0 where the last pivot is 0;
 * h_a and h_c receive a[nz] and c[nz]. */
int plc_trid_tables(int nx, int ny, int nz, double lx, double ly,
                    const double *h_dzf_global, double *h_rpiv, double *h_a,
                    double *h_c);
/* ---- data I/O: mod_dataIO (src/mod_dataIO.cc), outputMesh
 * (src/mod_mesh.cc:127-147), mod_monitor files (src/mod_monitor.cc) and the
 * time-marching driver (src/main.cc:114-222) ----
 * HDF5 files are written and read without libhdf5 (superblock 2, compact root
 * group, contiguous little-endian datasets), with the reference's datasets: a
 * field file holds the [nz][ny][nx] f64 dataset "u", "v", "w" or "p" and a
 * 1-element int dataset "nt"; a statistics file holds "<type>_stat" with
 * "nts", "nte", "nspl" (type u v w u2 v2 w2 uv uw vw p p2, PLC_STAT_* order).
 * Readers accept any file of that shape written by HDF5 1.10+ with the
 * latest-format property (superblock 2 or 3, compact groups, contiguous data);
 * others give PLC_ERR_IO. */
/* The HDF5 subset on plain host arrays (no context, no GPU).
 * plc_h5_write: nsets datasets in the root group; types[q] 0 = f64, 1 = i32;
 * dims holds the ndims[q] dimensions of each dataset in turn (slowest first).
 * plc_h5_read: dataset `name` converted to double into out (capacity
 * elements; out may be NULL to query the shape); *ndim in: capacity of dims,
 * out: the rank.  plc_h5_lookup3: the metadata checksum (Jenkins lookup3). */
int plc_h5_write(const char *path, int nsets, const char *const *names, const int *types,
                 const int *ndims, const long long *dims, const void *const *data);
int plc_h5_read(const char *path, const char *name, double *out, size_t capacity,
                long long *dims, int *ndim);
unsigned int plc_h5_lookup3(const void *key, size_t length, unsigned int initval);
/* inputMesh (src/mod_mesh.cc:78-93): nz spacings from a mesh.in text file
 * into dzf_global[1..nz], with dzf_global[0] and [nz+1] copied from the
 * neighbours (the dzf_global argument of plc_create when read_mesh = 1). */
int plc_read_mesh_in(const char *path, int nz, double *dzf_global);
/* Name of CUDA device `device` (the "Selected device" line of main.cc). */
int plc_device_name(int device, char *buf, int len);
/* Directory for the files written by plc_output_mesh / plc_output_init /
 * plc_output_data / plc_run (default: the working directory). */
int plc_set_output_dir(plc_ctx *ctx, const char *dir);
/* outputField (mod_dataIO.cc:86-101) of one field (PLC_U..PLC_P) at path.
 * u is written as outputData does (:141-147): u_crf added on the device,
 * downloaded, subtracted again, so the file holds the lab-frame velocity. */
int plc_write_field_h5(plc_ctx *ctx, const char *path, int field, int nt);
/* inputField (mod_dataIO.cc:68-84): the dataset named after the field into
 * the field's interior (halos kept), *nt = the file's "nt".  No frame shift:
 * call plc_finish_input after reading u, v, w. */
int plc_read_field_h5(plc_ctx *ctx, const char *path, int field, int *nt);
/* A statistics file of statistic `which` (outputField / inputField with
 * stat_info); the read restores nts/nte/nspl, *nte receives nte. */
int plc_write_stat_h5(plc_ctx *ctx, const char *path, int which);
int plc_read_stat_h5(plc_ctx *ctx, const char *path, int which, int *nte);
/* outputMesh: mesh_<nx>-<ny>-<nz>.h5 (xc, yc, zc) and mesh_<nz:05>.out. */
int plc_output_mesh(plc_ctx *ctx);
/* Restart (main.cc:59-88): inputData (mod_dataIO.cc:104-128) from
 * <fn_prefix_input_inst>_{u,v,w}.h5 with the timestamp checks, the frame
 * shift and boundary update (plc_finish_input), inputStatData (:232-252)
 * from <fn_prefix_input_stat>_<type>.h5 when nt_in + 1 > nt_init_stat + 1,
 * and the step counter set to nt_in. */
int plc_input_data(plc_ctx *ctx, int *nt_in);
/* initMonitor (mod_monitor.cc:208-310): creates the monitor text files of
 * the enabled monitors with their headers (truncating, as the reference's
 * out|ate open does) and clips region_ijk to the domain. */
int plc_output_init(plc_ctx *ctx);
/* outputData (mod_dataIO.cc:130-230) after step nt: monitors every
 * nt_out_moni, inst_<nt:08>_{u,v,w,p}.h5 every nt_out_inst, checkpoints
 * save_{u,v,w}.h5 (save_<nt:08>_... unless overwrite_save) every nt_out_save,
 * statistics files, automatic cleanup.  A period of 0 disables its output. */
int plc_output_data(plc_ctx *ctx, int nt);
/* freeMonitor: closes the monitor files. */
int plc_output_free(plc_ctx *ctx);
/* The main loop of main.cc:114-222 for nt = nt_start..nt_end: steps (graph
 * replays between the steps that need host work), checks every nt_check,
 * statistics started at nt_init_stat + 1, the screen line every nt_out_scrn
 * (verbose != 0) and plc_output_data. */
int plc_run(plc_ctx *ctx, int nt_start, int verbose);

/* ---- SM budget of a context ----
 * The persistent kernels of the step size their grids to the context's SM
 * budget (default: all SMs of the device).  A smaller budget lets several
 * contexts' steps run side by side; results do not depend on it.  Rebuilds
 * the captured step. */
int plc_set_sm_budget(plc_ctx *ctx, int sms);
int plc_get_sm_budget(const plc_ctx *ctx, int *sms);

/* ---- batched ensembles of independent channels (no reference counterpart) ----
 * n member contexts with their own parameters (any grid, Re, dt, precision)
 * on one device; one ensemble step is one CUDA graph launch whose branches
 * are the members' fused steps, or (PLC_ENS_BATCHED) whose nodes are the
 * step's stages, each one launch over a work list of (member, tile) items.  Checks, CFL-controlled dt and error words
 * stay per member (as plc_step); plc_ensemble_member gives a member's context
 * for every other entry point (upload, download, statistics, I/O). */
typedef struct plc_ensemble plc_ensemble;
#define PLC_ENS_CONCURRENT 0   /* all members at once, full SM budgets */
#define PLC_ENS_PROPORTIONAL 1 /* all at once, SMs shared in proportion to cost */
#define PLC_ENS_TWO_GROUPS 2   /* two cost-balanced groups one after the other */
#define PLC_ENS_SEQUENTIAL 3   /* one member after another */
#define PLC_ENS_BATCHED 4      /* each stage of the mixed-form members' step as one launch
                                  over all of them (per line length for the transforms);
                                  FP64 members as concurrent branches */
#define PLC_ENS_NUM_SCHEDULES 5
/* dzf_globals: NULL, or n pointers (each NULL or nz+2 spacings, as plc_create). */
int plc_ensemble_create(int n, const plc_params *prms, const double *const *dzf_globals,
                        int device, plc_ensemble **out);
int plc_ensemble_destroy(plc_ensemble *ens);
const char *plc_ensemble_last_error(const plc_ensemble *ens);
int plc_ensemble_size(const plc_ensemble *ens, int *n);
int plc_ensemble_member(plc_ensemble *ens, int i, plc_ctx **ctx);
/* plc_init_flow on every member. */
int plc_ensemble_init_flow(plc_ensemble *ens);
/* nsteps ensemble steps; every member advances nsteps steps. */
int plc_ensemble_step(plc_ensemble *ens, int nsteps);
/* The same bracketed by CUDA events on the ensemble's stream: *ms = device time. */
int plc_ensemble_step_timed(plc_ensemble *ens, int nsteps, double *ms);
/* A schedule PLC_ENS_*: member groups and SM budgets from the cost model
 * (grid points until plc_ensemble_autotune has measured each member). */
int plc_ensemble_set_schedule(plc_ensemble *ens, int scheme);
/* The schedule in use; groups and sm_budgets (n entries each) may be NULL. */
int plc_ensemble_schedule(const plc_ensemble *ens, int *scheme, int *groups, int *sm_budgets);
/* Autotuner: times each member alone (the cost model), the plan families,
 * tiles and RK z chunk of the batched schedule's launches (per line-length
 * group, on the mixed-form members), then every schedule over `steps`
 * ensemble steps, keeps the fastest and restores the members' u, v, w, p
 * (step counters and dt are untouched).  ms_per_scheme
 * (PLC_ENS_NUM_SCHEDULES entries, -1 = not applicable) may be NULL. */
int plc_ensemble_autotune(plc_ensemble *ens, int steps, float *ms_per_scheme);
/* The batched schedule's tuned choices: the chains of mixed-form members
 * stepped concurrently (1 or 2, cost-balanced), the RK stages' z planes per
 * block (0: each member's own), the resident blocks per SM of their
 * kernels, and the line-length groups tuned for the forward x, backward x
 * and y transforms (3 entries; any pointer may be NULL). */
int plc_ensemble_batch_choice(const plc_ensemble *ens, int *chains, int *rk_kchunk,
                              int *rk_blocks_per_sm, int *fft_groups);
/* Sets the batched schedule's chains (1 or 2) instead of the autotuner. */
int plc_ensemble_set_batch_chains(plc_ensemble *ens, int chains);
/* Programmatic dependent launch in the batched schedule: on != 0 launches
 * each batched kernel with programmatic stream serialisation, so that its
 * blocks become resident while the stage before it drains (they wait for
 * its completion before reading anything).  The autotuner times both and
 * keeps the faster unless PLC_ENS_PDL=0|1 pins it.  Results are the same
 * either way.  *on may be read with plc_ensemble_batch_pdl. */
int plc_ensemble_set_batch_pdl(plc_ensemble *ens, int on);
int plc_ensemble_batch_pdl(const plc_ensemble *ens, int *on);
/* Multi-GPU placement of members: longest-processing-time-first over the
 * given costs; gpu_of[i] in [0, n_gpus).  Host only. */
int plc_ensemble_partition(int n, const double *cost, int n_gpus, int *gpu_of);

/* ---- learned initialiser (no reference counterpart) ----
 * A conditional 3-D convolutional generator: Gaussian latent + Re_tau ->
 * u, v, w at the cell centres of an nx x ny x nz grid (4 levels, each
 * doubling the grid: nx, ny, nz divisible by 8), 3x3x3 convolutions periodic
 * in x, y and zero-padded at the walls, FiLM conditioning on Re_tau per
 * wall-normal plane, BF16 weights and activations with FP32 accumulation on
 * the tensor cores, FP32 master weights and Adam.  Trained on statistics of
 * DNS snapshots coarse-grained to its grid (PLC_GEN_NSTAT per plane: means of
 * u, v, w; their variances; the u-w covariance; lagged covariances of u, v, w
 * at 1, 2, 4, 8 cells along x and along y). */
typedef struct plc_gen plc_gen;
typedef struct plc_gen_config {
  int nx, ny, nz;          /* output grid of the generator, divisible by 8 */
  int channels[4];         /* per level, coarse to fine; multiples of 16, <= 128 */
  int latent_channels;     /* multiple of 16 */
  int batch;               /* samples per forward / training step */
  unsigned long long seed; /* initial weights */
} plc_gen_config;
#define PLC_GEN_NSTAT 31
int plc_gen_config_default(plc_gen_config *cfg);
int plc_gen_create(const plc_gen_config *cfg, int device, plc_gen **out);
int plc_gen_destroy(plc_gen *gen);
const char *plc_gen_last_error(const plc_gen *gen);
int plc_gen_num_params(const plc_gen *gen, long long *n);
/* FP32 master parameters: the conv weights W[tap][co][ci] of every layer,
 * then per layer the FiLM tables A0, A1, B0, B1 [z][co]. */
int plc_gen_get_params(plc_gen *gen, float *h);
int plc_gen_set_params(plc_gen *gen, const float *h);
/* Training targets: n entries of (Re_tau, nz x PLC_GEN_NSTAT statistics). */
int plc_gen_set_targets(plc_gen *gen, int n, const double *re_tau, const double *stats);
/* The Gaussian latent of a seed ([batch][nz/8][ny/8][nx/8][latent] floats). */
int plc_gen_latent(plc_gen *gen, unsigned long long seed, float *h);
/* Forward pass for batch Re_tau values; h_out (batch*nz*ny*nx*3, u v w
 * fastest) may be NULL.  plc_gen_output_stats: the statistics of the last
 * output (batch*nz*PLC_GEN_NSTAT). */
int plc_gen_forward(plc_gen *gen, const double *re_tau, unsigned long long latent_seed,
                    float *h_out);
int plc_gen_output_stats(plc_gen *gen, double *h_stats);
/* Loss of one batch against targets target_idx (with their Re_tau) and, if
 * h_grads != NULL, the gradient of every parameter. */
int plc_gen_loss_grad(plc_gen *gen, const int *target_idx, const double *re_tau,
                      unsigned long long latent_seed, double *loss, float *h_grads);
/* One Adam step (lr) on the gradients of the last plc_gen_loss_grad. */
int plc_gen_adam_step(plc_gen *gen, double lr);
/* iters Adam steps (warm-up, cosine decay from lr) on random batches of the
 * targets; h_loss (iters) may be NULL. */
int plc_gen_train(plc_gen *gen, int iters, double lr, unsigned long long seed, double *h_loss);
/* Statistics (nz x PLC_GEN_NSTAT) of a context's u + u_crf, v, w box-averaged
 * to the generator's grid (the context's grid a multiple of it). */
int plc_gen_stats_of(plc_gen *gen, plc_ctx *ctx, double *h_stats);
/* Proposes u, v, w for Re_tau into the context (its nz a multiple of the
 * generator's; interpolated onto the staggered grid, zero at the walls) and
 * projects them with plc_project. */
int plc_gen_propose(plc_gen *gen, plc_ctx *ctx, double re_tau, unsigned long long latent_seed);

/* Pinned host memory for fast uploads/downloads. */
int plc_host_alloc(size_t bytes, void **ptr);
int plc_host_free(void *ptr);

/* ---- allocation-free entry point ---- */
/* No counterpart in the reference.  The bulk mean of plc_mean
 * (sum(var*dzflzi)/nx_global/ny_global over the interior) for callers that
 * cannot allocate device memory -- for example a host application that keeps
 * all GPU memory in its own pool and forbids allocation after start-up, or a
 * time loop that must not take the implicit device synchronisation of
 * cudaMalloc/cudaFree -- and that therefore have no plc context.  The caller
 * passes the halo'd field d_var (nx, ny, nz interior), d_dzflzi (nz+2
 * entries) and d_mean (one double), all device memory, and a cudaStream_t
 * (NULL = default stream); the result is written to d_mean on that stream.
 * Nothing is allocated: the partial sums live in a static 128 KiB array of
 * the library (8192 double-double block sums, at least one per z plane),
 * held by every GPU that loads the library until exit, so nz is limited to
 * 8192 (PLC_ERR_SIZE beyond).  All calls share that array: calls that
 * overlap on the GPU race.  A call outside stream capture looks up the
 * array's address in the current CUDA context and remembers it; a call
 * during capture uses the remembered address, so make one call outside
 * capture first in each context (again after cudaDeviceReset).
 * Errors: plc_last_error(NULL). */
int plc_mean_noalloc(const double *d_var, const double *d_dzflzi, int nx, int ny,
                     int nz, int nx_global, int ny_global, double *d_mean,
                     void *stream);

#ifdef __cplusplus
}
#endif
#endif /* PLC_H */
