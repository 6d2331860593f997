/*
 * CPU oracle for the PowerLLEL_Channel DNS time step -- TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain FP64 C++ restatement of the reference's hot path
 * (xiejb6/PowerLLEL_Channel_SYCL, src/mod_calcVel.cc, mod_calcRHS.cc,
 * mod_updateBound.cc, mod_fft.cc, mod_poisson_solver.cc, mod_mesh.cc,
 * mod_utils.cc, mod_initFlow.cc, main.cc).  Every function cites the
 * reference lines it follows.  It is used by the tests, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker;
 * the product library never links or calls it.
 *
 * PARITY STATUS: pinned to the reference's own code, except for the DFT.
 * The reference ships no tests, golden vectors or fixtures, and its build
 * needs a SYCL compiler, oneMKL, oneDPL, MPI and HDF5, none of which is
 * here.  Its time-step modules are instead compiled unmodified from its
 * sources against host stand-ins for those libraries (oracle/reference_cpu,
 * output oracle/_ref), and tests/test_reference_pin.py checks every
 * function below against the reference's own: mesh, boundary updates, RK1,
 * RK2, calcRHS, correctVel, transform2CRF, CFL/divergence maxima, the
 * Thomas sweep and the initial v, w bit-identical; the bulk mean within the
 * error bound of a sum in any order; the transforms to 1e-14 and ten full
 * steps to 1e-12.  The one stage whose arithmetic is not the reference's
 * own is oneMKL's DFT (closed source, absent): both the stand-in and this
 * oracle compute the documented transform, checked against numpy.fft.  The
 * noise generator of the initial field follows the C++ standard's minstd
 * engine; oneDPL's exact stream is not available to compare.  Independent
 * checks remain as well: numpy/scipy golden values and manufactured-solution
 * / divergence / bulk-flux invariants (tests/test_oracle_*.py).
 *
 * Array layout (same as the reference's _Array3D with one halo cell on each
 * side, src/mod_type.hh:81-306): a field of interior size nx*ny*nz is stored
 * as (nx+2)*(ny+2)*(nz+2) doubles, x fastest; the reference's 1-based index
 * (i,j,k), 0 <= i <= nx+1, maps to  i + (nx+2)*(j + (ny+2)*k).
 * 1-D mesh arrays (dzf, dzf_inv, dzc_inv, dzflzi, dzf_global) hold nz+2
 * entries indexed k = 0..nz+1 (Array1DH1, src/mod_type.hh:16-67).
 * The spectral work array of the Poisson solver holds nx*ny*nz doubles with
 * no halos, x fastest (var_xpen, src/mod_poisson_solver.cc:196-198).
 */
#ifndef PLC_ORACLE_H
#define PLC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_grid {
  int nx, ny, nz;
  double lx, ly, lz;
  double dx, dy, dx_inv, dy_inv;
  double dt, re_inv, u_crf;
  int is_forced[3];
  double vel_force[3];
  /* 1-D mesh arrays, nz+2 entries each (k = 0..nz+1); owned by the caller */
  const double *dzf, *dzf_inv, *dzc_inv, *dzflzi;
} orc_grid;

typedef struct orc_value_index {
  double value;
  int ig, jg, kg;
} orc_value_index;

/* ---- mesh (src/mod_mesh.cc:13-125) ---- */
/* Fills dzf_global (nz+2) from the stretching function. */
void orc_mesh_by_func(int mesh_type, int stretch_func, double stretch_ratio,
                      int nz, double lz, double *dzf_global);
/* Derived arrays from dzf_global; every output has nz+2 entries. */
void orc_mesh_derived(int nz, double lz, const double *dzf_global,
                      double *dzf, double *dzf_inv, double *dzc,
                      double *dzc_inv, double *dzflzi, double *zc_global);

/* ---- velocity update (src/mod_calcVel.cc) ---- */
void orc_transform2crf(const orc_grid *g, double vel_crf, double *vel,
                       double *vel_force);
void orc_time_int_vel_rk1(const orc_grid *g, double u_crf, const double *u,
                          const double *v, const double *w, double *u1,
                          double *v1, double *w1);
void orc_time_int_vel_rk2(const orc_grid *g, double u_crf, double *u,
                          double *v, double *w, const double *u1,
                          const double *v1, const double *w1);
void orc_correct_vel(const orc_grid *g, const double *p, double *u, double *v,
                     double *w);
/* Writes the three forcing values (vel_force - mean) to force_out if not NULL. */
void orc_force_vel(const orc_grid *g, double *u, double *v, double *w,
                   double *force_out);

/* ---- RHS (src/mod_calcRHS.cc) ---- */
void orc_calc_rhs(const orc_grid *g, const double *u, const double *v,
                  const double *w, double *rhs);

/* ---- boundary update (src/mod_updateBound.cc) ---- */
void orc_update_bound_vel(const orc_grid *g, double u_crf, double *u,
                          double *v, double *w);
void orc_update_bound_p(const orc_grid *g, double *p);

/* ---- utilities (src/mod_utils.cc) ---- */
double orc_mean(const orc_grid *g, int nx_global, int ny_global,
                const double *var);
int orc_check_nan(const orc_grid *g, const double *var);
void orc_calc_max_cfl(const orc_grid *g, const double *u, const double *v,
                      const double *w, orc_value_index *out);
void orc_calc_max_div(const orc_grid *g, const double *u, const double *v,
                      const double *w, orc_value_index *out);

/* ---- FFT (src/mod_fft.cc) ---- */
/* Packed real forward DFT of one line (unscaled), out[0]=Re X0,
 * out[1]=Re X_{n/2}, out[2m]=Re X_m, out[2m+1]=Im X_m. */
void orc_rfft_packed(int n, const double *in, double *out);
/* Unscaled inverse of orc_rfft_packed (result is n times the input). */
void orc_irfft_packed(int n, const double *in, double *out);
void orc_get_eigen_values(int ist, int isz, int isz_global, double *lambda);

/* ---- Poisson solver (src/mod_poisson_solver.cc) ---- */
typedef struct orc_poisson orc_poisson;
orc_poisson *orc_poisson_init(int nx, int ny, int nz, double dx, double dy,
                              const double *dzf_global);
void orc_poisson_free(orc_poisson *ps);
double *orc_poisson_work(orc_poisson *ps); /* the nx*ny*nz spectral array */
const double *orc_poisson_b(const orc_poisson *ps); /* pre-factored 3-D b */
const double *orc_poisson_a(const orc_poisson *ps); /* nz */
const double *orc_poisson_c(const orc_poisson *ps); /* nz */
void orc_fft_fwd_xpen(orc_poisson *ps, const double *p, double *var);
void orc_fft_bwd_xpen(orc_poisson *ps, const double *var, double *p);
void orc_fft_fwd_ypen(orc_poisson *ps, double *var);
void orc_fft_bwd_ypen(orc_poisson *ps, double *var);
void orc_ssolve_trid(orc_poisson *ps, double *var);
void orc_poisson_execute(orc_poisson *ps, double *p);

/* ---- initial field (src/mod_initFlow.cc) ---- */
/* Project noise generator: minstd (multiplier 48271, modulus 2^31-1) seeded
 * with `seed`, jumped ahead by the cell's linear index, mapped to [0,1). */
double orc_noise_uniform(int seed, long long offset);
/* initial_field: 0 = "uni", 1 = "poi", 2 = "log". */
void orc_init_flow(const orc_grid *g, int initial_field, double u0,
                   double u_ref, double re, int init_with_noise,
                   double noise_intensity, const double *zc_global,
                   double *u, double *v, double *w);

/* ---- one full time step sequence (src/main.cc:116-154) ---- */
void orc_step(const orc_grid *g, orc_poisson *ps, int nsteps, double *u,
              double *v, double *w, double *u1, double *v1, double *w1,
              double *p);
/* nsteps of the main loop with a CFL-controlled dt (cfl_target > 0): dt =
 * cfl_target / (calcMaxCFL's value / dt) before step 1, after steps 1, 2, 4,
 * ... below nt_check and after every nt_check-th step.  dt_used (nsteps+1
 * entries, or NULL) receives the dt of each step and, last, the dt the next
 * step would use.  With cfl_target <= 0 dt stays g->dt. */
void orc_run_cfl(const orc_grid *g, orc_poisson *ps, int nsteps, int nt_check,
                 double cfl_target, double *u, double *v, double *w, double *u1,
                 double *v1, double *w1, double *p, double *dt_used);

/* ---- mod_statistics (src/mod_statistics.cc:30-106) ---- */
/* One sample of calcStat: adds to the enabled running sums (sums[q] != NULL,
 * nx*ny*nz doubles, x fastest, no halos): q = 0 u, 1 v, 2 w (cell-centred,
 * u + u_crf), 3 u*u, 4 v*v, 5 w*w, 6 u*v, 7 u*w, 8 v*w, 9 p, 10 p*p. */
void orc_calc_stat_sample(const orc_grid *g, double u_crf, const double *u, const double *v,
                          const double *w, const double *p, double *const *sums);

/* ---- mod_monitor (src/mod_monitor.cc:93-113, 117-158) ---- */
/* calcAndWriteSkf's plane mean: sum over (i,j) of re_inv*(vel(i,j,k_wall)+vel_crf)/dz,
 * divided by nx and ny (the sum in double-double, i.e. order independent). */
double orc_wall_tau(const orc_grid *g, int k_wall, double dz, const double *vel,
                    double vel_crf);
/* extractRegion: the box of size reg_sz starting at the 1-based interior
 * index reg_st, staggered -> centred along offset_dir (0 none, 1 x, 2 y,
 * 3 z); out is reg_sz[0]*reg_sz[1]*reg_sz[2], x fastest. */
void orc_extract_region(const orc_grid *g, const double *var, int offset_dir,
                        const int *reg_st, const int *reg_sz, double *out);

void orc_set_threads(int n);
int orc_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
