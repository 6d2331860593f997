// TEST INFRASTRUCTURE ONLY.
//
// A C interface to the reference's own time-step modules, compiled
// unmodified from the reference's sources (src/mod_calcVel.cc,
// mod_calcRHS.cc, mod_updateBound.cc, mod_utils.cc, mod_fft.cc,
// mod_poisson_solver.cc, mod_mesh.cc, mod_initFlow.cc, mod_mpi.cc,
// mod_variables.cc, decomp_2d.cc) against the host stand-ins under shim/
// (SYCL, one-rank MPI, the oneMKL DFT, oneDPL's minstd engine, {fmt}).  It
// drives them the way the reference's main program does (src/main.cc) on
// one rank, so that tests can check the project's CPU oracle -- and through
// it the CUDA library -- against the reference's own code.  Nothing in the
// product library uses it.
//
// Fields cross the interface in the reference's halo'd layout:
// (nx+2)*(ny+2)*(nz+2) doubles, x fastest.  Field numbers: 0 u, 1 v, 2 w,
// 3 u1, 4 v1, 5 w1, 6 p.

#include <array>
#include <cstring>
#include <string>
#include <string_view>

#include "decomp_2d.hh"
#include "mod_calcRHS.hh"
#include "mod_calcVel.hh"
#include "mod_fft.hh"
#include "mod_hdf5.hh"
#include "mod_initFlow.hh"
#include "mod_mesh.hh"
#include "mod_mpi.hh"
#include "mod_parameters.hh"
#include "mod_poisson_solver.hh"
#include "mod_type.hh"
#include "mod_updateBound.hh"
#include "mod_utils.hh"
#include "mod_variables.hh"

// the tridiagonal sweep of mod_poisson_solver.cc (external linkage there)
void ssolve_trid(int *sz, double *var);

// mod_mesh::outputMesh writes an HDF5 mesh file through mod_hdf5; the
// harness runs the modules for their arithmetic only, so these do nothing.
namespace mod_hdf5 {
hid_t createFile(std::string_view) { return 0; }
void closeFile(hid_t) {}
void write1d(hid_t, std::string_view, const Array1DH1 &) {}
}  // namespace mod_hdf5

namespace {

bool g_ready = false;
mod_utils::value_index_pair_t g_cfl, g_div;

Array3DH3 &field(int which) {
  using namespace mod_variables;
  switch (which) {
    case 0: return u;
    case 1: return v;
    case 2: return w;
    case 3: return u1;
    case 4: return v1;
    case 5: return w1;
    default: return p;
  }
}

size_t field_len() { return (size_t)(nx + 2) * (ny + 2) * (nz + 2); }

}  // namespace

extern "C" {

void ref_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
}

// readInputParam's values for one case (mod_parameters.cc:48-168, 259),
// then main.cc:36-61: initMPI, allocVariables, initMesh, init_poisson_solver,
// and initCheckCFLAndDiv (main.cc:90-92).
void ref_init(int nx_, int ny_, int nz_, double lx_, double ly_, double lz_, int mesh_type_,
              int stretch_func_, double stretch_ratio_, double re_, double u_ref_,
              double l_ref_, double dt_, double u_crf_, const int *is_forced_,
              const double *vel_force_) {
  p_row = p_col = 1;
  read_mesh = false;
  mesh_type = mesh_type_;
  stretch_func = stretch_func_;
  stretch_ratio = stretch_ratio_;
  nx = nx_;
  ny = ny_;
  nz = nz_;
  lx = lx_;
  ly = ly_;
  lz = lz_;
  dt = dt_;
  re = re_;
  u_ref = u_ref_;
  l_ref = l_ref_;
  re_inv = u_ref * l_ref / re;  // mod_parameters.cc:259
  smooth_wall_visc = false;
  u_crf = u_crf_;
  for (int d = 0; d < 3; ++d) {
    is_forced[d] = is_forced_[d] != 0;
    vel_force[d] = vel_force_[d];
  }
  mod_mpi::initMPI();
  mod_variables::allocVariables(mod_mpi::sz);
  mod_mesh::initMesh();
  init_poisson_solver(nx, ny, nz, mod_mesh::dx, mod_mesh::dy, mod_mesh::dzf_global.data(),
                      (char *)"PP", (char *)"PP", (char *)"NN", mod_mpi::neighbor_xyz);
  mod_utils::initCheckCFLAndDiv(g_cfl, g_div);
  g_ready = true;
}

// main.cc:224-236, except for decomp_2d's own finalisation:
// decomp_info_finalize (decomp_2d.cc:209-236) frees its two work buffers
// without clearing their pointers, so the next decomp_2d_init in the same
// process would free them again (the reference finalises once, at exit).
// The harness releases what freeMPI (mod_mpi.cc:111-118) releases apart
// from that -- the communicators and the halo types -- and keeps the
// decomposition tables, which the next initialisation replaces.
void ref_free() {
  if (!g_ready) return;
  mod_utils::freeCheckCFLAndDiv();
  free_poisson_solver();
  mod_mesh::freeMesh();
  mod_variables::freeVariables();
  MPI_Comm_free(&decomp_2d_comm_cart_x);
  MPI_Comm_free(&decomp_2d_comm_cart_y);
  MPI_Comm_free(&decomp_2d_comm_cart_z);
  MPI_Comm_free(&decomp_2d_comm_row);
  MPI_Comm_free(&decomp_2d_comm_col);
  for (int i = 0; i < 6; ++i) {
    MPI_Type_free(&mod_mpi::halotype_vel[i]);
    MPI_Type_free(&mod_mpi::halotype_one[i]);
  }
  g_ready = false;
}

void ref_set_dt(double dt_) { dt = dt_; }

void ref_set_field(int which, const double *src) {
  std::memcpy(field(which).data(), src, field_len() * sizeof(double));
}

void ref_get_field(int which, double *dst) {
  std::memcpy(dst, field(which).data(), field_len() * sizeof(double));
}

// 1-D mesh arrays, nz+2 entries (k = 0 .. nz+1): 0 dzf_global, 1 dzf,
// 2 dzf_inv, 3 dzc, 4 dzc_inv, 5 dzflzi, 6 zc_global, 7 visc_dzf_inv;
// dxy receives dx, dy, dx_inv, dy_inv.
void ref_get_mesh(int which, double *out, double *dxy) {
  using namespace mod_mesh;
  const Array1DH1 *a[8] = {&dzf_global, &dzf, &dzf_inv, &dzc, &dzc_inv, &dzflzi, &zc_global,
                           &visc_dzf_inv};
  for (int k = 0; k <= nz + 1; ++k) out[k] = (*a[which])(k);
  if (dxy) {
    dxy[0] = dx;
    dxy[1] = dy;
    dxy[2] = dx_inv;
    dxy[3] = dy_inv;
  }
}

// ---- module functions on the module's own fields ----
void ref_time_int_vel_rk1() {
  using namespace mod_variables;
  mod_calcVel::timeIntVelRK1(u_crf, u, v, w, u1, v1, w1);
}
void ref_time_int_vel_rk2() {
  using namespace mod_variables;
  mod_calcVel::timeIntVelRK2(u_crf, u, v, w, u1, v1, w1);
}
// set 0: u, v, w; set 1: u1, v1, w1
void ref_update_bound_vel(int set) {
  using namespace mod_variables;
  if (set == 1)
    mod_updateBound::updateBoundVel(u_crf, u1, v1, w1);
  else
    mod_updateBound::updateBoundVel(u_crf, u, v, w);
}
void ref_update_bound_p() { mod_updateBound::updateBoundP(mod_variables::p); }
void ref_calc_rhs() {
  using namespace mod_variables;
  mod_calcRHS::calcRHS(u, v, w, p);
}
void ref_poisson() { execute_poisson_solver(mod_variables::p); }
void ref_correct_vel() {
  using namespace mod_variables;
  mod_calcVel::correctVel(p, u, v, w);
}
void ref_force_vel() {
  using namespace mod_variables;
  mod_calcVel::forceVel(u, v, w);
}
// transform2CRF on field `which` with vel_force[0]-like scalar in/out
void ref_transform2crf(int which, double vel_crf, double *force) {
  double f = *force;
  mod_calcVel::transform2CRF(vel_crf, field(which), f);
  *force = f;
}
double ref_mean(int which, int nx_global, int ny_global) {
  return mod_utils::Mean(nx_global, ny_global, mod_mesh::dzflzi, field(which));
}
int ref_check_nan(int which) { return mod_utils::checkNaN(field(which), "var") ? 1 : 0; }
void ref_calc_max_cfl(double *value, int *ijk) {
  using namespace mod_variables;
  mod_utils::calcMaxCFL(dt, mod_mesh::dx_inv, mod_mesh::dy_inv, mod_mesh::dzf_inv, u, v, w,
                        g_cfl);
  *value = g_cfl.value;
  ijk[0] = g_cfl.ig;
  ijk[1] = g_cfl.jg;
  ijk[2] = g_cfl.kg;
}
void ref_calc_max_div(double *value, int *ijk) {
  using namespace mod_variables;
  mod_utils::calcMaxDiv(mod_mesh::dx_inv, mod_mesh::dy_inv, mod_mesh::dzf_inv, u, v, w, g_div);
  *value = g_div.value;
  ijk[0] = g_div.ig;
  ijk[1] = g_div.jg;
  ijk[2] = g_div.kg;
}

// ---- the Poisson solver's stages on a caller-owned spectral array ----
void ref_fft_fwd_x(double *var) { execute_fft_fwd_xpen(mod_variables::p, var); }
void ref_fft_bwd_x(const double *var) { execute_fft_bwd_xpen(var, mod_variables::p); }
void ref_fft_fwd_y(double *var) { execute_fft_fwd_ypen(var); }
void ref_fft_bwd_y(double *var) { execute_fft_bwd_ypen(var); }
void ref_ssolve_trid(double *var) { ssolve_trid(decomp_main.zsz.data(), var); }
void ref_eigen_values(int n, double *lambda) {
  get_eigen_values(1, n, n, (char *)"PP", lambda);
}

// main.cc:67-82: initFlow, transform2CRF, the velocity and pressure
// boundary updates.  initial_field: 0 "uni", 1 "poi", 2 "log".
void ref_init_flow(int initial_field_code, double u0_, int with_noise, double noise) {
  static const char *names[3] = {"uni", "poi", "log"};
  initial_field = names[initial_field_code];
  u0 = u0_;
  init_with_noise = with_noise != 0;
  noise_intensity = noise;
  using namespace mod_variables;
  mod_initFlow::initFlow(u, v, w);
  mod_calcVel::transform2CRF(u_crf, u, vel_force[0]);
  mod_updateBound::updateBoundVel(u_crf, u, v, w);
  mod_updateBound::updateBoundP(p);
}

double ref_vel_force(int d) { return vel_force[d]; }

// main.cc:116-154, nsteps times
void ref_step(int nsteps) {
  using namespace mod_variables;
  for (int s = 0; s < nsteps; ++s) {
    mod_calcVel::timeIntVelRK1(u_crf, u, v, w, u1, v1, w1);
    mod_updateBound::updateBoundVel(u_crf, u1, v1, w1);
    mod_calcVel::timeIntVelRK2(u_crf, u, v, w, u1, v1, w1);
    mod_updateBound::updateBoundVel(u_crf, u, v, w);
    mod_calcRHS::calcRHS(u, v, w, p);
    execute_poisson_solver(p);
    mod_updateBound::updateBoundP(p);
    mod_calcVel::correctVel(p, u, v, w);
    mod_calcVel::forceVel(u, v, w);
    mod_updateBound::updateBoundVel(u_crf, u, v, w);
  }
}

}  // extern "C"
