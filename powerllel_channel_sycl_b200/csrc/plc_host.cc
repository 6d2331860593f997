// Host-side set-up of libplc.so: mesh generation, Poisson coefficient tables,
// FFT plans and the param.json reader.  Compiled with -ffp-contract=off so
// that the floating-point steps are evaluated in the order written, which
// follows the reference's host loops term by term (the pivot table must be
// bit-identical to the reference's pre-factored b).

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "plc_internal.h"

namespace plc {

// mod_mesh.cc:95-125 (initMeshByFunc)
void host_mesh_by_func(int mesh_type, int stretch_func, double stretch_ratio,
                       int nz, double lz, double *dzf_global) {
  const double pi = M_PI;
  if (stretch_ratio == 0.0 || mesh_type == 0) {
    for (int k = 0; k <= nz + 1; ++k) dzf_global[k] = lz / nz;
    return;
  }
  std::vector<double> zf(nz + 2, 0.0);
  for (int k = 1; k <= nz; ++k) {
    const double z0 = k / (1.0 * nz);
    if (stretch_func == 0)
      zf[k] = 0.5 * (1.0 + tanh((z0 - 0.5) * stretch_ratio) / tanh(stretch_ratio / 2.0));
    else
      zf[k] = 0.5 * (1.0 + sin((z0 - 0.5) * stretch_ratio * pi) / sin(stretch_ratio * pi / 2.0));
  }
  for (int k = 1; k <= nz; ++k) dzf_global[k] = lz * (zf[k] - zf[k - 1]);
  dzf_global[0] = dzf_global[1];
  dzf_global[nz + 1] = dzf_global[nz];
}

// mod_mesh.cc:43-64 (derived z arrays of initMesh, single rank)
void host_mesh_derived(int nz, double lz, const double *dzf_global, double *dzf,
                       double *dzf_inv, double *dzc, double *dzc_inv,
                       double *dzflzi, double *zc_global) {
  for (int k = 0; k <= nz + 1; ++k) dzc[k] = dzc_inv[k] = 0.0;
  zc_global[0] = -0.5 * dzf_global[0];
  for (int k = 1; k <= nz + 1; ++k)
    zc_global[k] = zc_global[k - 1] + 0.5 * (dzf_global[k - 1] + dzf_global[k]);
  for (int k = 0; k <= nz + 1; ++k) {
    dzf[k] = dzf_global[k];
    dzf_inv[k] = 1.0 / dzf[k];
  }
  for (int k = 0; k <= nz; ++k) {
    dzc[k] = 0.5 * (dzf[k] + dzf[k + 1]);
    dzc_inv[k] = 1.0 / dzc[k];
  }
  for (int k = 0; k <= nz + 1; ++k) dzflzi[k] = dzf[k] / lz;
}

// mod_fft.cc:196-222 (periodic "PP" eigenvalues in the packed order)
void host_eigen_values(int ist, int isz, int isz_global, double *lambda) {
  const double pi = acos(-1.0);
  const int ien = ist + isz - 1;
  const int n = isz_global;
  std::vector<double> glb(n), aux(n);
  for (int i = 0; i < n; i++) aux[i] = 2.0 * (cos(2.0 * pi * (i - 0.0) / n) - 1.0);
  glb[0] = aux[0];
  glb[1] = aux[n / 2];
  for (int i = 2; i < n; i++) glb[i] = aux[i / 2];
  for (int i = ist; i <= ien; i++) lambda[i - ist] = glb[i - 1];
}

// Tridiagonal tables.  The reference builds a 3-D b[i,j,k] =
// b_tmp[k] + lambdax[i] + lambday[j] and eliminates it over k
// (mod_poisson_solver.cc:231-282, set_trid_coeff :35-98 with "NN").  Packed
// indices 2m and 2m+1 share the wavenumber m, so b only depends on the
// distinct pair (mx, my), mx in [0, nx/2], my in [0, ny/2]; the table holds
// 1/b for each distinct pair, computed with the same operations in the same
// order as the reference, and 0 where the final pivot is exactly 0 (the
// reference then sets the unknown to 0, :341-346).
void host_trid_tables(int nx, int ny, int nz, double dx, double dy,
                      const double *dzf_global, std::vector<double> &rpiv,
                      std::vector<double> &a, std::vector<double> &c) {
  std::vector<double> lx(nx), ly(ny);
  host_eigen_values(1, nx, nx, lx.data());
  for (int i = 0; i < nx; i++) lx[i] /= (dx * dx);
  host_eigen_values(1, ny, ny, ly.data());
  for (int i = 0; i < ny; i++) ly[i] /= (dy * dy);
  a.assign(nz, 0.0);
  c.assign(nz, 0.0);
  std::vector<double> b_tmp(nz);
  const double *dzf = dzf_global;
  const int dzf_st = -1;
  for (int k = 0; k < nz; k++) {
    a[k] = 2.0 / (dzf[k - dzf_st] * (dzf[k - 1 - dzf_st] + dzf[k - dzf_st]));
    c[k] = 2.0 / (dzf[k - dzf_st] * (dzf[k + 1 - dzf_st] + dzf[k - dzf_st]));
  }
  for (int i = 0; i < nz; i++) b_tmp[i] = -a[i] - c[i];
  const double factor = 1.0;  // Neumann at both walls
  b_tmp[0] += factor * a[0];
  a[0] *= fabs(factor) - 1.0;
  b_tmp[nz - 1] += factor * c[nz - 1];
  c[nz - 1] *= fabs(factor) - 1.0;

  const int MX = nx / 2 + 1, MY = ny / 2 + 1;
  auto rep = [](int m, int n) { return m == 0 ? 0 : (m == n / 2 ? 1 : 2 * m); };
  rpiv.assign((size_t)MX * MY * nz, 0.0);
  std::vector<double> bprev((size_t)MX * MY), bcur((size_t)MX * MY);
  for (int my = 0; my < MY; ++my)
    for (int mx = 0; mx < MX; ++mx) {
      const double lxy = lx[rep(mx, nx)] + ly[rep(my, ny)];
      bprev[(size_t)my * MX + mx] = b_tmp[0] + lxy;
    }
  for (size_t t = 0; t < bprev.size(); ++t) rpiv[t] = 1.0 / bprev[t];
  for (int k = 1; k < nz; ++k) {
    for (int my = 0; my < MY; ++my)
      for (int mx = 0; mx < MX; ++mx) {
        const size_t t = (size_t)my * MX + mx;
        const double lxy = lx[rep(mx, nx)] + ly[rep(my, ny)];
        double b = b_tmp[k] + lxy;
        const double a_tmp = a[k] / bprev[t];
        b -= (a_tmp * c[k - 1]);
        bcur[t] = b;
      }
    for (size_t t = 0; t < bcur.size(); ++t) rpiv[(size_t)k * MX * MY + t] = 1.0 / bcur[t];
    bprev.swap(bcur);
  }
  // zero final pivots (only the last plane is tested by the reference)
  for (size_t t = 0; t < bprev.size(); ++t)
    if (bprev[t] == 0.0) rpiv[(size_t)(nz - 1) * MX * MY + t] = 0.0;
}

// Roots of unity exp(-2 pi i t / n), t = 0..n-1, rounded from long double.
void host_twiddles(int n, std::vector<double> &re_im) {
  re_im.resize(2 * (size_t)n);
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int t = 0; t < n; ++t) {
    const long double ang = -two_pi * (long double)t / (long double)n;
    re_im[2 * t] = (double)cosl(ang);
    re_im[2 * t + 1] = (double)sinl(ang);
  }
}

// Radix sequence for a complex FFT of length n = 2^a 3^b (radices 16, 8, 4, 2, 3).
bool host_fft_factor(int n, int *radix, int *npass) {
  if (n < 1) return false;
  int m = n, a = 0, b = 0;
  while (m % 2 == 0) { m /= 2; ++a; }
  while (m % 3 == 0) { m /= 3; ++b; }
  if (m != 1) return false;
  int p = 0;
  while (a >= 4) { radix[p++] = 16; a -= 4; }
  if (a == 3) radix[p++] = 8;
  if (a == 2) radix[p++] = 4;
  if (a == 1) radix[p++] = 2;
  while (b-- > 0) radix[p++] = 3;
  if (p > 16) return false;
  *npass = p;
  return true;
}

// ---------------------------------------------------------------------------
// param.json reader.  The reference uses RapidJSON (mod_parameters.cc:220-260):
// a missing section is an error, a missing key keeps its default.
// ---------------------------------------------------------------------------
namespace {

struct JVal {
  enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
  bool b = false;
  double num = 0;
  std::string str;
  std::vector<JVal> arr;
  std::vector<std::pair<std::string, JVal>> obj;
  const JVal *find(const char *key) const {
    for (auto &kv : obj)
      if (kv.first == key) return &kv.second;
    return nullptr;
  }
};

struct JParser {
  const std::string &s;
  size_t p = 0;
  std::string err;
  explicit JParser(const std::string &src) : s(src) {}
  void ws() {
    while (p < s.size() && isspace((unsigned char)s[p])) ++p;
  }
  bool fail(const char *m) {
    if (err.empty()) {
      std::ostringstream o;
      o << m << " at offset " << p;
      err = o.str();
    }
    return false;
  }
  bool parse(JVal &v) {
    ws();
    if (p >= s.size()) return fail("unexpected end of input");
    char ch = s[p];
    if (ch == '{') return parse_obj(v);
    if (ch == '[') return parse_arr(v);
    if (ch == '"') {
      v.kind = JVal::Str;
      return parse_str(v.str);
    }
    if (s.compare(p, 4, "true") == 0) { v.kind = JVal::Bool; v.b = true; p += 4; return true; }
    if (s.compare(p, 5, "false") == 0) { v.kind = JVal::Bool; v.b = false; p += 5; return true; }
    if (s.compare(p, 4, "null") == 0) { v.kind = JVal::Null; p += 4; return true; }
    if (ch == '-' || ch == '+' || isdigit((unsigned char)ch) || ch == '.') {
      const char *b = s.c_str() + p;
      char *e = nullptr;
      v.num = strtod(b, &e);
      if (e == b) return fail("bad number");
      v.kind = JVal::Num;
      p += (size_t)(e - b);
      return true;
    }
    return fail("unexpected character");
  }
  bool parse_str(std::string &out) {
    if (s[p] != '"') return fail("expected string");
    ++p;
    out.clear();
    while (p < s.size() && s[p] != '"') {
      if (s[p] == '\\' && p + 1 < s.size()) {
        ++p;
        char e = s[p];
        out.push_back(e == 'n' ? '\n' : e == 't' ? '\t' : e);
      } else {
        out.push_back(s[p]);
      }
      ++p;
    }
    if (p >= s.size()) return fail("unterminated string");
    ++p;
    return true;
  }
  bool parse_arr(JVal &v) {
    v.kind = JVal::Arr;
    ++p;
    ws();
    if (p < s.size() && s[p] == ']') { ++p; return true; }
    for (;;) {
      JVal e;
      if (!parse(e)) return false;
      v.arr.push_back(std::move(e));
      ws();
      if (p < s.size() && s[p] == ',') { ++p; continue; }
      if (p < s.size() && s[p] == ']') { ++p; return true; }
      return fail("expected , or ]");
    }
  }
  bool parse_obj(JVal &v) {
    v.kind = JVal::Obj;
    ++p;
    ws();
    if (p < s.size() && s[p] == '}') { ++p; return true; }
    for (;;) {
      ws();
      std::string key;
      if (!parse_str(key)) return false;
      ws();
      if (p >= s.size() || s[p] != ':') return fail("expected :");
      ++p;
      JVal e;
      if (!parse(e)) return false;
      v.obj.emplace_back(std::move(key), std::move(e));
      ws();
      if (p < s.size() && s[p] == ',') { ++p; continue; }
      if (p < s.size() && s[p] == '}') { ++p; return true; }
      return fail("expected , or }");
    }
  }
};

bool get_num(const JVal *v, double &out) {
  if (!v) return false;
  if (v->kind == JVal::Num) { out = v->num; return true; }
  if (v->kind == JVal::Bool) { out = v->b ? 1.0 : 0.0; return true; }
  return false;
}

void rd(const JVal &node, const char *key, int &val) {
  double d;
  if (get_num(node.find(key), d)) val = (int)d;
}
void rd(const JVal &node, const char *key, double &val) {
  double d;
  if (get_num(node.find(key), d)) val = d;
}
void rd_str(const JVal &node, const char *key, char *dst, size_t cap) {
  const JVal *v = node.find(key);
  if (v && v->kind == JVal::Str) {
    snprintf(dst, cap, "%s", v->str.c_str());
  }
}
template <int N>
void rd_arr(const JVal &node, const char *key, int (&val)[N]) {
  const JVal *v = node.find(key);
  if (!v || v->kind != JVal::Arr) return;
  for (int i = 0; i < N && i < (int)v->arr.size(); ++i) {
    double d;
    if (get_num(&v->arr[i], d)) val[i] = (int)d;
  }
}
template <int N>
void rd_arr(const JVal &node, const char *key, double (&val)[N]) {
  const JVal *v = node.find(key);
  if (!v || v->kind != JVal::Arr) return;
  for (int i = 0; i < N && i < (int)v->arr.size(); ++i) {
    double d;
    if (get_num(&v->arr[i], d)) val[i] = d;
  }
}

}  // namespace

int host_parse_param_json(const char *path, plc_params *prm, std::string &err) {
  std::ifstream ifs(path);
  if (!ifs) {
    err = std::string("PowerLLEL.ERROR.readInputParam: Fail to open file ") + path + "!";
    return PLC_ERR_IO;
  }
  std::stringstream ss;
  ss << ifs.rdbuf();
  const std::string text = ss.str();
  JParser jp(text);
  JVal root;
  if (!jp.parse(root) || root.kind != JVal::Obj) {
    err = "PowerLLEL.ERROR.readInputParam: cannot parse " + std::string(path) + ": " +
          (jp.err.empty() ? std::string("top level is not an object") : jp.err);
    return PLC_ERR_IO;
  }
  auto section = [&](const char *name) -> const JVal * {
    const JVal *s = root.find(name);
    if (!s || s->kind != JVal::Obj) {
      err = std::string("PowerLLEL.ERROR.readInputParam: Problem with ") + name +
            " in the input file!";
      return nullptr;
    }
    return s;
  };
  const JVal *n;
  if (!(n = section("PARA"))) return PLC_ERR_IO;  // mod_parameters.cc:48-56
  rd(*n, "p_row", prm->p_row);
  rd(*n, "p_col", prm->p_col);
  if (!(n = section("MESH"))) return PLC_ERR_IO;  // :58-74
  rd(*n, "read_mesh", prm->read_mesh);
  rd(*n, "mesh_type", prm->mesh_type);
  rd(*n, "stretch_func", prm->stretch_func);
  rd(*n, "stretch_ratio", prm->stretch_ratio);
  rd(*n, "nx", prm->nx);
  rd(*n, "ny", prm->ny);
  rd(*n, "nz", prm->nz);
  rd(*n, "lx", prm->lx);
  rd(*n, "ly", prm->ly);
  rd(*n, "lz", prm->lz);
  if (!(n = section("TIME"))) return PLC_ERR_IO;  // :76-87
  rd(*n, "nt_end", prm->nt_end);
  rd(*n, "dt", prm->dt);
  rd(*n, "nt_check", prm->nt_check);
  rd(*n, "cfl_limit", prm->cfl_limit);
  rd(*n, "div_limit", prm->div_limit);
  rd(*n, "cfl_target", prm->cfl_target);  // B200 build extension
  if (!(n = section("RESTART"))) return PLC_ERR_IO;  // :89-98
  rd(*n, "is_restart", prm->is_restart);
  rd_str(*n, "fn_prefix_input_inst", prm->fn_prefix_input_inst, sizeof prm->fn_prefix_input_inst);
  rd_str(*n, "fn_prefix_input_stat", prm->fn_prefix_input_stat, sizeof prm->fn_prefix_input_stat);
  if (!(n = section("PHYSICAL"))) return PLC_ERR_IO;  // :100-115
  rd(*n, "re", prm->re);
  rd(*n, "u_ref", prm->u_ref);
  rd(*n, "l_ref", prm->l_ref);
  {
    const JVal *f = n->find("initial_field");
    if (f && f->kind == JVal::Str) {
      if (f->str == "uni") prm->initial_field = PLC_INIT_UNI;
      else if (f->str == "poi") prm->initial_field = PLC_INIT_POI;
      else if (f->str == "log") prm->initial_field = PLC_INIT_LOG;
      else if (f->str == "mpi") prm->initial_field = PLC_INIT_MPI;
      else {
        err = "PowerLLEL.ERROR.readInputParam: unknown initial_field " + f->str;
        return PLC_ERR_IO;
      }
    }
  }
  rd(*n, "u0", prm->u0);
  rd(*n, "init_with_noise", prm->init_with_noise);
  rd(*n, "noise_intensity", prm->noise_intensity);
  rd(*n, "smooth_wall_visc", prm->smooth_wall_visc);
  rd(*n, "u_crf", prm->u_crf);
  if (!(n = section("FORCE"))) return PLC_ERR_IO;  // :117-125
  rd_arr(*n, "is_forced", prm->is_forced);
  rd_arr(*n, "vel_force", prm->vel_force);
  if (!(n = section("STATISTICS"))) return PLC_ERR_IO;  // :127-137
  rd(*n, "nt_init_stat", prm->nt_init_stat);
  rd(*n, "sample_interval", prm->sample_interval);
  rd_arr(*n, "stat_which_var", prm->stat_which_var);
  if (!(n = section("OUTPUT"))) return PLC_ERR_IO;  // :139-153
  rd(*n, "nt_out_scrn", prm->nt_out_scrn);
  rd(*n, "nt_out_inst", prm->nt_out_inst);
  rd(*n, "nt_out_stat", prm->nt_out_stat);
  rd(*n, "nt_out_save", prm->nt_out_save);
  rd(*n, "overwrite_save", prm->overwrite_save);
  rd(*n, "auto_cleanup", prm->auto_cleanup);
  rd(*n, "num_retained", prm->num_retained);
  rd(*n, "nt_out_moni", prm->nt_out_moni);
  if (!(n = section("MONITOR"))) return PLC_ERR_IO;  // :155-168
  rd(*n, "out_forcing", prm->out_forcing);
  rd(*n, "out_probe_point", prm->out_probe_point);
  rd_arr(*n, "probe_ijk", prm->probe_ijk);
  rd_arr(*n, "out_skf_z", prm->out_skf_z);
  rd(*n, "out_region", prm->out_region);
  rd(*n, "nt_out_region", prm->nt_out_region);
  rd_arr(*n, "region_ijk", prm->region_ijk);
  // optional B200 section
  if (const JVal *b = root.find("B200")) {
    if (b->kind == JVal::Obj) {
      const JVal *pr = b->find("precision");
      if (pr && pr->kind == JVal::Str) {
        if (pr->str == "fp64") prm->precision = PLC_FP64;
        else if (pr->str == "mixed") prm->precision = PLC_MIXED;
        else {
          err = "PowerLLEL.ERROR.readInputParam: unknown precision " + pr->str;
          return PLC_ERR_IO;
        }
      }
      rd(*b, "cfl_target", prm->cfl_target);
      rd(*b, "init_vortex_amp", prm->init_vortex_amp);
    }
  }
  return PLC_OK;
}

}  // namespace plc
