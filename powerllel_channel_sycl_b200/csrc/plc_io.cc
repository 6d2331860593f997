// Data I/O of the channel solver: HDF5 fields, statistics and mesh files,
// restart, the monitor text files and the time-marching driver, with the
// reference's file names, datasets and text formats (src/mod_dataIO.cc,
// src/mod_mesh.cc:127-147, src/mod_monitor.cc:57-330, src/main.cc:59-222).
// Host code over the context's download/upload and monitor entry points;
// files go through the minimal HDF5 writer/reader of plc_h5.cc.

#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "plc_h5.h"
#include "plc_internal.h"

namespace plc {

struct IoState {
  std::string dir;  // prefix of every output file name ("" = working directory)
  bool monitor_ready = false;
  FILE *force = nullptr, *probe = nullptr, *skf[2] = {nullptr, nullptr};
  bool have_probe = false;
  int region[6] = {1, 1, 1, 1, 1, 1};  // clipped region_ijk
};

void io_free(plc_ctx *c) {
  if (!c || !c->io) return;
  IoState *s = c->io;
  for (FILE *f : {s->force, s->probe, s->skf[0], s->skf[1]})
    if (f) std::fclose(f);
  delete s;
  c->io = nullptr;
}

namespace {

// get_stat_type (mod_dataIO.cc:39-66)
const char *const kStatType[kStatVars] = {"u", "v", "w", "u2", "v2", "w2",
                                          "uv", "uw", "vw", "p", "p2"};

IoState &io_of(plc_ctx *c) {
  if (!c->io) c->io = new IoState;
  return *c->io;
}

std::string out_path(plc_ctx *c, const std::string &name) {
  const std::string &d = io_of(c).dir;
  return d.empty() ? name : d + "/" + name;
}

std::string fmt_str(const char *f, ...) __attribute__((format(printf, 1, 2)));
std::string fmt_str(const char *f, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, f);
  std::vsnprintf(buf, sizeof buf, f, ap);
  va_end(ap);
  return buf;
}

const char *field_tag(int field) {
  switch (field) {
    case PLC_U: return "u";
    case PLC_V: return "v";
    case PLC_W: return "w";
    case PLC_U1: return "u1";
    case PLC_V1: return "v1";
    case PLC_W1: return "w1";
    case PLC_P: return "p";
    default: return nullptr;
  }
}

// The interior (nz, ny, nx; x fastest) of a field downloaded in the halo'd
// reference layout.
int download_interior(plc_ctx *c, int field, std::vector<double> &out) {
  const int X = c->nx + 2, Y = c->ny + 2;
  std::vector<double> full((size_t)X * Y * (c->nz + 2));
  if (int rc = plc_download(c, field, full.data())) return rc;
  out.resize((size_t)c->nx * c->ny * c->nz);
  size_t q = 0;
  for (int k = 1; k <= c->nz; ++k)
    for (int j = 1; j <= c->ny; ++j)
      for (int i = 1; i <= c->nx; ++i) out[q++] = full[i + (size_t)X * (j + (size_t)Y * k)];
  return PLC_OK;
}

int upload_interior(plc_ctx *c, int field, const std::vector<double> &in) {
  const int X = c->nx + 2, Y = c->ny + 2;
  std::vector<double> full((size_t)X * Y * (c->nz + 2));
  if (int rc = plc_download(c, field, full.data())) return rc;  // keep the halos
  size_t q = 0;
  for (int k = 1; k <= c->nz; ++k)
    for (int j = 1; j <= c->ny; ++j)
      for (int i = 1; i <= c->nx; ++i) full[i + (size_t)X * (j + (size_t)Y * k)] = in[q++];
  return plc_upload(c, field, full.data());
}

int write_h5(plc_ctx *c, const std::string &path, const std::vector<h5::Dataset> &sets) {
  std::string err;
  if (!h5::write_file(path, sets, err)) return set_error(c, PLC_ERR_IO, "PowerLLEL.ERROR: " + err);
  return PLC_OK;
}

int read_h5(plc_ctx *c, const std::string &path, const std::string &name, std::vector<double> &out,
            std::vector<uint64_t> &dims) {
  std::string err;
  if (!h5::read_dataset(path, name, out, dims, err)) return set_error(c, PLC_ERR_IO, err);
  return PLC_OK;
}

int read_int(plc_ctx *c, const std::string &path, const char *name, int *val) {
  std::vector<double> v;
  std::vector<uint64_t> d;
  if (int rc = read_h5(c, path, name, v, d)) return rc;
  if (v.size() != 1) return set_error(c, PLC_ERR_IO, path + ": dataset '" + name + "' is not a scalar");
  *val = (int)v[0];
  return PLC_OK;
}

// outputField (mod_dataIO.cc:86-101): the 3-D dataset plus "nt", or the
// "nts", "nte", "nspl" of a statistics file
int output_field(plc_ctx *c, const std::string &path, const std::string &tag,
                 const std::vector<double> &var, int nt, const int *stat_info) {
  std::vector<h5::Dataset> sets;
  int ints[3];
  if (!stat_info) {
    ints[0] = nt;
    sets.push_back({"nt", h5::Type::I32, {1}, &ints[0]});
  } else {
    const char *names[3] = {"nts", "nte", "nspl"};
    for (int q = 0; q < 3; ++q) {
      ints[q] = stat_info[q];
      sets.push_back({names[q], h5::Type::I32, {1}, &ints[q]});
    }
  }
  sets.push_back({tag, h5::Type::F64, {(uint64_t)c->nz, (uint64_t)c->ny, (uint64_t)c->nx}, var.data()});
  return write_h5(c, path, sets);
}

int check_dims(plc_ctx *c, const std::string &path, const std::vector<uint64_t> &dims) {
  if (dims.size() != 3 || dims[0] != (uint64_t)c->nz || dims[1] != (uint64_t)c->ny ||
      dims[2] != (uint64_t)c->nx)
    return set_error(c, PLC_ERR_IO,
                     path + ": field dimensions differ from the context's (nz, ny, nx) = (" +
                         std::to_string(c->nz) + ", " + std::to_string(c->ny) + ", " +
                         std::to_string(c->nx) + ")");
  return PLC_OK;
}

// u written with u_crf added in place and removed again, as outputData does
// (mod_dataIO.cc:141-147): the context's u afterwards is (u + u_crf) - u_crf.
int write_u_lab_frame(plc_ctx *c, const std::string &path, int nt) {
  const double u_crf = c->prm.u_crf;
  std::vector<double> var;
  if (u_crf != 0.0)
    if (int rc = shift_field(c, PLC_U, -u_crf)) return rc;
  int rc = download_interior(c, PLC_U, var);
  if (u_crf != 0.0) {
    const int rc2 = shift_field(c, PLC_U, u_crf);
    if (rc == PLC_OK) rc = rc2;
  }
  if (rc) return rc;
  return output_field(c, path, "u", var, nt, nullptr);
}

int write_plain(plc_ctx *c, const std::string &path, int field, int nt) {
  std::vector<double> var;
  if (int rc = download_interior(c, field, var)) return rc;
  return output_field(c, path, field_tag(field), var, nt, nullptr);
}

int write_stat(plc_ctx *c, const std::string &path, int which) {
  std::vector<double> var((size_t)c->nx * c->ny * c->nz);
  if (int rc = plc_stat_download(c, which, var.data())) return rc;
  const int info[3] = {c->stat_nts, c->stat_nte, c->stat_nspl};
  return output_field(c, path, std::string(kStatType[which]) + "_stat", var, 0, info);
}

void note(const std::string &s) {
  std::fputs(s.c_str(), stdout);
  std::fflush(stdout);
}

// initMonitor (mod_monitor.cc:208-310).  The reference opens the files with
// out|ate, which truncates them, restart or not: so does this.
int monitor_init(plc_ctx *c) {
  IoState &s = io_of(c);
  plc_params &P = c->prm;
  FILE **files[4] = {&s.force, &s.probe, &s.skf[0], &s.skf[1]};
  for (FILE **f : files)
    if (*f) {
      std::fclose(*f);
      *f = nullptr;
    }
  auto open = [&](const char *name, FILE *&f) -> int {
    f = std::fopen(out_path(c, name).c_str(), "w");
    if (!f) return set_error(c, PLC_ERR_IO, "PowerLLEL.ERROR: cannot create " + out_path(c, name));
    return PLC_OK;
  };
  if (P.out_forcing) {
    if (int rc = open("monitor_forcing.out", s.force)) return rc;
    std::fprintf(s.force, "%9s%15s%15s%15s\n", "nt", "u_mean", "v_mean", "w_mean");
  }
  if (P.out_probe_point) {
    const int ig = P.probe_ijk[0], jg = P.probe_ijk[1], kg = P.probe_ijk[2];
    s.have_probe = ig >= 1 && ig <= c->nx && jg >= 1 && jg <= c->ny && kg >= 1 && kg <= c->nz;
    if (int rc = open("monitor_probe.out", s.probe)) return rc;
    if (s.have_probe) {
      std::fprintf(s.probe, "Probe point (%4d,%4d,%4d):\n", ig, jg, kg);
      std::fprintf(s.probe, "%9s%15s%15s%15s%15s\n", "nt", "u", "v", "w", "p");
    }
  }
  const char *skf_names[2] = {"monitor_skf_z1.out", "monitor_skf_z2.out"};
  for (int wall = 0; wall < 2; ++wall)
    if (P.out_skf_z[wall]) {
      if (int rc = open(skf_names[wall], s.skf[wall])) return rc;
      std::fprintf(s.skf[wall], "%9s%15s%15s\n", "nt", "u_tau", "cf");
    }
  if (P.out_region) {  // :271-279, clipped to the domain in place as the reference does
    int *r = P.region_ijk;
    r[0] = std::max(r[0], 1);
    r[1] = std::min(r[1], c->nx);
    r[2] = std::max(r[2], 1);
    r[3] = std::min(r[3], c->ny);
    r[4] = std::max(r[4], 1);
    r[5] = std::min(r[5], c->nz);
    std::memcpy(s.region, r, sizeof s.region);
  }
  for (FILE *f : {s.force, s.probe, s.skf[0], s.skf[1]})
    if (f) std::fflush(f);
  s.monitor_ready = true;
  return PLC_OK;
}

// extractAndWriteRegion (mod_monitor.cc:160-205): monitor_region_{nt:08}.h5
// with "nt" and u (x-centred, + u_crf), v, w (centred), p over the region
int write_region(plc_ctx *c, int nt) {
  const int *r = io_of(c).region;
  const int gx = r[1] - r[0] + 1, gy = r[3] - r[2] + 1, gz = r[5] - r[4] + 1;
  if (gx <= 0 || gy <= 0 || gz <= 0) return PLC_OK;  // no part of the region in the domain
  const size_t n = (size_t)gx * gy * gz;
  std::vector<double> buf[4];
  const int fields[4] = {PLC_U, PLC_V, PLC_W, PLC_P};
  std::vector<h5::Dataset> sets;
  int ntv = nt;
  sets.push_back({"nt", h5::Type::I32, {1}, &ntv});
  for (int q = 0; q < 4; ++q) {
    buf[q].resize(n);
    if (int rc = plc_extract_region(c, r, fields[q], buf[q].data())) return rc;
    sets.push_back({field_tag(fields[q]), h5::Type::F64,
                    {(uint64_t)gz, (uint64_t)gy, (uint64_t)gx}, buf[q].data()});
  }
  return write_h5(c, out_path(c, fmt_str("monitor_region_%08d.h5", nt)), sets);
}

// outputMonitor (mod_monitor.cc:312-326)
int output_monitor(plc_ctx *c, int nt) {
  IoState &s = io_of(c);
  const plc_params &P = c->prm;
  if (!s.monitor_ready)
    if (int rc = monitor_init(c)) return rc;
  if (P.out_forcing && s.force &&
      (P.is_forced[0] || P.is_forced[1] || P.is_forced[2])) {
    double m[3];
    if (int rc = plc_monitor_forcing(c, m)) return rc;
    std::fprintf(s.force, "%9d%15.7E%15.7E%15.7E\n", nt, m[0], m[1], m[2]);
    std::fflush(s.force);
  }
  if (P.out_probe_point && s.have_probe) {
    double q[4];
    if (int rc = plc_monitor_probe(c, P.probe_ijk[0], P.probe_ijk[1], P.probe_ijk[2], q)) return rc;
    std::fprintf(s.probe, "%9d%15.7E%15.7E%15.7E%15.7E\n", nt, q[0], q[1], q[2], q[3]);
    std::fflush(s.probe);
  }
  for (int wall = 0; wall < 2; ++wall)
    if (P.out_skf_z[wall] && s.skf[wall]) {
      double u_tau, cf;
      if (int rc = plc_monitor_skf(c, wall, &u_tau, &cf)) return rc;
      std::fprintf(s.skf[wall], "%9d%15.7E%15.7E\n", nt, u_tau, cf);
      std::fflush(s.skf[wall]);
    }
  if (P.out_region && P.nt_out_region > 0 && nt % P.nt_out_region == 0)
    if (int rc = write_region(c, nt)) return rc;
  return PLC_OK;
}

// outputStatData (mod_dataIO.cc:254-302)
int output_stat_data(plc_ctx *c, int nt, bool verbose) {
  const plc_params &P = c->prm;
  if (!c->stat_ready) return PLC_OK;
  if (P.nt_out_save > 0 && nt % P.nt_out_save == 0) {
    if (verbose) note("PowerLLEL.NOTE.outputStatData: Writing checkpoint fields of statistics ...\n");
    // the reference versions these names when overwrite_save is set
    // (:261-264), the opposite of the field checkpoints
    const std::string dump = P.overwrite_save ? fmt_str("_%08d_", nt) : std::string("_");
    for (int i = 0; i < kStatVars; ++i) {
      if (!P.stat_which_var[i]) continue;
      if (int rc = write_stat(c, out_path(c, "save" + dump + "stat_" + kStatType[i] + ".h5"), i))
        return rc;
      if (verbose)
        note(fmt_str("PowerLLEL.NOTE.outputStatData: Finish writing checkpoint field <%s_stat>!\n",
                     kStatType[i]));
    }
  }
  if (P.nt_out_stat > 0 && (nt - P.nt_init_stat) % P.nt_out_stat == 0) {
    if (verbose) note("PowerLLEL.NOTE.outputStatData: Writing statistics fields ...\n");
    const std::string prefix = fmt_str("stat_%08d-%08d_", c->stat_nts, c->stat_nte);
    for (int i = 0; i < kStatVars; ++i) {
      if (!P.stat_which_var[i]) continue;
      if (int rc = write_stat(c, out_path(c, prefix + kStatType[i] + ".h5"), i)) return rc;
      if (verbose)
        note(fmt_str("PowerLLEL.NOTE.outputStatData: Finish writing stat. field <%s_stat>!\n",
                     kStatType[i]));
    }
  }
  return PLC_OK;
}

int output_data(plc_ctx *c, int nt, bool verbose) {
  const plc_params &P = c->prm;
  if (P.nt_out_moni > 0 && nt % P.nt_out_moni == 0)
    if (int rc = output_monitor(c, nt)) return rc;
  const char *uvwp[4] = {"u", "v", "w", "p"};
  if (P.nt_out_inst > 0 && nt % P.nt_out_inst == 0) {
    if (verbose) note("PowerLLEL.NOTE.outputData: Writing instantaneous fields ...\n");
    const std::string prefix = fmt_str("inst_%08d_", nt);
    for (int q = 0; q < 4; ++q) {
      const std::string path = out_path(c, prefix + uvwp[q] + ".h5");
      const int field = q == 3 ? PLC_P : q;
      if (int rc = q == 0 ? write_u_lab_frame(c, path, nt) : write_plain(c, path, field, nt)) return rc;
      if (verbose)
        note(fmt_str("PowerLLEL.NOTE.outputData: Finish writing inst. field <%s>!\n", uvwp[q]));
    }
  }
  if (P.nt_out_save > 0 && nt % P.nt_out_save == 0) {
    if (verbose) note("PowerLLEL.NOTE.outputData: Writing checkpoint fields ...\n");
    const std::string dump = P.overwrite_save ? std::string("_") : fmt_str("_%08d_", nt);
    for (int q = 0; q < 3; ++q) {
      const std::string path = out_path(c, "save" + dump + uvwp[q] + ".h5");
      if (int rc = q == 0 ? write_u_lab_frame(c, path, nt) : write_plain(c, path, q, nt)) return rc;
      if (verbose)
        note(fmt_str("PowerLLEL.NOTE.outputData: Finish writing checkpoint field <%s>!\n", uvwp[q]));
    }
  }
  if (nt > P.nt_init_stat)
    if (int rc = output_stat_data(c, nt, verbose)) return rc;
  // automatic cleanup of versioned checkpoints (:205-227)
  if (!P.overwrite_save && P.auto_cleanup && P.nt_out_save > 0 && nt % P.nt_out_save == 0) {
    const int nt_cleanup = nt - (P.num_retained + 1) * P.nt_out_save;
    const std::string prefix = out_path(c, fmt_str("save_%08d_", nt_cleanup));
    if (nt_cleanup > 0) {
      if (verbose) note("PowerLLEL.NOTE.outputData: Automatically cleanup of inst. checkpoint files ...\n");
      for (int q = 0; q < 3; ++q) std::remove((prefix + uvwp[q] + ".h5").c_str());
    }
    if (nt_cleanup > P.nt_init_stat) {
      if (verbose) note("PowerLLEL.NOTE.outputData: Automatically cleanup of stat. checkpoint files ...\n");
      for (int i = 0; i < kStatVars; ++i)
        if (P.stat_which_var[i]) std::remove((prefix + "stat_" + kStatType[i] + ".h5").c_str());
    }
  }
  return PLC_OK;
}

// The first step t >= nt after which the driver has host work to do (the
// screen line, monitors, field or statistics files, the start of the
// statistics), or nt_end.
int next_event(const plc_ctx *c, int nt, int nt_end) {
  const plc_params &P = c->prm;
  long long best = nt_end;
  // smallest t >= from with (t - offset) a multiple of period
  auto mult = [&](long long from, int period, long long offset) {
    if (period <= 0) return;
    const long long r = ((from - offset) % period + period) % period;
    best = std::min(best, r == 0 ? from : from + (period - r));
  };
  mult(nt, P.nt_out_scrn, 0);
  mult(nt, P.nt_out_moni, 0);
  mult(nt, P.nt_out_inst, 0);
  mult(nt, P.nt_out_save, 0);
  const long long first_stat = (long long)P.nt_init_stat + 1;
  if (nt <= first_stat) best = std::min(best, first_stat);
  mult(std::max<long long>(nt, first_stat), P.nt_out_stat, P.nt_init_stat);
  return (int)std::max<long long>(best, nt);
}

}  // namespace
}  // namespace plc

using namespace plc;

extern "C" {

unsigned int plc_h5_lookup3(const void *key, size_t length, unsigned int initval) {
  return h5::lookup3(static_cast<const uint8_t *>(key), length, initval);
}

int plc_h5_write(const char *path, int nsets, const char *const *names, const int *types,
                 const int *ndims, const long long *dims, const void *const *data) {
  if (!path || nsets < 0 || (nsets > 0 && (!names || !types || !ndims || !dims || !data)))
    return set_error(nullptr, PLC_ERR_ARG, "null argument");
  std::vector<h5::Dataset> sets(nsets);
  const long long *d = dims;
  for (int q = 0; q < nsets; ++q) {
    if (!names[q] || !data[q] || ndims[q] < 1 || ndims[q] > 32 || std::strlen(names[q]) > 255 ||
        (types[q] != 0 && types[q] != 1))
      return set_error(nullptr, PLC_ERR_ARG, "bad dataset description");
    sets[q].name = names[q];
    sets[q].type = types[q] == 0 ? h5::Type::F64 : h5::Type::I32;
    for (int r = 0; r < ndims[q]; ++r) {
      if (d[r] < 0) return set_error(nullptr, PLC_ERR_ARG, "negative dimension");
      sets[q].dims.push_back((uint64_t)d[r]);
    }
    d += ndims[q];
    sets[q].data = data[q];
  }
  std::string err;
  if (!h5::write_file(path, sets, err)) return set_error(nullptr, PLC_ERR_IO, err);
  return PLC_OK;
}

int plc_h5_read(const char *path, const char *name, double *out, size_t capacity,
                long long *dims, int *ndim) {
  if (!path || !name || !ndim) return set_error(nullptr, PLC_ERR_ARG, "null argument");
  std::vector<double> v;
  std::vector<uint64_t> d;
  std::string err;
  if (!h5::read_dataset(path, name, v, d, err)) return set_error(nullptr, PLC_ERR_IO, err);
  const int cap_dims = *ndim;
  *ndim = (int)d.size();
  if (dims)
    for (int r = 0; r < (int)d.size() && r < cap_dims; ++r) dims[r] = (long long)d[r];
  if (out) {
    if (v.size() > capacity) return set_error(nullptr, PLC_ERR_ARG, "output buffer too small");
    std::memcpy(out, v.data(), v.size() * sizeof(double));
  }
  return PLC_OK;
}

int plc_read_mesh_in(const char *path, int nz, double *dzf_global) {
  if (!path || !dzf_global || nz < 1) return set_error(nullptr, PLC_ERR_ARG, "bad argument");
  // inputMesh (mod_mesh.cc:78-93): nz whitespace-separated spacings, the
  // ghost entries copied from their neighbours
  FILE *f = std::fopen(path, "r");
  if (!f)
    return set_error(nullptr, PLC_ERR_IO,
                     std::string("PowerLLEL.ERROR.inputMesh: File ") + path + " doesn't exist!");
  for (int k = 1; k <= nz; ++k)
    if (std::fscanf(f, "%lf", &dzf_global[k]) != 1) {
      std::fclose(f);
      return set_error(nullptr, PLC_ERR_IO,
                       fmt_str("PowerLLEL.ERROR.inputMesh: %s holds fewer than nz = %d values", path, nz));
    }
  std::fclose(f);
  dzf_global[0] = dzf_global[1];
  dzf_global[nz + 1] = dzf_global[nz];
  return PLC_OK;
}

int plc_device_name(int device, char *buf, int len) {
  if (!buf || len < 1) return set_error(nullptr, PLC_ERR_ARG, "bad argument");
  cudaDeviceProp prop;
  const cudaError_t e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) return set_error(nullptr, PLC_ERR_CUDA, cudaGetErrorString(e));
  std::snprintf(buf, (size_t)len, "%s", prop.name);
  return PLC_OK;
}

int plc_set_output_dir(plc_ctx *c, const char *dir) {
  if (!c) return set_error(nullptr, PLC_ERR_ARG, "null context");
  io_of(c).dir = dir ? dir : "";
  return PLC_OK;
}

int plc_write_field_h5(plc_ctx *c, const char *path, int field, int nt) {
  if (!c || !path) return set_error(c, PLC_ERR_ARG, "null argument");
  if (!field_tag(field)) return set_error(c, PLC_ERR_ARG, "bad field id");
  return field == PLC_U ? write_u_lab_frame(c, path, nt) : write_plain(c, path, field, nt);
}

int plc_read_field_h5(plc_ctx *c, const char *path, int field, int *nt) {
  if (!c || !path) return set_error(c, PLC_ERR_ARG, "null argument");
  const char *tag = field_tag(field);
  if (!tag) return set_error(c, PLC_ERR_ARG, "bad field id");
  std::vector<double> var;
  std::vector<uint64_t> dims;
  int t = 0;
  if (int rc = read_int(c, path, "nt", &t)) return rc;
  if (int rc = read_h5(c, path, tag, var, dims)) return rc;
  if (int rc = check_dims(c, path, dims)) return rc;
  if (int rc = upload_interior(c, field, var)) return rc;
  if (nt) *nt = t;
  return PLC_OK;
}

int plc_write_stat_h5(plc_ctx *c, const char *path, int which) {
  if (!c || !path) return set_error(c, PLC_ERR_ARG, "null argument");
  if (which < 0 || which >= kStatVars) return set_error(c, PLC_ERR_ARG, "bad statistic id");
  return write_stat(c, path, which);
}

int plc_read_stat_h5(plc_ctx *c, const char *path, int which, int *nte) {
  if (!c || !path) return set_error(c, PLC_ERR_ARG, "null argument");
  if (which < 0 || which >= kStatVars) return set_error(c, PLC_ERR_ARG, "bad statistic id");
  int info[3];
  const char *names[3] = {"nts", "nte", "nspl"};
  for (int q = 0; q < 3; ++q)
    if (int rc = read_int(c, path, names[q], &info[q])) return rc;
  std::vector<double> var;
  std::vector<uint64_t> dims;
  if (int rc = read_h5(c, path, std::string(kStatType[which]) + "_stat", var, dims)) return rc;
  if (int rc = check_dims(c, path, dims)) return rc;
  if (int rc = plc_stat_upload(c, which, var.data(), info[0], info[1], info[2])) return rc;
  if (nte) *nte = info[1];
  return PLC_OK;
}

int plc_output_mesh(plc_ctx *c) {
  if (!c) return set_error(nullptr, PLC_ERR_ARG, "null context");
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  // mod_mesh.cc:31-37 and :49-53
  std::vector<double> xc(nx), yc(ny), zc(nz);
  const double xc0 = -0.5 * c->dx, yc0 = -0.5 * c->dy;
  for (int i = 1; i <= nx; ++i) xc[i - 1] = xc0 + i * c->dx;
  for (int j = 1; j <= ny; ++j) yc[j - 1] = yc0 + j * c->dy;
  for (int k = 1; k <= nz; ++k) zc[k - 1] = c->h_zc_global[k];
  const std::string name = fmt_str("mesh_%d-%d-%d.h5", nx, ny, nz);
  if (int rc = write_h5(c, out_path(c, name),
                        {{"xc", h5::Type::F64, {(uint64_t)nx}, xc.data()},
                         {"yc", h5::Type::F64, {(uint64_t)ny}, yc.data()},
                         {"zc", h5::Type::F64, {(uint64_t)nz}, zc.data()}}))
    return rc;
  const std::string text = out_path(c, fmt_str("mesh_%05d.out", nz));
  FILE *f = std::fopen(text.c_str(), "w");
  if (!f) return set_error(c, PLC_ERR_IO, "PowerLLEL.ERROR: cannot create " + text);
  std::fprintf(f, "%4s%s%21s%s%22s%s\n", "", "k", "", "dzf", "", "zc");
  for (int k = 1; k <= nz; ++k)
    std::fprintf(f, "%05d %23.15E %23.15E\n", k, c->h_dzf_global[k], c->h_zc_global[k]);
  if (std::fclose(f) != 0) return set_error(c, PLC_ERR_IO, "PowerLLEL.ERROR: write error on " + text);
  return PLC_OK;
}

int plc_input_data(plc_ctx *c, int *nt_in) {
  if (!c) return set_error(nullptr, PLC_ERR_ARG, "null context");
  const plc_params &P = c->prm;
  // inputData (mod_dataIO.cc:104-128)
  const std::string prefix = P.fn_prefix_input_inst;
  int nt_u = 0;
  const char *uvw[3] = {"u", "v", "w"};
  for (int q = 0; q < 3; ++q) {
    int nt_q = 0;
    if (int rc = plc_read_field_h5(c, (prefix + "_" + uvw[q] + ".h5").c_str(), q, &nt_q)) return rc;
    if (q == 0) nt_u = nt_q;
    else if (nt_q != nt_u)
      return set_error(c, PLC_ERR_IO,
                       fmt_str("PowerLLEL.ERROR.inputData: The timestamp of <%s> does not match "
                               "with that of <u>!",
                               uvw[q]));
  }
  // main.cc:77-82
  if (int rc = plc_finish_input(c)) return rc;
  // main.cc:84-88, inputStatData (mod_dataIO.cc:232-252)
  const int nt_start = nt_u + 1;
  if (nt_start > P.nt_init_stat + 1) {
    if (int rc = plc_stat_init(c)) return rc;
    for (int i = 0; i < kStatVars; ++i) {
      if (!P.stat_which_var[i]) continue;
      const std::string path = std::string(P.fn_prefix_input_stat) + "_" + kStatType[i] + ".h5";
      int nte = 0;
      if (int rc = plc_read_stat_h5(c, path.c_str(), i, &nte)) return rc;
      if (nte != nt_u)
        return set_error(c, PLC_ERR_IO,
                         fmt_str("PowerLLEL.ERROR.inputStatData: The timestamp of <%s_stat> does "
                                 "not match with that of inst. field!",
                                 kStatType[i]));
    }
  }
  c->nstep = nt_u;
  if (nt_in) *nt_in = nt_u;
  return PLC_OK;
}

int plc_output_init(plc_ctx *c) {
  if (!c) return set_error(nullptr, PLC_ERR_ARG, "null context");
  return monitor_init(c);
}

int plc_output_data(plc_ctx *c, int nt) {
  if (!c) return set_error(nullptr, PLC_ERR_ARG, "null context");
  return output_data(c, nt, false);
}

int plc_output_free(plc_ctx *c) {
  if (!c) return set_error(nullptr, PLC_ERR_ARG, "null context");
  io_free(c);
  return PLC_OK;
}

int plc_run(plc_ctx *c, int nt_start, int verbose) {
  if (!c) return set_error(nullptr, PLC_ERR_ARG, "null context");
  const plc_params &P = c->prm;
  if (nt_start < 1) return set_error(c, PLC_ERR_ARG, "nt_start < 1");
  if (!io_of(c).monitor_ready)
    if (int rc = monitor_init(c)) return rc;
  c->nstep = nt_start - 1;  // the checks run on multiples of nt_check of nt
  if (verbose) {
    note(fmt_str("PowerLLEL.NOTE: Simulation starts at nt = %9d!\n", nt_start));
    note("********************************************************************************\n");
    note(fmt_str("%9s  %17s  %14s  %10s  %10s\n", "nt", "speed(wSteps/Day)", "remaining time",
                 "cfl_max", "div_max"));
  }
  using clock = std::chrono::steady_clock;
  auto t0 = clock::now();
  int nt = nt_start;
  while (nt <= P.nt_end) {
    // steps without host work run back to back from the captured graph
    const int stop = next_event(c, nt, P.nt_end);
    if (int rc = plc_step(c, stop - nt + 1)) return rc;
    nt = stop;
    // main.cc:180-190: the reference samples statistics once, at nt_init_stat + 1
    if (nt == P.nt_init_stat + 1) {
      if (int rc = plc_stat_init(c)) return rc;
      if (verbose) note(fmt_str("PowerLLEL.NOTE: Statistical process starts at nt = %d!\n", nt));
      if (int rc = plc_calc_stat(c, nt)) return rc;
    }
    if (P.nt_out_scrn > 0 && nt % P.nt_out_scrn == 0) {  // main.cc:192-212
      const double wtime = std::chrono::duration<double>(clock::now() - t0).count();
      if (verbose) {
        int t = (int)((P.nt_end - nt) * wtime / P.nt_out_scrn);
        const int t_d = t / 86400;
        int t_res = t % 86400;
        const int t_h = t_res / 3600;
        t_res %= 3600;
        const int t_m = t_res / 60, t_s = t_res % 60;
        const std::string remaining = fmt_str("%3dd%2dh%2dm%2ds", t_d, t_h, t_m, t_s);
        const double speed = P.nt_out_scrn * 3600.0 * 24.0 / wtime / 10000;
        note(fmt_str("%9d  %17.3f  %14s  %10.3E  %10.3E\n", nt, speed, remaining.c_str(),
                     c->last_cfl.value, c->last_div.value));
      }
    }
    if (int rc = output_data(c, nt, verbose != 0)) return rc;
    if (P.nt_out_scrn > 0 && nt % P.nt_out_scrn == 0) t0 = clock::now();
    ++nt;
  }
  if (verbose) {
    note("********************************************************************************\n");
    note("PowerLLEL.NOTE: Simulation ends successfully!\n");
  }
  return PLC_OK;
}

}  // extern "C"
