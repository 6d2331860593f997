// plc_main: the channel solver as a program, in place of the reference's
// executable (src/main.cc): reads param.json (or the path given as the first
// argument) from the working directory, builds the mesh (mesh.in when
// read_mesh), writes the mesh files, starts from the initial field or the
// checkpoint files, and runs the main loop with its checks, statistics,
// screen line and output files.  One GPU (p_row = p_col = 1); the device is
// the second argument (default 0).  Exit status 0 on success, 1 where the
// reference aborts (bad parameters, missing files, a failed check).

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "plc.h"

static int fail(plc_ctx *ctx, const char *what) {
  std::fprintf(stderr, "%s\n%s\n", what, plc_last_error(ctx));
  std::fflush(stderr);
  if (ctx) plc_destroy(ctx);
  return 1;
}

int main(int argc, char **argv) {
  const char *param = argc > 1 ? argv[1] : "param.json";
  const int device = argc > 2 ? std::atoi(argv[2]) : 0;
  std::printf(
      "================================================================================\n"
      "                      PowerLLEL_channel (DNS, 2ndFD + RK2)                      \n"
      "================================================================================\n"
      "PowerLLEL.NOTE: Initialization starts ...\n");
  std::fflush(stdout);

  plc_params prm;
  plc_params_default(&prm);
  if (plc_params_read_json(param, &prm) != PLC_OK) return fail(nullptr, "PowerLLEL.ERROR: reading the parameters failed");
  if (plc_params_check(&prm) != PLC_OK) return fail(nullptr, "PowerLLEL.ERROR: invalid parameters");

  std::vector<double> dzf;
  if (prm.read_mesh) {
    dzf.assign((size_t)prm.nz + 2, 0.0);
    if (plc_read_mesh_in("mesh.in", prm.nz, dzf.data()) != PLC_OK)
      return fail(nullptr, "PowerLLEL.ERROR: reading mesh.in failed");
  }
  plc_ctx *ctx = nullptr;
  if (plc_create(&prm, prm.read_mesh ? dzf.data() : nullptr, device, &ctx) != PLC_OK)
    return fail(nullptr, "PowerLLEL.ERROR: initialization failed");
  if (plc_output_init(ctx) != PLC_OK) return fail(ctx, "PowerLLEL.ERROR: initMonitor failed");
  if (plc_output_mesh(ctx) != PLC_OK) return fail(ctx, "PowerLLEL.ERROR: outputMesh failed");

  int nt_start = 1;
  if (prm.is_restart) {
    std::printf("PowerLLEL.NOTE: Initializing flow from checkpoint fields ...\n");
    int nt_in = 0;
    if (plc_input_data(ctx, &nt_in) != PLC_OK) return fail(ctx, "PowerLLEL.ERROR: inputData failed");
    nt_start = nt_in + 1;
  } else {
    std::printf("PowerLLEL.NOTE: Initializing flow according to input parameters ...\n");
    if (plc_init_flow(ctx) != PLC_OK) return fail(ctx, "PowerLLEL.ERROR: initFlow failed");
  }
  char name[256] = "unknown";
  plc_device_name(device, name, sizeof name);
  std::printf("PowerLLEL.NOTE: Initialization ends successfully!\n");
  std::printf("PowerLLEL.NOTE: Selected device is: CUDA, %s \n", name);
  std::fflush(stdout);

  if (plc_run(ctx, nt_start, 1) != PLC_OK) return fail(ctx, "PowerLLEL.ERROR: the main loop stopped");
  plc_destroy(ctx);
  return 0;
}
