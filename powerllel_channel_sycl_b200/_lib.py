"""ctypes binding of libplc.so (the C ABI declared in include/plc.h).

The library is built in-tree (``powerllel_channel_sycl_b200/lib/libplc.so``)
by ``powerllel_channel_sycl_b200.build.build()``.  There is no fallback: if
the shared library is missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libplc.so")

PLC_OK = 0
ERRORS = {
    -1: "PLC_ERR_ARG", -2: "PLC_ERR_SIZE", -3: "PLC_ERR_DECOMP", -4: "PLC_ERR_CUDA",
    -5: "PLC_ERR_CHECK", -6: "PLC_ERR_IO", -7: "PLC_ERR_NOMEM", -8: "PLC_ERR_STATE",
}
FIELDS = {"u": 0, "v": 1, "w": 2, "u1": 3, "v1": 4, "w1": 5, "p": 6, "spec": 7}
INIT_FIELDS = {"uni": 0, "poi": 1, "log": 2, "mpi": 3}
PRECISION = {"fp64": 0, "mixed": 1}


class PlcParams(C.Structure):
    """Mirror of ``plc_params`` (include/plc.h); every key of param.json."""
    _fields_ = [
        ("p_row", C.c_int), ("p_col", C.c_int),
        ("read_mesh", C.c_int), ("mesh_type", C.c_int), ("stretch_func", C.c_int),
        ("stretch_ratio", C.c_double),
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
        ("nt_end", C.c_int), ("nt_check", C.c_int),
        ("dt", C.c_double), ("cfl_limit", C.c_double), ("div_limit", C.c_double),
        ("is_restart", C.c_int),
        ("fn_prefix_input_inst", C.c_char * 128), ("fn_prefix_input_stat", C.c_char * 128),
        ("re", C.c_double), ("u_ref", C.c_double), ("l_ref", C.c_double),
        ("initial_field", C.c_int),
        ("u0", C.c_double),
        ("init_with_noise", C.c_int),
        ("noise_intensity", C.c_double),
        ("smooth_wall_visc", C.c_int),
        ("u_crf", C.c_double),
        ("is_forced", C.c_int * 3), ("vel_force", C.c_double * 3),
        ("nt_init_stat", C.c_int), ("sample_interval", C.c_int),
        ("stat_which_var", C.c_int * 11),
        ("nt_out_scrn", C.c_int), ("nt_out_inst", C.c_int), ("nt_out_stat", C.c_int),
        ("nt_out_save", C.c_int),
        ("overwrite_save", C.c_int), ("auto_cleanup", C.c_int), ("num_retained", C.c_int),
        ("nt_out_moni", C.c_int),
        ("out_forcing", C.c_int), ("out_probe_point", C.c_int),
        ("probe_ijk", C.c_int * 3),
        ("out_skf_z", C.c_int * 2),
        ("out_region", C.c_int), ("nt_out_region", C.c_int),
        ("region_ijk", C.c_int * 6),
        ("precision", C.c_int),
        ("cfl_target", C.c_double),
        ("init_vortex_amp", C.c_double),
    ]


class PlcValueIndex(C.Structure):
    _fields_ = [("value", C.c_double), ("ig", C.c_int), ("jg", C.c_int), ("kg", C.c_int)]


class PlcError(RuntimeError):
    def __init__(self, code: int, message: str):
        self.code = code
        self.name = ERRORS.get(code, str(code))
        super().__init__(f"{self.name}: {message}")


_lock = threading.Lock()
_lib = None

_vp = C.c_void_p
_dp = C.c_void_p  # device pointers travel as integers
_hp = C.c_void_p  # host pointers (numpy .ctypes.data)
_int = C.c_int
_dbl = C.c_double

_SIGS = {
    "plc_params_default": [C.POINTER(PlcParams)],
    "plc_params_read_json": [C.c_char_p, C.POINTER(PlcParams)],
    "plc_params_check": [C.POINTER(PlcParams)],
    "plc_create": [C.POINTER(PlcParams), _hp, _int, C.POINTER(_vp)],
    "plc_destroy": [_vp],
    "plc_sync": [_vp],
    "plc_get_mesh": [_vp, _int, _hp],
    "plc_field_ptr": [_vp, _int, C.POINTER(_vp), C.POINTER(C.c_size_t)],
    "plc_field_ptr_f32": [_vp, _int, C.POINTER(_vp), C.POINTER(C.c_size_t), C.POINTER(_int)],
    "plc_fft_tiles": [_vp, C.POINTER(_int), C.POINTER(_int), C.POINTER(_int)],
    "plc_fft_plans": [_vp, C.POINTER(_int), C.POINTER(_int)],
    "plc_fft_plan_x_fwd": [_vp, C.POINTER(_int)],
    "plc_rk_kchunk": [_vp, C.POINTER(_int)],
    "plc_rk2_carry": [_vp, C.POINTER(_int)],
    "plc_upload": [_vp, _int, _hp],
    "plc_download": [_vp, _int, _hp],
    "plc_get_dt": [_vp, C.POINTER(_dbl)],
    "plc_step_forcing": [_vp, _hp, _hp],
    "plc_set_dt": [_vp, _dbl],
    "plc_transform2crf": [_vp, _dbl, _dp, C.POINTER(_dbl)],
    "plc_time_int_vel_rk1": [_vp, _dbl, _dp, _dp, _dp, _dp, _dp, _dp],
    "plc_time_int_vel_rk2": [_vp, _dbl, _dp, _dp, _dp, _dp, _dp, _dp],
    "plc_correct_vel": [_vp, _dp, _dp, _dp, _dp],
    "plc_force_vel": [_vp, _dp, _dp, _dp, _hp],
    "plc_calc_rhs": [_vp, _dp, _dp, _dp, _dp],
    "plc_update_bound_vel": [_vp, _dbl, _dp, _dp, _dp],
    "plc_impose_bc_vel": [_vp, _dp, _dp, _dp, _dbl],
    "plc_update_bound_p": [_vp, _dp],
    "plc_init_poisson_solver": [_vp, _hp, C.c_char_p, C.c_char_p, C.c_char_p],
    "plc_execute_poisson_solver": [_vp, _dp],
    "plc_free_poisson_solver": [_vp],
    "plc_solve_trid": [_vp, _dp],
    "plc_fft_fwd_xpen": [_vp, _dp, _dp],
    "plc_fft_bwd_xpen": [_vp, _dp, _dp],
    "plc_fft_fwd_ypen": [_vp, _dp],
    "plc_fft_bwd_ypen": [_vp, _dp],
    "plc_get_eigen_values": [_int, _int, _int, C.c_char_p, _hp],
    "plc_mean": [_vp, _int, _int, _dp, C.POINTER(_dbl)],
    "plc_check_nan": [_vp, _dp, C.POINTER(_int)],
    "plc_calc_max_cfl": [_vp, _dp, _dp, _dp, C.POINTER(PlcValueIndex)],
    "plc_calc_max_div": [_vp, _dp, _dp, _dp, C.POINTER(PlcValueIndex)],
    "plc_init_flow": [_vp],
    "plc_finish_input": [_vp],
    "plc_stat_init": [_vp],
    "plc_stat_free": [_vp],
    "plc_calc_stat": [_vp, _int],
    "plc_stat_info": [_vp, C.POINTER(_int), C.POINTER(_int), C.POINTER(_int)],
    "plc_stat_download": [_vp, _int, _hp],
    "plc_stat_upload": [_vp, _int, _hp, _int, _int, _int],
    "plc_stat_profiles": [_vp, _hp],
    "plc_monitor_forcing": [_vp, _hp],
    "plc_monitor_probe": [_vp, _int, _int, _int, _hp],
    "plc_monitor_skf": [_vp, _int, C.POINTER(_dbl), C.POINTER(_dbl)],
    "plc_extract_region": [_vp, C.POINTER(_int), _int, _hp],
    "plc_step": [_vp, _int],
    "plc_last_check": [_vp, C.POINTER(_int), C.POINTER(PlcValueIndex), C.POINTER(PlcValueIndex)],
    "plc_check": [_vp, C.POINTER(_int), C.POINTER(PlcValueIndex), C.POINTER(PlcValueIndex)],
    "plc_step_count": [_vp, C.POINTER(C.c_longlong)],
    "plc_set_step_count": [_vp, C.c_longlong],
    "plc_h5_write": [C.c_char_p, _int, C.POINTER(C.c_char_p), C.POINTER(_int), C.POINTER(_int),
                     C.POINTER(C.c_longlong), C.POINTER(_vp)],
    "plc_h5_read": [C.c_char_p, C.c_char_p, _hp, C.c_size_t, C.POINTER(C.c_longlong),
                    C.POINTER(_int)],
    "plc_read_mesh_in": [C.c_char_p, _int, _hp],
    "plc_device_name": [_int, C.c_char_p, _int],
    "plc_project": [_vp],
    "plc_mean_profile": [_vp, _hp],
    "plc_gen_config_default": [_vp],
    "plc_gen_create": [_vp, _int, C.POINTER(_vp)],
    "plc_gen_destroy": [_vp],
    "plc_gen_num_params": [_vp, C.POINTER(C.c_longlong)],
    "plc_gen_get_params": [_vp, _hp],
    "plc_gen_set_params": [_vp, _hp],
    "plc_gen_set_targets": [_vp, _int, _hp, _hp],
    "plc_gen_latent": [_vp, C.c_ulonglong, _hp],
    "plc_gen_forward": [_vp, _hp, C.c_ulonglong, _hp],
    "plc_gen_output_stats": [_vp, _hp],
    "plc_gen_loss_grad": [_vp, _hp, _hp, C.c_ulonglong, C.POINTER(_dbl), _hp],
    "plc_gen_adam_step": [_vp, _dbl],
    "plc_gen_train": [_vp, _int, _dbl, C.c_ulonglong, _hp],
    "plc_gen_stats_of": [_vp, _vp, _hp],
    "plc_gen_propose": [_vp, _vp, _dbl, C.c_ulonglong],
    "plc_set_sm_budget": [_vp, _int],
    "plc_get_sm_budget": [_vp, C.POINTER(_int)],
    "plc_ensemble_create": [_int, C.POINTER(PlcParams), C.POINTER(_vp), _int, C.POINTER(_vp)],
    "plc_ensemble_destroy": [_vp],
    "plc_ensemble_size": [_vp, C.POINTER(_int)],
    "plc_ensemble_member": [_vp, _int, C.POINTER(_vp)],
    "plc_ensemble_init_flow": [_vp],
    "plc_ensemble_step": [_vp, _int],
    "plc_ensemble_step_timed": [_vp, _int, C.POINTER(_dbl)],
    "plc_ensemble_set_schedule": [_vp, _int],
    "plc_ensemble_schedule": [_vp, C.POINTER(_int), C.POINTER(_int), C.POINTER(_int)],
    "plc_ensemble_autotune": [_vp, _int, C.POINTER(C.c_float)],
    "plc_ensemble_batch_choice": [_vp, C.POINTER(_int), C.POINTER(_int), C.POINTER(_int),
                                  C.POINTER(_int)],
    "plc_ensemble_set_batch_chains": [_vp, _int],
    "plc_ensemble_set_batch_pdl": [_vp, _int],
    "plc_ensemble_batch_pdl": [_vp, C.POINTER(_int)],
    "plc_ensemble_partition": [_int, C.POINTER(_dbl), _int, C.POINTER(_int)],
    "plc_set_output_dir": [_vp, C.c_char_p],
    "plc_write_field_h5": [_vp, C.c_char_p, _int, _int],
    "plc_read_field_h5": [_vp, C.c_char_p, _int, C.POINTER(_int)],
    "plc_write_stat_h5": [_vp, C.c_char_p, _int],
    "plc_read_stat_h5": [_vp, C.c_char_p, _int, C.POINTER(_int)],
    "plc_output_mesh": [_vp],
    "plc_input_data": [_vp, C.POINTER(_int)],
    "plc_output_init": [_vp],
    "plc_output_data": [_vp, _int],
    "plc_output_free": [_vp],
    "plc_run": [_vp, _int, _int],
    "plc_kernels_per_step": [_vp, C.POINTER(_int)],
    "plc_get_stream": [_vp, C.POINTER(_vp)],
    "plc_step_timed": [_vp, _int, C.POINTER(_dbl)],
    "plc_profile_step": [_vp, _int, C.POINTER(C.c_float), C.POINTER(_int)],
    "plc_mesh_by_func": [_int, _int, _dbl, _int, _dbl, _hp],
    "plc_trid_tables": [_int, _int, _int, _dbl, _dbl, _hp, _hp, _hp, _hp],
    "plc_host_alloc": [C.c_size_t, C.POINTER(_vp)],
    "plc_host_free": [_vp],
    "plc_mean_noalloc": [_dp, _dp, _int, _int, _int, _int, _int, _dp, _vp],
}


def exported_symbols():
    """Names of the entry points this binding expects (all declared in plc.h)."""
    return sorted(list(_SIGS) + ["plc_last_error", "plc_step_kernel_name",
                                 "plc_step_kernel_name_ctx", "plc_h5_lookup3",
                                 "plc_ensemble_last_error", "plc_gen_last_error"])


def lib():
    """Load libplc.so, failing loudly when it is absent."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"libplc.so not found at {LIB_PATH}; build it with "
                "`python -c 'import powerllel_channel_sycl_b200.build as b; b.build()'`")
        L = C.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.plc_last_error.argtypes = [_vp]
        L.plc_last_error.restype = C.c_char_p
        L.plc_step_kernel_name.argtypes = [_int]
        L.plc_step_kernel_name.restype = C.c_char_p
        L.plc_step_kernel_name_ctx.argtypes = [_vp, _int]
        L.plc_step_kernel_name_ctx.restype = C.c_char_p
        L.plc_gen_last_error.argtypes = [_vp]
        L.plc_gen_last_error.restype = C.c_char_p
        L.plc_ensemble_last_error.argtypes = [_vp]
        L.plc_ensemble_last_error.restype = C.c_char_p
        L.plc_h5_lookup3.argtypes = [_vp, C.c_size_t, C.c_uint]
        L.plc_h5_lookup3.restype = C.c_uint
        _lib = L
        return L


def check(rc: int, ctx=None) -> None:
    if rc != PLC_OK:
        msg = lib().plc_last_error(ctx)
        raise PlcError(rc, msg.decode() if msg else "")
