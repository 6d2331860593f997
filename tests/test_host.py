"""Host-side logic of libplc.so that needs no GPU: exported C ABI, param.json
reader and checks, mesh and tridiagonal tables (bit-identical to the oracle),
and the loud failure when no device is present."""
import ctypes as C
import json
import os
import re

import numpy as np
import pytest

import oracle
import powerllel_channel_sycl_b200 as plc
from powerllel_channel_sycl_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TEMPLATE = {
    "PARA": {"p_row": 1, "p_col": 1},
    "MESH": {"read_mesh": False, "mesh_type": 1, "stretch_func": 0, "stretch_ratio": 3.0,
             "nx": 128, "ny": 128, "nz": 128, "lx": 12.566370614359172, "ly": 6.283185307179586,
             "lz": 2.0},
    "TIME": {"nt_end": 1000, "dt": 1.0e-3, "nt_check": 100, "cfl_limit": 1.0, "div_limit": 1.0e-9},
    "RESTART": {"is_restart": False, "fn_prefix_input_inst": "save", "fn_prefix_input_stat": "save"},
    "PHYSICAL": {"re": 2800, "u_ref": 1.0, "l_ref": 1.0, "initial_field": "poi", "u0": 1.0,
                 "init_with_noise": True, "noise_intensity": 0.5, "smooth_wall_visc": False,
                 "u_crf": 0.0},
    "FORCE": {"is_forced": [True, False, False], "vel_force": [1.0, 0.0, 0.0]},
    "STATISTICS": {"nt_init_stat": 100000, "sample_interval": 10,
                   "stat_which_var": [True] * 11},
    "OUTPUT": {"nt_out_scrn": 100, "nt_out_inst": 100000, "nt_out_stat": 100000,
               "nt_out_save": 100000, "overwrite_save": False, "auto_cleanup": True,
               "num_retained": 0, "nt_out_moni": 100},
    "MONITOR": {"out_forcing": False, "out_probe_point": False, "probe_ijk": [64, 64, 64],
                "out_skf_z": [True, True], "out_region": False, "nt_out_region": 100,
                "region_ijk": [60, 68, 60, 68, 1, 128]},
}


def declared_functions():
    text = open(os.path.join(ROOT, "include", "plc.h")).read()
    return sorted(set(re.findall(r"^(?:int|const char \*)\s*(plc_\w+)\(", text, re.M)))


def test_every_declared_symbol_is_exported():
    L = _lib.lib()
    names = declared_functions()
    assert len(names) >= 45
    for name in names:
        assert hasattr(L, name), name
    # and the Python binding covers every declared entry point
    assert set(names) <= set(_lib.exported_symbols()), set(names) - set(_lib.exported_symbols())


def test_param_json_template(tmp_path):
    path = tmp_path / "param.json"
    path.write_text(json.dumps(TEMPLATE, indent=2))
    prm = plc.read_param_json(str(path))
    assert (prm.nx, prm.ny, prm.nz) == (128, 128, 128)
    assert prm.stretch_ratio == 3.0 and prm.mesh_type == 1 and prm.stretch_func == 0
    assert prm.lx == 12.566370614359172 and prm.dt == 1e-3 and prm.nt_check == 100
    assert prm.div_limit == 1e-9 and prm.re == 2800 and prm.initial_field == 1
    assert prm.init_with_noise == 1 and prm.noise_intensity == 0.5
    assert list(prm.is_forced) == [1, 0, 0] and list(prm.vel_force) == [1.0, 0.0, 0.0]
    assert list(prm.stat_which_var) == [1] * 11 and prm.sample_interval == 10
    assert prm.overwrite_save == 0 and prm.nt_out_moni == 100
    assert list(prm.region_ijk) == [60, 68, 60, 68, 1, 128]
    assert prm.fn_prefix_input_stat == b"save"
    assert _lib.lib().plc_params_check(C.byref(prm)) == 0


def test_param_json_missing_key_keeps_default(tmp_path):
    d = json.loads(json.dumps(TEMPLATE))
    del d["PHYSICAL"]["u_crf"]
    del d["OUTPUT"]["overwrite_save"]
    path = tmp_path / "param.json"
    path.write_text(json.dumps(d))
    prm = plc.read_param_json(str(path))
    assert prm.u_crf == 0.0 and prm.overwrite_save == 1  # mod_parameters.hh defaults


def test_param_json_missing_section_is_an_error(tmp_path):
    d = json.loads(json.dumps(TEMPLATE))
    del d["FORCE"]
    path = tmp_path / "param.json"
    path.write_text(json.dumps(d))
    with pytest.raises(plc.PlcError) as e:
        plc.read_param_json(str(path))
    assert "Problem with FORCE" in str(e.value)
    with pytest.raises(plc.PlcError):
        plc.read_param_json(str(tmp_path / "missing.json"))
    bad = tmp_path / "bad.json"
    bad.write_text("{ \"PARA\": { \"p_row\": 1, } ")
    with pytest.raises(plc.PlcError):
        plc.read_param_json(str(bad))


@pytest.mark.parametrize("kw,code", [
    (dict(nx=127), -2), (dict(nz=63), -2), (dict(nx=40), -2), (dict(ny=10), -2),
    (dict(p_row=2), -3), (dict(dt=0.0), -1), (dict(precision=2), -1),
    (dict(precision=1, nx=96, ny=18), -2), (dict(precision=1, nx=6, ny=64), -2),
    (dict(precision=1), 0), (dict(precision=0, nx=96, ny=18), 0)])
def test_param_check_errors(kw, code):
    base = dict(nx=128, ny=64, nz=64, lx=1.0, ly=1.0, lz=2.0, dt=1e-3, re=100.0, u_ref=1.0,
                l_ref=1.0)
    base.update(kw)
    prm = plc.make_params(**base)
    assert _lib.lib().plc_params_check(C.byref(prm)) == code


def test_mesh_bit_identical_to_oracle():
    for nz, ratio, func in [(64, 1.5, 0), (256, 1.8, 0), (48, 1.2, 1), (32, 0.0, 0)]:
        d = np.zeros(nz + 2)
        assert _lib.lib().plc_mesh_by_func(1, func, ratio, nz, 2.0, d.ctypes.data) == 0
        c = oracle.Case(8, 8, nz, stretch_ratio=ratio, stretch_func=func)
        np.testing.assert_array_equal(d, c.dzf_global)


@pytest.mark.parametrize("nx,ny,nz,ratio", [(32, 24, 16, 1.5), (128, 64, 64, 1.5), (48, 12, 30, 1.8),
                                            (8, 6, 2, 1.5)])
def test_pivot_table_bit_identical_to_reference_b(nx, ny, nz, ratio):
    """1/b of the table equals 1/b of the reference's pre-factored 3-D b for
    every (i, j, k) (same operations in the same order)."""
    c = oracle.Case(nx, ny, nz, stretch_ratio=ratio)
    a_ref, b_ref, c_ref = c.pivots()
    MX, MY = nx // 2 + 1, ny // 2 + 1
    rp = np.zeros(MX * MY * nz)
    a = np.zeros(nz)
    cc = np.zeros(nz)
    assert _lib.lib().plc_trid_tables(nx, ny, nz, c.lx, c.ly, c.dzf_global.ctypes.data,
                                      rp.ctypes.data, a.ctypes.data, cc.ctypes.data) == 0
    np.testing.assert_array_equal(a, a_ref)
    np.testing.assert_array_equal(cc, c_ref)
    rp = rp.reshape(nz, MY, MX)
    mx = np.array([0 if i == 0 else (nx // 2 if i == 1 else i // 2) for i in range(nx)])
    my = np.array([0 if j == 0 else (ny // 2 if j == 1 else j // 2) for j in range(ny)])
    table = rp[:, my[:, None], mx[None, :]]
    with np.errstate(divide="ignore"):
        expect = 1.0 / b_ref
    last_zero = b_ref[-1] == 0.0
    expect[-1][last_zero] = 0.0
    np.testing.assert_array_equal(table, expect)


def test_eigen_values_match_oracle():
    for n in (6, 64, 384, 768):
        np.testing.assert_array_equal(plc.get_eigen_values(1, n, n), oracle.eigen_values(n))
    with pytest.raises(plc.PlcError):
        plc.get_eigen_values(1, 8, 8, "DD")


def test_no_device_fails_loudly():
    """Without a usable GPU the product path raises; it never computes on the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(plc.PlcError) as e:
        plc.Channel(nx=16, ny=8, nz=8, lx=1.0, ly=1.0, lz=2.0, dt=1e-3, re=100.0, u_ref=1.0,
                    l_ref=1.0)
    assert e.value.code == -4


def test_ensemble_entry_points_reject_null():
    """The ensemble's schedule setters and getters check their arguments on
    the host (no device needed): a null ensemble is an argument error."""
    import ctypes as C
    from powerllel_channel_sycl_b200._lib import lib
    L = lib()
    on = C.c_int(-1)
    assert L.plc_ensemble_set_batch_pdl(None, 1) == -1
    assert L.plc_ensemble_batch_pdl(None, C.byref(on)) == -1
    assert on.value == -1
    assert L.plc_ensemble_set_batch_chains(None, 2) == -1
    assert L.plc_ensemble_batch_choice(None, None, None, None, None) == -1
    assert L.plc_ensemble_step(None, 1) == -1
