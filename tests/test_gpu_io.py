"""Data I/O on the device fields: HDF5 field and statistics files, restart,
mesh files, the monitor text files and the main-loop driver (mod_dataIO,
outputMesh, mod_monitor, main.cc), read back with the test-side HDF5 reader."""
from __future__ import annotations

import re

import numpy as np
import pytest

from h5read import H5File
from helpers import case_kwargs, channel_params, interior, oracle_case, rel_l2

pytestmark = pytest.mark.gpu

NAMES = ("u", "v", "w", "u2", "v2", "w2", "uv", "uw", "vw", "p", "p2")


def make_channel(nx=32, ny=24, nz=16, precision=0, u_crf=0.0, **extra):
    from powerllel_channel_sycl_b200 import Channel
    prm = channel_params(**case_kwargs(nx, ny, nz, u_crf=u_crf))
    prm.precision = precision
    for key, val in extra.items():
        cur = getattr(prm, key)
        if isinstance(cur, bytes):
            setattr(prm, key, str(val).encode())
        elif hasattr(cur, "__len__"):
            for i, x in enumerate(val):
                cur[i] = x
        else:
            setattr(prm, key, val)
    return Channel(prm)


@pytest.mark.parametrize("u_crf", [0.0, 0.3])
def test_field_file_u_lab_frame(tmp_path, u_crf):
    """u is written as u + u_crf; the context's u becomes (u + u_crf) - u_crf."""
    ch = make_channel(u_crf=u_crf)
    ch.initFlow()
    ch.step(3)
    u0 = ch.download("u")
    path = tmp_path / "u.h5"
    ch.outputField(path, "u", 3)
    f = H5File(path)
    assert f.names() == ["nt", "u"]
    assert f.dataset("nt").tolist() == [3]
    got = f.dataset("u")
    assert got.shape == (16, 24, 32)
    assert np.array_equal(got, interior(u0) + u_crf)
    u1 = ch.download("u")
    assert np.array_equal(interior(u1), (interior(u0) + u_crf) - u_crf)
    halo = np.ones(u0.shape, bool)
    halo[1:-1, 1:-1, 1:-1] = False
    assert np.array_equal(u1[halo], u0[halo])  # halos untouched, as the reference's +=/-=


def test_field_file_read_keeps_halos(tmp_path):
    ch = make_channel()
    ch.initFlow()
    ch.step(2)
    v0, p0 = ch.download("v"), ch.download("p")
    ch.outputField(tmp_path / "v.h5", "v", 2)
    ch.outputField(tmp_path / "p.h5", "p", 2)
    assert np.array_equal(H5File(tmp_path / "p.h5").dataset("p"), interior(p0))
    junk = np.full(v0.shape, 7.0)
    ch.upload("v", junk)
    assert ch.inputField(tmp_path / "v.h5", "v") == 2
    v1 = ch.download("v")
    assert np.array_equal(interior(v1), interior(v0))
    assert np.all(v1[0] == 7.0) and np.all(v1[:, :, 0] == 7.0)


def test_stat_file_roundtrip(tmp_path):
    ch = make_channel(stat_which_var=[1] * 11, nt_init_stat=0, sample_interval=1)
    ch.initFlow()
    ch.initStat()
    for nt in (1, 2, 3):
        ch.step(1)
        ch.calcStat(nt)
    info = ch.stat_info
    sums = {n: ch.stat(n) for n in NAMES}
    for n in NAMES:
        ch.outputStatField(tmp_path / f"stat_{n}.h5", n)
    f = H5File(tmp_path / "stat_uv.h5")
    assert f.names() == ["nspl", "nte", "nts", "uv_stat"]
    assert [int(f.dataset(k)[0]) for k in ("nts", "nte", "nspl")] == [1, 3, 3]
    assert np.array_equal(f.dataset("uv_stat"), sums["uv"])
    ch2 = make_channel(stat_which_var=[1] * 11)
    ch2.initStat()
    for n in NAMES:
        assert ch2.inputStatField(tmp_path / f"stat_{n}.h5", n) == 3
        assert np.array_equal(ch2.stat(n), sums[n]), n
    assert ch2.stat_info == info


@pytest.mark.parametrize("u_crf", [0.0, 0.3])
def test_restart(tmp_path, u_crf):
    """save files at nt = 5, then 5 more steps, against a second context that
    restarts from the files (inputData + inputStatData) and takes the same 5."""
    common = dict(u_crf=u_crf, nt_out_save=5, overwrite_save=1, stat_which_var=[1] * 11,
                  nt_init_stat=0, sample_interval=1, nt_out_stat=0, nt_check=5,
                  cfl_limit=10.0, div_limit=1e-8)
    a = make_channel(**common)
    a.set_output_dir(tmp_path)
    a.initFlow()
    a.initStat()
    for nt in range(1, 6):
        a.step(1)
        a.calcStat(nt)
    a.outputData(5)
    # the reference versions the statistics checkpoints when overwrite_save is set
    assert (tmp_path / "save_u.h5").exists() and (tmp_path / "save_00000005_stat_u.h5").exists()
    a.step(5)
    b = make_channel(fn_prefix_input_inst=tmp_path / "save",
                     fn_prefix_input_stat=tmp_path / "save_00000005_stat", **common)
    assert b.inputData() == 5
    assert b.step_count == 5
    assert b.stat_info == {"nts": 1, "nte": 5, "nspl": 5}
    b.step(5)
    for name in "uvw":
        ua, ub = a.download(name), b.download(name)
        if u_crf == 0.0:
            assert np.array_equal(ua, ub), name
        else:
            # a's halos kept the values from before the in-place (u + u_crf) - u_crf
            # of the checkpoint write, b's were recomputed from the rounded interior
            assert rel_l2(ub, ua) < 1e-13, name
    assert np.array_equal(a.stat("uw"), b.stat("uw"))


def test_restart_timestamp_and_shape_errors(tmp_path):
    from powerllel_channel_sycl_b200 import PlcError
    a = make_channel()
    a.initFlow()
    a.outputField(tmp_path / "save_u.h5", "u", 5)
    a.outputField(tmp_path / "save_v.h5", "v", 6)
    a.outputField(tmp_path / "save_w.h5", "w", 5)
    b = make_channel(fn_prefix_input_inst=tmp_path / "save")
    with pytest.raises(PlcError) as e:
        b.inputData()
    assert e.value.code == -6 and "timestamp of <v>" in str(e.value)
    c = make_channel(nx=16, ny=24, nz=32)
    with pytest.raises(PlcError) as e:
        c.inputField(tmp_path / "save_u.h5", "u")
    assert e.value.code == -6 and "dimensions" in str(e.value)


def test_mesh_files(tmp_path):
    ch = make_channel()
    ch.set_output_dir(tmp_path)
    ch.outputMesh()
    case = oracle_case(**case_kwargs(32, 24, 16))
    f = H5File(tmp_path / "mesh_32-24-16.h5")
    assert f.names() == ["xc", "yc", "zc"]
    dx, dy = case.lx / 32, case.ly / 24
    assert np.array_equal(f.dataset("xc"), -0.5 * dx + np.arange(1, 33) * dx)
    assert np.array_equal(f.dataset("yc"), -0.5 * dy + np.arange(1, 25) * dy)
    assert np.array_equal(f.dataset("zc"), case.zc_global[1:-1])
    lines = (tmp_path / "mesh_00016.out").read_text().splitlines()
    assert lines[0] == " " * 4 + "k" + " " * 21 + "dzf" + " " * 22 + "zc"
    assert len(lines) == 17
    k, dzf, zc = lines[3].split()
    assert k == "00003" and re.fullmatch(r"\d\.\d{15}E[+-]\d\d", dzf)
    assert float(dzf) == pytest.approx(case.dzf_global[3], rel=1e-15)
    assert float(zc) == pytest.approx(case.zc_global[3], rel=1e-15)


def test_run_driver_outputs(tmp_path, capfd):
    """main.cc's loop with every output on, against plain stepping."""
    cfg = dict(nt_end=20, nt_check=5, cfl_limit=10.0, div_limit=1e-8, nt_out_scrn=10,
               nt_out_moni=5, nt_out_inst=10, nt_out_save=10, overwrite_save=0, auto_cleanup=1,
               num_retained=0, nt_init_stat=10, sample_interval=1, nt_out_stat=10,
               stat_which_var=[1] * 11, out_forcing=1, out_probe_point=1, probe_ijk=[3, 4, 5],
               out_skf_z=[1, 1], out_region=1, nt_out_region=10, region_ijk=[0, 100, 2, 5, 3, 6])
    ch = make_channel(**cfg)
    ch.set_output_dir(tmp_path)
    ch.initFlow()
    ch.outputMesh()
    ch.run(1, verbose=True)
    twin = make_channel(nt_check=5, cfl_limit=10.0, div_limit=1e-8)
    twin.initFlow()
    twin.step(20)
    for name in "uvwp":
        assert np.array_equal(ch.download(name), twin.download(name)), name
    assert ch.step_count == 20
    names = sorted(p.name for p in tmp_path.iterdir())
    expect = {"mesh_32-24-16.h5", "mesh_00016.out", "monitor_forcing.out", "monitor_probe.out",
              "monitor_skf_z1.out", "monitor_skf_z2.out", "monitor_region_00000010.h5",
              "monitor_region_00000020.h5", "save_00000020_u.h5", "save_00000020_v.h5",
              "save_00000020_w.h5", "stat_00000011-00000011_u.h5", "save_stat_u.h5"}
    expect |= {f"inst_{nt:08d}_{q}.h5" for nt in (10, 20) for q in "uvwp"}
    assert expect <= set(names), expect - set(names)
    # nt = 20 removed the versioned checkpoint of nt = 10 (num_retained = 0)
    assert "save_00000010_u.h5" not in names
    # the reference samples the statistics once, at nt_init_stat + 1
    f = H5File(tmp_path / "stat_00000011-00000011_u.h5")
    assert [int(f.dataset(k)[0]) for k in ("nts", "nte", "nspl")] == [11, 11, 1]
    inst = H5File(tmp_path / "inst_00000020_p.h5")
    assert inst.dataset("nt").tolist() == [20]
    assert np.array_equal(inst.dataset("p"), interior(ch.download("p")))
    # monitor files: headers and the last line against the monitor entry points
    lines = (tmp_path / "monitor_forcing.out").read_text().splitlines()
    assert lines[0] == f"{'nt':>9}{'u_mean':>15}{'v_mean':>15}{'w_mean':>15}"
    assert [int(x.split()[0]) for x in lines[1:]] == [5, 10, 15, 20]
    m = ch.monitor_forcing()
    assert lines[-1] == f"{20:9d}" + "".join(f"{x:15.7E}" for x in m)
    lines = (tmp_path / "monitor_probe.out").read_text().splitlines()
    assert lines[0] == "Probe point (   3,   4,   5):"
    q = ch.monitor_probe(3, 4, 5)
    assert lines[-1] == f"{20:9d}" + "".join(f"{x:15.7E}" for x in q)
    for wall in (0, 1):
        lines = (tmp_path / f"monitor_skf_z{wall + 1}.out").read_text().splitlines()
        ut, cf = ch.monitor_skf(wall)
        assert lines[0] == f"{'nt':>9}{'u_tau':>15}{'cf':>15}"
        assert lines[-1] == f"{20:9d}{ut:15.7E}{cf:15.7E}"
    reg = H5File(tmp_path / "monitor_region_00000020.h5")
    assert reg.names() == ["nt", "p", "u", "v", "w"]
    for name in "uvwp":
        got = reg.dataset(name)
        assert got.shape == (4, 4, 32)
        assert np.array_equal(got, ch.extract_region([0, 100, 2, 5, 3, 6], name)), name
    out = capfd.readouterr().out
    assert "PowerLLEL.NOTE: Simulation starts at nt =         1!" in out
    rows = [ln for ln in out.splitlines()
            if re.fullmatch(r"\s+\d+\s+\d+\.\d{3}\s+\s*\d+d\s*\d+h\s*\d+m\s*\d+s\s+"
                            r"\d\.\d{3}E[+-]\d\d\s+\d\.\d{3}E[+-]\d\d", ln)]
    assert [int(r.split()[0]) for r in rows] == [10, 20]


def test_mixed_field_files(tmp_path):
    ch = make_channel(precision=1)
    ch.initFlow()
    ch.step(2)
    w0 = ch.download("w")
    ch.outputField(tmp_path / "w.h5", "w", 2)
    got = H5File(tmp_path / "w.h5").dataset("w")
    assert np.array_equal(got, interior(w0))
    ch.upload("w", np.zeros(w0.shape))
    ch.inputField(tmp_path / "w.h5", "w")
    assert np.array_equal(interior(ch.download("w")), interior(w0))
