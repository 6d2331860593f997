"""plc_main, the solver as a program in place of the reference's executable:
param.json in the working directory, mesh files, checkpoints, monitors, and
a restart from the checkpoint files that reproduces the uninterrupted run."""
from __future__ import annotations

import json
import os
import shutil
import subprocess

import numpy as np
import pytest

from h5read import H5File
from test_host import TEMPLATE

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROGRAM = os.path.join(ROOT, "powerllel_channel_sycl_b200", "lib", "plc_main")


def params(**over):
    d = json.loads(json.dumps(TEMPLATE))
    d["MESH"].update(nx=32, ny=24, nz=16, stretch_ratio=1.5)
    d["TIME"].update(nt_end=20, nt_check=5, dt=2e-3)
    d["PHYSICAL"].update(noise_intensity=0.1)
    d["OUTPUT"].update(nt_out_scrn=10, nt_out_inst=20, nt_out_save=10, overwrite_save=False,
                       auto_cleanup=True, num_retained=1, nt_out_moni=5)
    d["MONITOR"].update(out_forcing=True, out_probe_point=True, probe_ijk=[4, 5, 6],
                        out_skf_z=[True, True], out_region=False)
    for sec, kv in over.items():
        d[sec].update(kv)
    return d


def run(cwd, prm):
    (cwd / "param.json").write_text(json.dumps(prm, indent=2))
    r = subprocess.run([PROGRAM], cwd=cwd, capture_output=True, text=True, timeout=300)
    return r


def test_program_run_and_restart(tmp_path):
    first = tmp_path / "first"
    first.mkdir()
    r = run(first, params())
    assert r.returncode == 0, r.stdout + r.stderr
    assert "PowerLLEL.NOTE: Simulation ends successfully!" in r.stdout
    assert "Selected device is: CUDA, " in r.stdout
    names = set(os.listdir(first))
    assert {"mesh_32-24-16.h5", "mesh_00016.out", "monitor_forcing.out", "monitor_probe.out",
            "monitor_skf_z1.out", "monitor_skf_z2.out", "save_00000010_u.h5",
            "save_00000020_w.h5", "inst_00000020_p.h5"} <= names
    # the same run through the library's Python interface
    from powerllel_channel_sycl_b200 import Channel, read_param_json
    ch = Channel(read_param_json(str(first / "param.json")))
    ch.initFlow()
    ch.step(20)
    for q in "uvw":
        got = H5File(first / f"save_00000020_{q}.h5").dataset(q)
        assert np.array_equal(got, ch.download(q)[1:-1, 1:-1, 1:-1]), q
    lines = (first / "monitor_forcing.out").read_text().splitlines()
    assert len(lines) == 5 and lines[-1].split()[0] == "20"

    # restart from the checkpoint of nt = 10 in another directory
    second = tmp_path / "second"
    second.mkdir()
    for q in "uvw":
        shutil.copy(first / f"save_00000010_{q}.h5", second)
    r = run(second, params(RESTART={"is_restart": True, "fn_prefix_input_inst": "save_00000010"}))
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Simulation starts at nt =        11!" in r.stdout
    for q in "uvw":
        a = H5File(first / f"save_00000020_{q}.h5").dataset(q)
        b = H5File(second / f"save_00000020_{q}.h5").dataset(q)
        assert np.array_equal(a, b), q


def test_program_read_mesh_and_errors(tmp_path):
    dzf = np.linspace(0.5, 1.5, 16)
    dzf *= 2.0 / dzf.sum()
    (tmp_path / "mesh.in").write_text("\n".join(f"{x:.17e}" for x in dzf) + "\n")
    r = run(tmp_path, params(MESH={"read_mesh": True}, TIME={"nt_end": 2}))
    assert r.returncode == 0, r.stdout + r.stderr
    rows = (tmp_path / "mesh_00016.out").read_text().splitlines()[1:]
    assert np.allclose([float(x.split()[1]) for x in rows], dzf, rtol=1e-15, atol=0)
    # a restart whose checkpoint is missing stops like the reference
    r = run(tmp_path, params(RESTART={"is_restart": True, "fn_prefix_input_inst": "none"}))
    assert r.returncode == 1
    assert "none_u.h5 doesn't exist" in r.stderr
    # a failed divergence check stops the run
    r = run(tmp_path, params(TIME={"div_limit": 1e-300, "nt_end": 5}))
    assert r.returncode == 1 and "checkDiv" in r.stderr
