"""Host-side mirror of the reference's module interface over libplc.so.

A :class:`Channel` owns one device context (fields u, v, w, u1, v1, w1, p and
the spectral work array, the mesh, the Poisson solver state and a CUDA
stream).  Its methods carry the reference's names and argument meaning:

=====================================  ==========================================
reference (src/...)                    Channel method
=====================================  ==========================================
mod_calcVel::transform2CRF             ``transform2CRF(vel_crf, vel)``
mod_calcVel::timeIntVelRK1             ``timeIntVelRK1(u_crf, u, v, w, u1, v1, w1)``
mod_calcVel::timeIntVelRK2             ``timeIntVelRK2(u_crf, u, v, w, u1, v1, w1)``
mod_calcVel::correctVel                ``correctVel(p, u, v, w)``
mod_calcVel::forceVel                  ``forceVel(u, v, w)``
mod_calcRHS::calcRHS                   ``calcRHS(u, v, w, rhs)``
mod_updateBound::updateBoundVel        ``updateBoundVel(u_crf, u, v, w)``
mod_updateBound::imposeBCVel           ``imposeBCVel(u, v, w, u_crf)``
mod_updateBound::updateBoundP          ``updateBoundP(p)``
init/execute/free_poisson_solver       ``init_poisson_solver(...)`` etc.
execute_fft_{fwd,bwd}_{x,y}pen         ``execute_fft_fwd_xpen(p, var)`` etc.
get_eigen_values                       :func:`get_eigen_values`
mod_utils::Mean/checkNaN/calcMaxCFL/.. ``Mean(nx, ny, var)`` etc.
main.cc:116-154 (one time step)        ``step(nsteps)``
=====================================  ==========================================

Array arguments name a context field ("u", "v", "w", "u1", "v1", "w1", "p",
"spec") or are raw device addresses (int).  Failures raise
:class:`PlcError` with the library's message; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Mapping

import numpy as np

from ._lib import (FIELDS, INIT_FIELDS, PRECISION, PlcError, PlcParams, PlcValueIndex, check,
                   lib)

__all__ = ["Channel", "make_params", "read_param_json", "get_eigen_values", "PlcError"]


def make_params(**kw) -> PlcParams:
    """plc_params with the reference defaults, overridden by keyword arguments."""
    prm = PlcParams()
    check(lib().plc_params_default(C.byref(prm)))
    for key, val in kw.items():
        if key == "initial_field" and isinstance(val, str):
            val = INIT_FIELDS[val]
        if key == "precision" and isinstance(val, str):
            val = PRECISION[val]
        if not hasattr(prm, key):
            raise KeyError(f"unknown parameter {key}")
        cur = getattr(prm, key)
        if isinstance(cur, bytes):
            setattr(prm, key, val.encode() if isinstance(val, str) else val)
        elif hasattr(cur, "__len__"):
            arr = getattr(prm, key)
            for i, x in enumerate(val):
                arr[i] = x
        else:
            setattr(prm, key, val)
    return prm


def read_param_json(path: str) -> PlcParams:
    """readInputParam (mod_parameters.cc:220-260) into plc_params."""
    prm = PlcParams()
    check(lib().plc_params_default(C.byref(prm)))
    check(lib().plc_params_read_json(path.encode(), C.byref(prm)))
    return prm


def get_eigen_values(ist: int, isz: int, isz_global: int, bctype: str = "PP") -> np.ndarray:
    out = np.zeros(isz)
    check(lib().plc_get_eigen_values(ist, isz, isz_global, bctype.encode(), out.ctypes.data))
    return out


def _vi(r: PlcValueIndex):
    return r.value, (r.ig, r.jg, r.kg)


class Channel:
    """One channel case on one GPU (a plc_ctx)."""

    def __init__(self, params: PlcParams | Mapping | None = None, dzf_global=None, device: int = 0,
                 **kw):
        if params is None or isinstance(params, Mapping):
            params = make_params(**dict(params or {}), **kw)
        elif kw:
            raise TypeError("pass either a PlcParams or keyword parameters")
        self.params = params
        self._dzf = None
        if dzf_global is not None:
            self._dzf = np.ascontiguousarray(dzf_global, dtype=np.float64)
        ctx = C.c_void_p()
        rc = lib().plc_create(C.byref(params), self._dzf.ctypes.data if self._dzf is not None else None,
                              device, C.byref(ctx))
        check(rc)
        self._ctx = ctx
        self.nx, self.ny, self.nz = params.nx, params.ny, params.nz
        self.mixed = params.precision == PRECISION["mixed"]

    @classmethod
    def _wrap(cls, ctx, params: PlcParams, owner):
        """A view of a context owned elsewhere (an ensemble member)."""
        self = cls.__new__(cls)
        self.params = params
        self._dzf = None
        self._ctx = ctx
        self._owner = owner  # keeps the owner alive; close() does not destroy
        self.nx, self.ny, self.nz = params.nx, params.ny, params.nz
        self.mixed = params.precision == PRECISION["mixed"]
        return self

    # -- lifetime ---------------------------------------------------------------
    def close(self):
        if getattr(self, "_owner", None) is not None:
            self._ctx = None
            return
        if getattr(self, "_ctx", None):
            lib().plc_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc):
        check(rc, self._ctx)

    # -- memory -----------------------------------------------------------------
    @property
    def shape(self):
        return (self.nz + 2, self.ny + 2, self.nx + 2)

    @property
    def spec_shape(self):
        return (self.nz, self.ny, self.nx)

    def ptr(self, f) -> int:
        if isinstance(f, int) and f not in FIELDS.values():
            return f
        fid = FIELDS[f] if isinstance(f, str) else int(f)
        p = C.c_void_p()
        n = C.c_size_t()
        self._check(lib().plc_field_ptr(self._ctx, fid, C.byref(p), C.byref(n)))
        return p.value

    @property
    def fft_tiles(self):
        """Line pairs per tile (x forward, x backward, y) and the plan
        families of the backward x, the y and the forward x transforms chosen
        by the autotuner."""
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        self._check(lib().plc_fft_tiles(self._ctx, C.byref(a), C.byref(b), C.byref(c)))
        px, py, pxf = C.c_int(), C.c_int(), C.c_int()
        self._check(lib().plc_fft_plans(self._ctx, C.byref(px), C.byref(py)))
        self._check(lib().plc_fft_plan_x_fwd(self._ctx, C.byref(pxf)))
        return {"x_fwd": a.value, "x_bwd": b.value, "y": c.value, "plan_x": px.value,
                "plan_y": py.value, "plan_x_fwd": pxf.value}

    @property
    def rk_kchunk(self) -> int:
        """z planes per block of the RK stages chosen by the autotuner."""
        k = C.c_int()
        self._check(lib().plc_rk_kchunk(self._ctx, C.byref(k)))
        return k.value

    @property
    def rk2_carry(self) -> bool:
        """Whether the mixed form's second RK stage carries its z-face terms
        (the autotuner's choice)."""
        k = C.c_int()
        self._check(lib().plc_rk2_carry(self._ctx, C.byref(k)))
        return bool(k.value)

    def ptr_f32(self, f):
        """(device pointer, element count, row pitch) of an FP32 field of a mixed context."""
        fid = FIELDS[f] if isinstance(f, str) else int(f)
        p = C.c_void_p()
        n = C.c_size_t()
        pitch = C.c_int()
        self._check(lib().plc_field_ptr_f32(self._ctx, fid, C.byref(p), C.byref(n),
                                            C.byref(pitch)))
        return p.value, n.value, pitch.value

    def upload(self, field: str, arr: np.ndarray):
        fid = FIELDS[field]
        shape = self.spec_shape if field == "spec" else self.shape
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.shape != shape:
            raise ValueError(f"{field}: expected shape {shape}, got {a.shape}")
        self._check(lib().plc_upload(self._ctx, fid, a.ctypes.data))

    def download(self, field: str) -> np.ndarray:
        fid = FIELDS[field]
        shape = self.spec_shape if field == "spec" else self.shape
        out = np.empty(shape)
        self._check(lib().plc_download(self._ctx, fid, out.ctypes.data))
        return out

    def mesh(self, which: str) -> np.ndarray:
        ids = {"dzf_global": 0, "dzf": 1, "dzf_inv": 2, "dzc": 3, "dzc_inv": 4, "dzflzi": 5,
               "zc_global": 6}
        out = np.zeros(self.nz + 2)
        check(lib().plc_get_mesh(self._ctx, ids[which], out.ctypes.data))
        return out

    def sync(self):
        self._check(lib().plc_sync(self._ctx))

    @property
    def dt(self) -> float:
        d = C.c_double()
        self._check(lib().plc_get_dt(self._ctx, C.byref(d)))
        return d.value

    @dt.setter
    def dt(self, value: float):
        self._check(lib().plc_set_dt(self._ctx, float(value)))

    def step_forcing(self):
        """(mean, force) of the last step's bulk forcing, 3 each: the mean of
        each forced component before the forcing and vel_force - mean (a
        48-byte read of what the step computed on the device)."""
        mean = np.zeros(3)
        force = np.zeros(3)
        self._check(lib().plc_step_forcing(self._ctx, mean.ctypes.data, force.ctypes.data))
        return mean, force

    # -- mod_calcVel --------------------------------------------------------------
    def transform2CRF(self, vel_crf: float, vel="u", vel_force: float = 0.0) -> float:
        vf = C.c_double(vel_force)
        self._check(lib().plc_transform2crf(self._ctx, vel_crf, self.ptr(vel), C.byref(vf)))
        return vf.value

    def timeIntVelRK1(self, u_crf=None, u="u", v="v", w="w", u1="u1", v1="v1", w1="w1"):
        u_crf = self.params.u_crf if u_crf is None else u_crf
        self._check(lib().plc_time_int_vel_rk1(self._ctx, u_crf, self.ptr(u), self.ptr(v),
                                               self.ptr(w), self.ptr(u1), self.ptr(v1),
                                               self.ptr(w1)))

    def timeIntVelRK2(self, u_crf=None, u="u", v="v", w="w", u1="u1", v1="v1", w1="w1"):
        u_crf = self.params.u_crf if u_crf is None else u_crf
        self._check(lib().plc_time_int_vel_rk2(self._ctx, u_crf, self.ptr(u), self.ptr(v),
                                               self.ptr(w), self.ptr(u1), self.ptr(v1),
                                               self.ptr(w1)))

    def correctVel(self, p="p", u="u", v="v", w="w"):
        self._check(lib().plc_correct_vel(self._ctx, self.ptr(p), self.ptr(u), self.ptr(v),
                                          self.ptr(w)))

    def forceVel(self, u="u", v="v", w="w") -> np.ndarray:
        f = np.zeros(3)
        self._check(lib().plc_force_vel(self._ctx, self.ptr(u), self.ptr(v), self.ptr(w),
                                        f.ctypes.data))
        return f

    # -- mod_calcRHS --------------------------------------------------------------
    def calcRHS(self, u="u", v="v", w="w", rhs="p"):
        self._check(lib().plc_calc_rhs(self._ctx, self.ptr(u), self.ptr(v), self.ptr(w),
                                       self.ptr(rhs)))

    # -- mod_updateBound ------------------------------------------------------------
    def updateBoundVel(self, u_crf=None, u="u", v="v", w="w"):
        u_crf = self.params.u_crf if u_crf is None else u_crf
        self._check(lib().plc_update_bound_vel(self._ctx, u_crf, self.ptr(u), self.ptr(v),
                                               self.ptr(w)))

    def imposeBCVel(self, u="u", v="v", w="w", u_crf=None):
        u_crf = self.params.u_crf if u_crf is None else u_crf
        self._check(lib().plc_impose_bc_vel(self._ctx, self.ptr(u), self.ptr(v), self.ptr(w),
                                            u_crf))

    def updateBoundP(self, p="p"):
        self._check(lib().plc_update_bound_p(self._ctx, self.ptr(p)))

    # -- Poisson solver / FFT -------------------------------------------------------
    def init_poisson_solver(self, dzf_global=None, bctype_x="PP", bctype_y="PP", bctype_z="NN"):
        d = self.mesh("dzf_global") if dzf_global is None else np.ascontiguousarray(
            dzf_global, dtype=np.float64)
        self._check(lib().plc_init_poisson_solver(self._ctx, d.ctypes.data, bctype_x.encode(),
                                                  bctype_y.encode(), bctype_z.encode()))

    def execute_poisson_solver(self, p="p"):
        self._check(lib().plc_execute_poisson_solver(self._ctx, self.ptr(p)))

    def free_poisson_solver(self):
        self._check(lib().plc_free_poisson_solver(self._ctx))

    def solve_trid(self, var="spec"):
        self._check(lib().plc_solve_trid(self._ctx, self.ptr(var)))

    def execute_fft_fwd_xpen(self, p="p", var="spec"):
        self._check(lib().plc_fft_fwd_xpen(self._ctx, self.ptr(p), self.ptr(var)))

    def execute_fft_bwd_xpen(self, var="spec", p="p"):
        self._check(lib().plc_fft_bwd_xpen(self._ctx, self.ptr(var), self.ptr(p)))

    def execute_fft_fwd_ypen(self, var="spec"):
        self._check(lib().plc_fft_fwd_ypen(self._ctx, self.ptr(var)))

    def execute_fft_bwd_ypen(self, var="spec"):
        self._check(lib().plc_fft_bwd_ypen(self._ctx, self.ptr(var)))

    # -- mod_utils -----------------------------------------------------------------
    def Mean(self, nx_global=None, ny_global=None, var="u") -> float:
        m = C.c_double()
        self._check(lib().plc_mean(self._ctx, nx_global or self.nx, ny_global or self.ny,
                                   self.ptr(var), C.byref(m)))
        return m.value

    def checkNaN(self, var="u") -> bool:
        r = C.c_int()
        self._check(lib().plc_check_nan(self._ctx, self.ptr(var), C.byref(r)))
        return bool(r.value)

    def calcMaxCFL(self, u="u", v="v", w="w"):
        r = PlcValueIndex()
        self._check(lib().plc_calc_max_cfl(self._ctx, self.ptr(u), self.ptr(v), self.ptr(w),
                                           C.byref(r)))
        return _vi(r)

    def calcMaxDiv(self, u="u", v="v", w="w"):
        r = PlcValueIndex()
        self._check(lib().plc_calc_max_div(self._ctx, self.ptr(u), self.ptr(v), self.ptr(w),
                                           C.byref(r)))
        return _vi(r)

    # -- initial field and the fused step -------------------------------------------
    # -- mod_statistics -----------------------------------------------------------
    STAT_NAMES = ("u", "v", "w", "u2", "v2", "w2", "uv", "uw", "vw", "p", "p2")

    def initStat(self):
        """allocStat + initStat: zeroed sums of the statistics enabled by stat_which_var."""
        self._check(lib().plc_stat_init(self._ctx))

    def freeStat(self):
        self._check(lib().plc_stat_free(self._ctx))

    def calcStat(self, nt: int):
        """calcStat: one sample when (nt - nt_init_stat) % sample_interval == 0."""
        self._check(lib().plc_calc_stat(self._ctx, int(nt)))

    @property
    def stat_info(self):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        self._check(lib().plc_stat_info(self._ctx, C.byref(a), C.byref(b), C.byref(c)))
        return {"nts": a.value, "nte": b.value, "nspl": c.value}

    def stat(self, which) -> np.ndarray:
        """A running sum, (nz, ny, nx)."""
        q = self.STAT_NAMES.index(which) if isinstance(which, str) else int(which)
        out = np.empty((self.nz, self.ny, self.nx))
        self._check(lib().plc_stat_download(self._ctx, q, out.ctypes.data))
        return out

    def set_stat(self, which, arr, nts: int, nte: int, nspl: int):
        q = self.STAT_NAMES.index(which) if isinstance(which, str) else int(which)
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.shape != (self.nz, self.ny, self.nx):
            raise ValueError("statistic arrays are (nz, ny, nx)")
        self._check(lib().plc_stat_upload(self._ctx, q, a.ctypes.data, nts, nte, nspl))

    def stat_profiles(self) -> dict:
        """Plane means of each statistic divided by the samples, name -> (nz,)."""
        out = np.zeros((len(self.STAT_NAMES), self.nz))
        self._check(lib().plc_stat_profiles(self._ctx, out.ctypes.data))
        return dict(zip(self.STAT_NAMES, out))

    # -- mod_monitor --------------------------------------------------------------
    def monitor_forcing(self) -> np.ndarray:
        out = np.zeros(3)
        self._check(lib().plc_monitor_forcing(self._ctx, out.ctypes.data))
        return out

    def monitor_probe(self, ig: int, jg: int, kg: int) -> np.ndarray:
        """u + u_crf, v, w, p at the 1-based interior point."""
        out = np.zeros(4)
        self._check(lib().plc_monitor_probe(self._ctx, ig, jg, kg, out.ctypes.data))
        return out

    def monitor_skf(self, wall: int = 0):
        """(u_tau, cf) at the bottom (0) or top (1) wall."""
        ut, cf = C.c_double(), C.c_double()
        self._check(lib().plc_monitor_skf(self._ctx, wall, C.byref(ut), C.byref(cf)))
        return ut.value, cf.value

    def re_tau(self) -> float:
        """Friction Reynolds number u_tau * h / nu from both walls' u_tau, h = lz/2."""
        ut = 0.5 * (self.monitor_skf(0)[0] + self.monitor_skf(1)[0])
        nu = self.params.u_ref * self.params.l_ref / self.params.re  # re_inv
        return ut * (0.5 * self.params.lz) / nu

    def extract_region(self, region_ijk, field: str = "u") -> np.ndarray:
        """The box {i0,i1,j0,j1,k0,k1} (1-based, clipped), shape (nk, nj, ni)."""
        r = [int(x) for x in region_ijk]
        r[0], r[1] = max(r[0], 1), min(r[1], self.nx)
        r[2], r[3] = max(r[2], 1), min(r[3], self.ny)
        r[4], r[5] = max(r[4], 1), min(r[5], self.nz)
        out = np.zeros((r[5] - r[4] + 1, r[3] - r[2] + 1, r[1] - r[0] + 1))
        arr = (C.c_int * 6)(*r)
        self._check(lib().plc_extract_region(self._ctx, arr, FIELDS[field], out.ctypes.data))
        return out

    def initFlow(self):
        self._check(lib().plc_init_flow(self._ctx))

    def project(self):
        """Makes u, v, w divergence-free with the solver's own projection."""
        self._check(lib().plc_project(self._ctx))

    def mean_profile(self) -> np.ndarray:
        """Plane means of u + u_crf, k = 1..nz."""
        out = np.empty(self.nz)
        self._check(lib().plc_mean_profile(self._ctx, out.ctypes.data))
        return out

    def finish_input(self):
        """transform2CRF and the boundary update after uploading u, v, w (main.cc:77-82)."""
        self._check(lib().plc_finish_input(self._ctx))

    @property
    def step_count(self) -> int:
        n = C.c_longlong()
        self._check(lib().plc_step_count(self._ctx, C.byref(n)))
        return n.value

    @step_count.setter
    def step_count(self, n: int):
        self._check(lib().plc_set_step_count(self._ctx, int(n)))

    @property
    def sm_budget(self) -> int:
        n = C.c_int()
        self._check(lib().plc_get_sm_budget(self._ctx, C.byref(n)))
        return n.value

    @sm_budget.setter
    def sm_budget(self, sms: int):
        self._check(lib().plc_set_sm_budget(self._ctx, int(sms)))

    # ---- data I/O (mod_dataIO, outputMesh, mod_monitor files, main loop) ----
    def set_output_dir(self, path):
        self._check(lib().plc_set_output_dir(self._ctx, os.fsencode(str(path))))

    def outputField(self, path, field: str, nt: int):
        """HDF5 file of one field (u in the lab frame, as outputData writes it)."""
        self._check(lib().plc_write_field_h5(self._ctx, os.fsencode(str(path)), FIELDS[field], int(nt)))

    def inputField(self, path, field: str) -> int:
        """Reads a field file into the field's interior; returns its nt."""
        nt = C.c_int()
        self._check(lib().plc_read_field_h5(self._ctx, os.fsencode(str(path)), FIELDS[field],
                                            C.byref(nt)))
        return nt.value

    def outputStatField(self, path, which):
        q = self.STAT_NAMES.index(which) if isinstance(which, str) else int(which)
        self._check(lib().plc_write_stat_h5(self._ctx, os.fsencode(str(path)), q))

    def inputStatField(self, path, which) -> int:
        """Reads a statistics file (sum and nts/nte/nspl); returns nte."""
        q = self.STAT_NAMES.index(which) if isinstance(which, str) else int(which)
        nte = C.c_int()
        self._check(lib().plc_read_stat_h5(self._ctx, os.fsencode(str(path)), q, C.byref(nte)))
        return nte.value

    def outputMesh(self):
        self._check(lib().plc_output_mesh(self._ctx))

    def inputData(self) -> int:
        """Restart from <fn_prefix_input_inst>_{u,v,w}.h5 (and statistics); returns nt_in."""
        nt = C.c_int()
        self._check(lib().plc_input_data(self._ctx, C.byref(nt)))
        return nt.value

    def initMonitor(self):
        self._check(lib().plc_output_init(self._ctx))

    def outputData(self, nt: int):
        self._check(lib().plc_output_data(self._ctx, int(nt)))

    def freeMonitor(self):
        self._check(lib().plc_output_free(self._ctx))

    def run(self, nt_start: int = 1, verbose: bool = False):
        """The main loop of main.cc for nt_start..nt_end with checks, statistics and outputs."""
        self._check(lib().plc_run(self._ctx, int(nt_start), 1 if verbose else 0))

    def step(self, nsteps: int = 1):
        self._check(lib().plc_step(self._ctx, int(nsteps)))

    def step_timed(self, nsteps: int) -> float:
        """Run nsteps fused steps; returns their device time in ms (CUDA events)."""
        ms = C.c_double()
        self._check(lib().plc_step_timed(self._ctx, int(nsteps), C.byref(ms)))
        return ms.value

    def check(self):
        ok = C.c_int()
        c, d = PlcValueIndex(), PlcValueIndex()
        self._check(lib().plc_check(self._ctx, C.byref(ok), C.byref(c), C.byref(d)))
        return bool(ok.value), _vi(c), _vi(d)

    def last_check(self):
        ok = C.c_int()
        c, d = PlcValueIndex(), PlcValueIndex()
        self._check(lib().plc_last_check(self._ctx, C.byref(ok), C.byref(c), C.byref(d)))
        return bool(ok.value), _vi(c), _vi(d)

    @property
    def stream(self) -> int:
        """The context's cudaStream_t as an integer handle."""
        h = C.c_void_p()
        self._check(lib().plc_get_stream(self._ctx, C.byref(h)))
        return h.value or 0

    def profile_step(self, nsteps: int = 1):
        """Per-kernel device time (ms, summed over nsteps) of the fused step."""
        ms = (C.c_float * 16)()
        n = C.c_int()
        self._check(lib().plc_profile_step(self._ctx, int(nsteps), ms, C.byref(n)))
        return {lib().plc_step_kernel_name_ctx(self._ctx, i).decode(): float(ms[i])
                for i in range(n.value)}

    @property
    def kernels_per_step(self) -> int:
        n = C.c_int()
        self._check(lib().plc_kernels_per_step(self._ctx, C.byref(n)))
        return n.value
