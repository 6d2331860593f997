"""CPU oracle for the PowerLLEL_Channel DNS time step (test infrastructure).

This package wraps ``oracle/_build/liboracle.so`` (a plain FP64 C++
restatement of the reference hot path, see ``oracle.h``) for the tests,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``.  It is
the checker, never the product: the product library in
``powerllel_channel_sycl_b200`` neither imports nor links it.

Parity status: parity unpinned (the reference ships no golden vectors and
cannot be built here); the restatement is checked against numpy/scipy and
analytic invariants in ``tests/test_oracle_*.py``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lock = threading.Lock()
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


class OrcGrid(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
        ("dx", C.c_double), ("dy", C.c_double),
        ("dx_inv", C.c_double), ("dy_inv", C.c_double),
        ("dt", C.c_double), ("re_inv", C.c_double), ("u_crf", C.c_double),
        ("is_forced", C.c_int * 3), ("vel_force", C.c_double * 3),
        ("dzf", C.POINTER(C.c_double)), ("dzf_inv", C.POINTER(C.c_double)),
        ("dzc_inv", C.POINTER(C.c_double)), ("dzflzi", C.POINTER(C.c_double)),
    ]


class OrcValueIndex(C.Structure):
    _fields_ = [("value", C.c_double), ("ig", C.c_int), ("jg", C.c_int), ("kg", C.c_int)]


def build() -> str:
    """Compile the oracle library with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        G = C.POINTER(OrcGrid)
        vp = C.c_void_p
        sig = {
            "orc_mesh_by_func": (None, [C.c_int, C.c_int, C.c_double, C.c_int, C.c_double, _dp]),
            "orc_mesh_derived": (None, [C.c_int, C.c_double, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
            "orc_transform2crf": (None, [G, C.c_double, _dp, C.POINTER(C.c_double)]),
            "orc_time_int_vel_rk1": (None, [G, C.c_double, _dp, _dp, _dp, _dp, _dp, _dp]),
            "orc_time_int_vel_rk2": (None, [G, C.c_double, _dp, _dp, _dp, _dp, _dp, _dp]),
            "orc_correct_vel": (None, [G, _dp, _dp, _dp, _dp]),
            "orc_force_vel": (None, [G, _dp, _dp, _dp, _dp]),
            "orc_calc_rhs": (None, [G, _dp, _dp, _dp, _dp]),
            "orc_update_bound_vel": (None, [G, C.c_double, _dp, _dp, _dp]),
            "orc_update_bound_p": (None, [G, _dp]),
            "orc_mean": (C.c_double, [G, C.c_int, C.c_int, _dp]),
            "orc_check_nan": (C.c_int, [G, _dp]),
            "orc_calc_max_cfl": (None, [G, _dp, _dp, _dp, C.POINTER(OrcValueIndex)]),
            "orc_calc_max_div": (None, [G, _dp, _dp, _dp, C.POINTER(OrcValueIndex)]),
            "orc_rfft_packed": (None, [C.c_int, _dp, _dp]),
            "orc_irfft_packed": (None, [C.c_int, _dp, _dp]),
            "orc_get_eigen_values": (None, [C.c_int, C.c_int, C.c_int, _dp]),
            "orc_poisson_init": (vp, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _dp]),
            "orc_poisson_free": (None, [vp]),
            "orc_poisson_work": (C.POINTER(C.c_double), [vp]),
            "orc_poisson_b": (C.POINTER(C.c_double), [vp]),
            "orc_poisson_a": (C.POINTER(C.c_double), [vp]),
            "orc_poisson_c": (C.POINTER(C.c_double), [vp]),
            "orc_fft_fwd_xpen": (None, [vp, _dp, _dp]),
            "orc_fft_bwd_xpen": (None, [vp, _dp, _dp]),
            "orc_fft_fwd_ypen": (None, [vp, _dp]),
            "orc_fft_bwd_ypen": (None, [vp, _dp]),
            "orc_ssolve_trid": (None, [vp, _dp]),
            "orc_poisson_execute": (None, [vp, _dp]),
            "orc_noise_uniform": (C.c_double, [C.c_int, C.c_longlong]),
            "orc_init_flow": (None, [G, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                                     C.c_double, _dp, _dp, _dp, _dp]),
            "orc_step": (None, [G, vp, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
            "orc_run_cfl": (None, [G, vp, C.c_int, C.c_int, C.c_double, _dp, _dp, _dp, _dp,
                                   _dp, _dp, _dp, _dp]),
            "orc_calc_stat_sample": (None, [G, C.c_double, _dp, _dp, _dp, _dp,
                                            C.POINTER(C.c_void_p)]),
            "orc_wall_tau": (C.c_double, [G, C.c_int, C.c_double, _dp, C.c_double]),
            "orc_extract_region": (None, [G, _dp, C.c_int, C.POINTER(C.c_int),
                                          C.POINTER(C.c_int), _dp]),
            "orc_set_threads": (None, [C.c_int]),
            "orc_get_threads": (C.c_int, []),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
        return L


INITIAL_FIELDS = {"uni": 0, "poi": 1, "log": 2}


class Case:
    """A channel case on the host: parameters, mesh, fields and Poisson state.

    Field arrays are numpy float64 arrays of shape (nz+2, ny+2, nx+2), i.e.
    the reference's halo'd layout with x fastest.
    """

    def __init__(self, nx, ny, nz, lx=4 * np.pi, ly=2 * np.pi, lz=2.0, dt=2e-3, re=2800.0,
                 u_ref=1.0, l_ref=1.0, mesh_type=1, stretch_func=0, stretch_ratio=1.5,
                 u_crf=0.0, is_forced=(True, False, False), vel_force=(1.0, 0.0, 0.0),
                 dzf_global=None):
        L = lib()
        self.nx, self.ny, self.nz = nx, ny, nz
        self.lx, self.ly, self.lz = lx, ly, lz
        self.dt, self.re, self.u_ref, self.l_ref = dt, re, u_ref, l_ref
        self.u_crf = u_crf
        self.is_forced = tuple(bool(x) for x in is_forced)
        self.vel_force = tuple(float(x) for x in vel_force)
        if dzf_global is None:
            dzf_global = np.zeros(nz + 2)
            L.orc_mesh_by_func(mesh_type, stretch_func, stretch_ratio, nz, lz, dzf_global)
        self.dzf_global = np.ascontiguousarray(dzf_global, dtype=np.float64)
        self.dzf = np.zeros(nz + 2)
        self.dzf_inv = np.zeros(nz + 2)
        self.dzc = np.zeros(nz + 2)
        self.dzc_inv = np.zeros(nz + 2)
        self.dzflzi = np.zeros(nz + 2)
        self.zc_global = np.zeros(nz + 2)
        L.orc_mesh_derived(nz, lz, self.dzf_global, self.dzf, self.dzf_inv, self.dzc,
                           self.dzc_inv, self.dzflzi, self.zc_global)
        g = OrcGrid()
        g.nx, g.ny, g.nz = nx, ny, nz
        g.lx, g.ly, g.lz = lx, ly, lz
        g.dx = lx / nx
        g.dy = ly / ny
        g.dx_inv = 1.0 / g.dx
        g.dy_inv = 1.0 / g.dy
        g.dt = dt
        g.re_inv = u_ref * l_ref / re  # mod_parameters.cc:259
        g.u_crf = u_crf
        for d in range(3):
            g.is_forced[d] = int(self.is_forced[d])
            g.vel_force[d] = self.vel_force[d]
        dptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
        g.dzf, g.dzf_inv, g.dzc_inv, g.dzflzi = (dptr(self.dzf), dptr(self.dzf_inv),
                                                 dptr(self.dzc_inv), dptr(self.dzflzi))
        self.g = g
        self._ps = None

    # -- shapes ---------------------------------------------------------------
    @property
    def shape(self):
        return (self.nz + 2, self.ny + 2, self.nx + 2)

    def zeros(self):
        return np.zeros(self.shape)

    @property
    def gp(self):
        return C.byref(self.g)

    # -- Poisson state ----------------------------------------------------------
    @property
    def ps(self):
        if self._ps is None:
            self._ps = lib().orc_poisson_init(self.nx, self.ny, self.nz, self.g.dx, self.g.dy,
                                              self.dzf_global)
        return self._ps

    def __del__(self):
        try:
            if self._ps is not None:
                lib().orc_poisson_free(self._ps)
        except Exception:
            pass

    def pivots(self):
        """Pre-factored 3-D diagonal b (nz, ny, nx) and 1-D a, c (nz)."""
        n = self.nx * self.ny * self.nz
        L = lib()
        b = np.ctypeslib.as_array(L.orc_poisson_b(self.ps), shape=(n,)).copy()
        a = np.ctypeslib.as_array(L.orc_poisson_a(self.ps), shape=(self.nz,)).copy()
        c = np.ctypeslib.as_array(L.orc_poisson_c(self.ps), shape=(self.nz,)).copy()
        return a, b.reshape(self.nz, self.ny, self.nx), c

    # -- initial field ----------------------------------------------------------
    def init_flow(self, initial_field="poi", u0=1.0, init_with_noise=True,
                  noise_intensity=0.1):
        u, v, w = self.zeros(), self.zeros(), self.zeros()
        lib().orc_init_flow(self.gp, INITIAL_FIELDS[initial_field], u0, self.u_ref, self.re,
                            int(init_with_noise), noise_intensity, self.zc_global, u, v, w)
        # main.cc:78-82
        vf = C.c_double(self.vel_force[0])
        lib().orc_transform2crf(self.gp, self.u_crf, u, C.byref(vf))
        self.update_bound_vel(u, v, w)
        return u, v, w

    # -- module functions -------------------------------------------------------
    def rk1(self, u, v, w, u1, v1, w1):
        lib().orc_time_int_vel_rk1(self.gp, self.u_crf, u, v, w, u1, v1, w1)

    def rk2(self, u, v, w, u1, v1, w1):
        lib().orc_time_int_vel_rk2(self.gp, self.u_crf, u, v, w, u1, v1, w1)

    def calc_rhs(self, u, v, w, p):
        lib().orc_calc_rhs(self.gp, u, v, w, p)

    def correct_vel(self, p, u, v, w):
        lib().orc_correct_vel(self.gp, p, u, v, w)

    def force_vel(self, u, v, w):
        f = np.zeros(3)
        lib().orc_force_vel(self.gp, u, v, w, f)
        return f

    def update_bound_vel(self, u, v, w):
        lib().orc_update_bound_vel(self.gp, self.u_crf, u, v, w)

    def update_bound_p(self, p):
        lib().orc_update_bound_p(self.gp, p)

    def mean(self, var, nxg=None, nyg=None):
        return lib().orc_mean(self.gp, nxg or self.nx, nyg or self.ny, var)

    def poisson(self, p):
        lib().orc_poisson_execute(self.ps, p)

    def fft_fwd_x(self, p, var):
        lib().orc_fft_fwd_xpen(self.ps, p, var)

    def fft_bwd_x(self, var, p):
        lib().orc_fft_bwd_xpen(self.ps, var, p)

    def fft_fwd_y(self, var):
        lib().orc_fft_fwd_ypen(self.ps, var)

    def fft_bwd_y(self, var):
        lib().orc_fft_bwd_ypen(self.ps, var)

    def trid(self, var):
        lib().orc_ssolve_trid(self.ps, var)

    def max_cfl(self, u, v, w):
        r = OrcValueIndex()
        lib().orc_calc_max_cfl(self.gp, u, v, w, C.byref(r))
        return r.value, (r.ig, r.jg, r.kg)

    def max_div(self, u, v, w):
        r = OrcValueIndex()
        lib().orc_calc_max_div(self.gp, u, v, w, C.byref(r))
        return r.value, (r.ig, r.jg, r.kg)

    def check_nan(self, var):
        return bool(lib().orc_check_nan(self.gp, var))

    def calc_stat_sample(self, u, v, w, p, sums, u_crf=None):
        """One calcStat sample into sums: a list of 11 arrays (nz, ny, nx) or None."""
        ptrs = (C.c_void_p * 11)(*[None if a is None else a.ctypes.data for a in sums])
        lib().orc_calc_stat_sample(self.gp, self.u_crf if u_crf is None else u_crf,
                                   u, v, w, p, ptrs)

    def wall_tau(self, vel, k_wall, vel_crf=None):
        """calcAndWriteSkf's tau_w at k_wall (1 or nz), dz = dzf(k_wall)/2."""
        dz = 0.5 * self.dzf[k_wall]
        return lib().orc_wall_tau(self.gp, k_wall, dz, vel,
                                  self.u_crf if vel_crf is None else vel_crf)

    def extract_region(self, var, offset_dir, reg_st, reg_sz):
        out = np.zeros((reg_sz[2], reg_sz[1], reg_sz[0]))
        st = (C.c_int * 3)(*reg_st)
        sz = (C.c_int * 3)(*reg_sz)
        lib().orc_extract_region(self.gp, var, offset_dir, st, sz, out)
        return out

    def step(self, u, v, w, u1, v1, w1, p, nsteps=1):
        lib().orc_step(self.gp, self.ps, nsteps, u, v, w, u1, v1, w1, p)

    def run_cfl(self, u, v, w, u1, v1, w1, p, nsteps, nt_check, cfl_target):
        """nsteps of main.cc's loop with the CFL-controlled dt; returns the dt
        of every step followed by the dt the next step would use."""
        dts = np.zeros(nsteps + 1)
        lib().orc_run_cfl(self.gp, self.ps, nsteps, nt_check, cfl_target, u, v, w, u1, v1, w1,
                          p, dts)
        return dts


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def get_threads() -> int:
    return int(lib().orc_get_threads())


def rfft_packed(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros_like(x)
    lib().orc_rfft_packed(x.size, x, out)
    return out


def irfft_packed(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros_like(x)
    lib().orc_irfft_packed(x.size, x, out)
    return out


def eigen_values(n):
    lam = np.zeros(n)
    lib().orc_get_eigen_values(1, n, n, lam)
    return lam
