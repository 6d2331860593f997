"""The reference's own time-step modules, run on the CPU -- TEST INFRASTRUCTURE ONLY.

``oracle/_ref/libplcref.so`` is built by ``oracle/reference_cpu/Makefile``
from the reference's unmodified sources (src/mod_calcVel.cc, mod_calcRHS.cc,
mod_updateBound.cc, mod_utils.cc, mod_fft.cc, mod_poisson_solver.cc,
mod_mesh.cc, mod_initFlow.cc, mod_mpi.cc, mod_variables.cc, decomp_2d.cc)
compiled against host stand-ins for SYCL, one-rank MPI, the oneMKL DFT,
oneDPL's minstd engine and {fmt} (``oracle/reference_cpu/shim``).  The
tests use it to pin the oracle restatement (``oracle.Case``) to the
reference's own code.  The reference keeps its state in module globals, so
one ``ReferenceModules`` instance is live at a time; creating another frees
the previous one.

Fields are numpy float64 arrays of shape (nz+2, ny+2, nx+2), the reference's
halo'd layout with x fastest.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libplcref.so")
REF_SRC = os.environ.get("PLC_REFERENCE_SRC", "/root/reference/src")

FIELDS = {"u": 0, "v": 1, "w": 2, "u1": 3, "v1": 4, "w1": 5, "p": 6}
MESH = {"dzf_global": 0, "dzf": 1, "dzf_inv": 2, "dzc": 3, "dzc_inv": 4, "dzflzi": 5,
        "zc_global": 6, "visc_dzf_inv": 7}
INITIAL_FIELDS = {"uni": 0, "poi": 1, "log": 2}

_lock = threading.Lock()
_lib = None
_live = None


class _quiet_stdout:
    """Sends the reference's progress notes (fmt::print to stdout, e.g.
    outputMesh's "Finish writing file" lines) to /dev/null while a call
    runs, so that a caller's own stdout (a benchmark's JSON line) stays clean."""

    def __enter__(self):
        self._libc = C.CDLL(None)
        self._libc.fflush(None)
        self._saved = os.dup(1)
        self._null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self._null, 1)
        return self

    def __exit__(self, *exc):
        self._libc.fflush(None)
        os.dup2(self._saved, 1)
        os.close(self._saved)
        os.close(self._null)
        return False


def available() -> bool:
    """True when the reference build exists (or can be made from the sources here)."""
    if os.path.exists(LIB_PATH):
        return True
    return os.path.isdir(REF_SRC)


def build() -> None:
    """Compile the reference modules when their sources are present."""
    if not os.path.isdir(REF_SRC):
        return
    subprocess.run(["make", "-s", "-C", os.path.join(HERE, "reference_cpu"),
                    f"REF_SRC={REF_SRC}"], check=True)


def lib():
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
        ip = C.POINTER(C.c_int)
        d = C.c_double
        sig = {
            "ref_set_threads": (None, [C.c_int]),
            "ref_init": (None, [C.c_int, C.c_int, C.c_int, d, d, d, C.c_int, C.c_int, d, d, d, d,
                                d, d, ip, C.POINTER(C.c_double)]),
            "ref_free": (None, []),
            "ref_set_dt": (None, [d]),
            "ref_set_field": (None, [C.c_int, dp]),
            "ref_get_field": (None, [C.c_int, dp]),
            "ref_get_mesh": (None, [C.c_int, dp, dp]),
            "ref_time_int_vel_rk1": (None, []),
            "ref_time_int_vel_rk2": (None, []),
            "ref_update_bound_vel": (None, [C.c_int]),
            "ref_update_bound_p": (None, []),
            "ref_calc_rhs": (None, []),
            "ref_poisson": (None, []),
            "ref_correct_vel": (None, []),
            "ref_force_vel": (None, []),
            "ref_transform2crf": (None, [C.c_int, d, C.POINTER(C.c_double)]),
            "ref_mean": (d, [C.c_int, C.c_int, C.c_int]),
            "ref_check_nan": (C.c_int, [C.c_int]),
            "ref_calc_max_cfl": (None, [C.POINTER(C.c_double), ip]),
            "ref_calc_max_div": (None, [C.POINTER(C.c_double), ip]),
            "ref_fft_fwd_x": (None, [dp]),
            "ref_fft_bwd_x": (None, [dp]),
            "ref_fft_fwd_y": (None, [dp]),
            "ref_fft_bwd_y": (None, [dp]),
            "ref_ssolve_trid": (None, [dp]),
            "ref_eigen_values": (None, [C.c_int, dp]),
            "ref_init_flow": (None, [C.c_int, d, C.c_int, d]),
            "ref_vel_force": (d, [C.c_int]),
            "ref_step": (None, [C.c_int]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
        return L


def set_threads(n: int) -> None:
    lib().ref_set_threads(int(n))


class ReferenceModules:
    """The reference's modules set up for one channel case (main.cc:36-61)."""

    def __init__(self, nx, ny, nz, lx=4 * np.pi, ly=2 * np.pi, lz=2.0, dt=2e-3, re=2800.0,
                 u_ref=1.0, l_ref=1.0, mesh_type=1, stretch_func=0, stretch_ratio=1.5,
                 u_crf=0.0, is_forced=(True, False, False), vel_force=(1.0, 0.0, 0.0)):
        global _live
        L = lib()
        if _live is not None:
            _live.close()
        self.nx, self.ny, self.nz = nx, ny, nz
        forced = (C.c_int * 3)(*[int(bool(x)) for x in is_forced])
        vf = (C.c_double * 3)(*[float(x) for x in vel_force])
        with _quiet_stdout():
            L.ref_init(nx, ny, nz, lx, ly, lz, mesh_type, stretch_func, stretch_ratio, re, u_ref,
                       l_ref, dt, u_crf, forced, vf)
        self._open = True
        _live = self

    def close(self):
        global _live
        if self._open:
            lib().ref_free()
            self._open = False
            if _live is self:
                _live = None

    @property
    def shape(self):
        return (self.nz + 2, self.ny + 2, self.nx + 2)

    def set(self, name, arr):
        lib().ref_set_field(FIELDS[name], np.ascontiguousarray(arr, dtype=np.float64))

    def get(self, name):
        out = np.zeros(self.shape)
        lib().ref_get_field(FIELDS[name], out)
        return out

    def mesh(self, name):
        out = np.zeros(self.nz + 2)
        dxy = np.zeros(4)
        lib().ref_get_mesh(MESH[name], out, dxy)
        return out

    def dxy(self):
        out = np.zeros(self.nz + 2)
        dxy = np.zeros(4)
        lib().ref_get_mesh(0, out, dxy)
        return dxy

    def set_dt(self, dt):
        lib().ref_set_dt(dt)

    # module functions on the module's own fields
    def rk1(self):
        lib().ref_time_int_vel_rk1()

    def rk2(self):
        lib().ref_time_int_vel_rk2()

    def update_bound_vel(self, which=0):
        lib().ref_update_bound_vel(which)

    def update_bound_p(self):
        lib().ref_update_bound_p()

    def calc_rhs(self):
        lib().ref_calc_rhs()

    def poisson(self):
        lib().ref_poisson()

    def correct_vel(self):
        lib().ref_correct_vel()

    def force_vel(self):
        lib().ref_force_vel()

    def transform2crf(self, name, vel_crf, vel_force):
        f = C.c_double(vel_force)
        lib().ref_transform2crf(FIELDS[name], vel_crf, C.byref(f))
        return f.value

    def mean(self, name, nxg=None, nyg=None):
        return lib().ref_mean(FIELDS[name], nxg or self.nx, nyg or self.ny)

    def check_nan(self, name):
        return bool(lib().ref_check_nan(FIELDS[name]))

    def max_cfl(self):
        v = C.c_double()
        ijk = (C.c_int * 3)()
        lib().ref_calc_max_cfl(C.byref(v), ijk)
        return v.value, tuple(ijk)

    def max_div(self):
        v = C.c_double()
        ijk = (C.c_int * 3)()
        lib().ref_calc_max_div(C.byref(v), ijk)
        return v.value, tuple(ijk)

    # Poisson stages on a caller-owned spectral array (nx*ny*nz)
    def fft_fwd_x(self, var):
        lib().ref_fft_fwd_x(var)

    def fft_bwd_x(self, var):
        lib().ref_fft_bwd_x(var)

    def fft_fwd_y(self, var):
        lib().ref_fft_fwd_y(var)

    def fft_bwd_y(self, var):
        lib().ref_fft_bwd_y(var)

    def trid(self, var):
        lib().ref_ssolve_trid(var)

    def eigen_values(self, n):
        lam = np.zeros(n)
        lib().ref_eigen_values(n, lam)
        return lam

    def init_flow(self, initial_field="poi", u0=1.0, init_with_noise=True, noise_intensity=0.1):
        lib().ref_init_flow(INITIAL_FIELDS[initial_field], u0, int(init_with_noise),
                            noise_intensity)
        return self.get("u"), self.get("v"), self.get("w")

    def vel_force(self, d=0):
        return lib().ref_vel_force(d)

    def step(self, nsteps=1):
        lib().ref_step(nsteps)
