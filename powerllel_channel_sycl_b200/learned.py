"""Learned initialiser over the C ABI (plc_gen_*): the conditional generator,
its training data from the batched DNS, and the spin-up judge.

No counterpart in the reference, whose initial fields are laminar profiles
plus cell noise (mod_initFlow.cc).  ``Generator.propose`` writes a projected
(divergence-free) developed-turbulence guess for a given Re_tau into a
channel; ``spinup`` steps a channel until the stationarity criteria hold
(Re_tau within 1 % and the mean profile within 1 % in L2 over a 2000-step
window) and is the judge of both the generator and the laminar fallback.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from typing import Sequence

import numpy as np

from ._lib import PlcError, lib

NSTAT = 31


class GenConfig(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("channels", C.c_int * 4), ("latent_channels", C.c_int),
                ("batch", C.c_int), ("seed", C.c_ulonglong)]


def _check(rc, gen=None):
    if rc != 0:
        msg = lib().plc_gen_last_error(gen)
        raise PlcError(rc, msg.decode() if msg else "")


def config(**kw) -> GenConfig:
    cfg = GenConfig()
    _check(lib().plc_gen_config_default(C.byref(cfg)))
    for k, v in kw.items():
        if k == "channels":
            for i, c in enumerate(v):
                cfg.channels[i] = c
        else:
            setattr(cfg, k, v)
    return cfg


def cfg_dict(cfg: GenConfig) -> dict:
    return dict(nx=cfg.nx, ny=cfg.ny, nz=cfg.nz, channels=list(cfg.channels),
                latent_channels=cfg.latent_channels, batch=cfg.batch)


class Generator:
    def __init__(self, cfg: GenConfig | None = None, device: int = 0, **kw):
        self.cfg = cfg if cfg is not None else config(**kw)
        g = C.c_void_p()
        _check(lib().plc_gen_create(C.byref(self.cfg), device, C.byref(g)))
        self._g = g
        n = C.c_longlong()
        self._check(lib().plc_gen_num_params(self._g, C.byref(n)))
        self.nparams = n.value

    def _check(self, rc):
        _check(rc, self._g)

    def close(self):
        if getattr(self, "_g", None):
            lib().plc_gen_destroy(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def shape(self):
        return self.cfg.nz, self.cfg.ny, self.cfg.nx

    @property
    def params(self) -> np.ndarray:
        h = np.empty(self.nparams, np.float32)
        self._check(lib().plc_gen_get_params(self._g, h.ctypes.data))
        return h

    @params.setter
    def params(self, h):
        h = np.ascontiguousarray(h, dtype=np.float32)
        assert h.size == self.nparams
        self._check(lib().plc_gen_set_params(self._g, h.ctypes.data))

    def latent(self, seed: int) -> np.ndarray:
        c = self.cfg
        shape = (c.batch, c.nz // 8, c.ny // 8, c.nx // 8, c.latent_channels)
        h = np.empty(shape, np.float32)
        self._check(lib().plc_gen_latent(self._g, C.c_ulonglong(seed), h.ctypes.data))
        return h

    def set_targets(self, re_tau: Sequence[float], stats: np.ndarray):
        re = np.ascontiguousarray(re_tau, dtype=np.float64)
        st = np.ascontiguousarray(stats, dtype=np.float64)
        assert st.shape == (re.size, self.cfg.nz, NSTAT)
        self._check(lib().plc_gen_set_targets(self._g, re.size, re.ctypes.data, st.ctypes.data))

    def forward(self, re_tau, seed: int = 0, download: bool = True):
        re = np.ascontiguousarray(np.broadcast_to(re_tau, (self.cfg.batch,)), dtype=np.float64)
        out = np.empty((self.cfg.batch,) + self.shape + (3,), np.float32) if download else None
        self._check(lib().plc_gen_forward(self._g, re.ctypes.data, C.c_ulonglong(seed),
                                          out.ctypes.data if download else None))
        return out

    def output_stats(self) -> np.ndarray:
        h = np.empty((self.cfg.batch, self.cfg.nz, NSTAT))
        self._check(lib().plc_gen_output_stats(self._g, h.ctypes.data))
        return h

    def loss_grad(self, target_idx, re_tau, seed: int = 0, grads: bool = True):
        t = np.ascontiguousarray(target_idx, dtype=np.int32)
        re = np.ascontiguousarray(re_tau, dtype=np.float64)
        loss = C.c_double()
        g = np.empty(self.nparams, np.float32) if grads else None
        self._check(lib().plc_gen_loss_grad(self._g, t.ctypes.data, re.ctypes.data,
                                            C.c_ulonglong(seed), C.byref(loss),
                                            g.ctypes.data if grads else None))
        return loss.value, g

    def adam_step(self, lr: float):
        self._check(lib().plc_gen_adam_step(self._g, float(lr)))

    def train(self, iters: int, lr: float = 2e-3, seed: int = 1) -> np.ndarray:
        h = np.empty(iters)
        self._check(lib().plc_gen_train(self._g, int(iters), float(lr), C.c_ulonglong(seed),
                                        h.ctypes.data))
        return h

    def stats_of(self, channel) -> np.ndarray:
        h = np.empty((self.cfg.nz, NSTAT))
        self._check(lib().plc_gen_stats_of(self._g, channel._ctx, h.ctypes.data))
        return h

    def propose(self, channel, re_tau: float, seed: int = 0):
        self._check(lib().plc_gen_propose(self._g, channel._ctx, float(re_tau),
                                          C.c_ulonglong(seed)))

    def save(self, path):
        np.savez(path, params=self.params, **{k: np.asarray(v) for k, v in cfg_dict(self.cfg).items()})

    @classmethod
    def load(cls, path, device: int = 0, batch: int | None = None):
        d = np.load(path)
        cfg = config(nx=int(d["nx"]), ny=int(d["ny"]), nz=int(d["nz"]),
                     channels=[int(c) for c in d["channels"]],
                     latent_channels=int(d["latent_channels"]),
                     batch=int(batch if batch is not None else d["batch"]))
        g = cls(cfg, device=device)
        g.params = d["params"]
        return g


# ---- Re_tau <-> bulk Reynolds number ----------------------------------------
def re_from_re_tau(re_tau: float) -> float:
    """re (= Re_b / 2 with u_ref = l_ref = 1) for a target Re_tau, from
    Re_tau ~ 0.09 Re_b^0.88 (the channel-flow correlation of Pope, 2000)."""
    return 0.5 * (re_tau / 0.09) ** (1.0 / 0.88)


# ---- the spin-up judge -------------------------------------------------------
def spinup(channel, max_steps: int, window: int = 2000, every: int = 100, tol: float = 0.01,
           min_re_tau: float = 0.0, callback=None) -> dict:
    """Steps the channel until Re_tau (both walls) stays within tol of its
    window mean and the plane-mean u profile within tol in relative L2 over
    the last `window` steps, with Re_tau >= min_re_tau (the turbulent branch).
    Returns the steps taken (None if max_steps passed first), the history and
    the wall-clock time."""
    hist_n, hist_re, hist_u = [], [], []
    need = window // every + 1
    t0 = time.perf_counter()
    n = 0
    stationary_at = None
    while n < max_steps:
        channel.step(every)
        n += every
        hist_n.append(n)
        hist_re.append(channel.re_tau())
        hist_u.append(channel.mean_profile())
        if callback:
            callback(n, hist_re[-1])
        if len(hist_re) >= need:
            re = np.array(hist_re[-need:])
            us = np.array(hist_u[-need:])
            um = us.mean(axis=0)
            ok_re = np.max(np.abs(re - re.mean())) <= tol * re.mean()
            ok_u = np.max(np.linalg.norm(us - um, axis=1)) <= tol * np.linalg.norm(um)
            if ok_re and ok_u and re.mean() >= min_re_tau:
                stationary_at = n
                break
    return {"steps": stationary_at, "steps_run": n, "re_tau": np.array(hist_re),
            "n": np.array(hist_n), "wall_s": time.perf_counter() - t0}
