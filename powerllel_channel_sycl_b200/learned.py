"""Learned initialiser over the C ABI (plc_gen_*): the conditional generator,
its training data from the batched DNS, and the spin-up judge.

No counterpart in the reference, whose initial fields are laminar profiles
plus cell noise (mod_initFlow.cc).  ``Generator.propose`` writes a projected
(divergence-free) developed-turbulence guess for a given Re_tau into a
channel; ``spinup`` steps a channel until the stationarity criteria hold
(Re_tau and the mean profile, averaged over a 2000-step window, within 1 %
of the previous window's) and is the judge of both the generator and the
laminar fallback.
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
    """Steps the channel until it is statistically stationary: the means over
    the last `window` steps of Re_tau (both walls, sampled every `every`
    steps) and of the plane-mean u profile agree with those of the window
    before within tol (relative; the profile in L2), with the mean Re_tau at
    least min_re_tau (the turbulent branch; laminar flow also becomes
    stationary).  Returns the step count at which that first held (None if
    max_steps passed first), the history and the wall-clock time."""
    per = window // every
    hist_n, hist_re, hist_u = [], [], []
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
        if len(hist_re) >= 2 * per:
            re_now = np.mean(hist_re[-per:])
            re_before = np.mean(hist_re[-2 * per:-per])
            u_now = np.mean(hist_u[-per:], axis=0)
            u_before = np.mean(hist_u[-2 * per:-per], axis=0)
            ok_re = abs(re_now - re_before) <= tol * re_now
            ok_u = np.linalg.norm(u_now - u_before) <= tol * np.linalg.norm(u_now)
            if ok_re and ok_u and re_now >= min_re_tau:
                stationary_at = n
                break
    return {"steps": stationary_at, "steps_run": n, "re_tau": np.array(hist_re),
            "n": np.array(hist_n), "wall_s": time.perf_counter() - t0}


# ---- training data from the batched DNS ----------------------------------------
def member_specs(n: int = 16, seed: int = 7, re_tau_range=(120.0, 400.0)) -> list:
    """n channels of the 4pi x 2pi x 2 box (tanh 1.5) with Re_tau drawn
    uniformly in re_tau_range; grids grow with Re_tau and are multiples of
    the generator's 64 x 48 x 64."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        rt = float(rng.uniform(*re_tau_range))
        if rt < 200:
            nx, ny, nz = 128, 96, 64
        elif rt < 300:
            nx, ny, nz = 192, 144, 128
        else:
            nx, ny, nz = 256, 192, 128
        out.append(dict(nx=nx, ny=ny, nz=nz, re_tau_target=rt, re=re_from_re_tau(rt)))
    return out


def channel_params_for(spec: dict, precision="mixed", cfl_target=0.4, nt_check=50,
                       vortices=0.15, noise=0.1):
    from .channel import make_params
    return make_params(nx=spec["nx"], ny=spec["ny"], nz=spec["nz"], lx=4 * math.pi,
                       ly=2 * math.pi, lz=2.0, mesh_type=1, stretch_func=0, stretch_ratio=1.5,
                       re=spec["re"], u_ref=1.0, l_ref=1.0, dt=1e-3, nt_check=nt_check,
                       cfl_limit=1.0, div_limit=1e-6, initial_field="poi", init_with_noise=1,
                       noise_intensity=noise, is_forced=[1, 0, 0], vel_force=[1.0, 0.0, 0.0],
                       precision=precision, cfl_target=cfl_target, init_vortex_amp=vortices)


def collect(gen: Generator, specs: list, spin_steps: int, snap_every: int = 500,
            n_snap: int = 10, device: int = 0, log=print) -> dict:
    """Runs the members as one batched ensemble from laminar + noise +
    vortices, then takes n_snap snapshots every snap_every steps: per member
    the generator-grid statistics and Re_tau of each snapshot."""
    from .ensemble import Ensemble
    ens = Ensemble([channel_params_for(s) for s in specs], device=device)
    ens.initFlow()
    ens.autotune(steps=3)
    t0 = time.perf_counter()
    done = 0
    while done < spin_steps:
        k = min(5000, spin_steps - done)
        ens.step(k)
        done += k
        if log:
            log(f"spin-up {done}/{spin_steps} steps, Re_tau "
                + " ".join(f"{m.re_tau():.0f}" for m in ens.members)
                + f"  ({time.perf_counter() - t0:.0f} s)")
    stats = np.zeros((len(specs), n_snap, gen.cfg.nz, NSTAT))
    re_tau = np.zeros((len(specs), n_snap))
    for q in range(n_snap):
        ens.step(snap_every)
        for i, m in enumerate(ens.members):
            stats[i, q] = gen.stats_of(m)
            re_tau[i, q] = m.re_tau()
    ens.close()
    return {"stats": stats, "re_tau": re_tau,
            "re": np.array([s["re"] for s in specs]),
            "grids": np.array([[s["nx"], s["ny"], s["nz"]] for s in specs]),
            "spin_steps": spin_steps, "snap_every": snap_every,
            "wall_s": time.perf_counter() - t0}


def targets_from(data: dict, min_re_tau: float = 110.0):
    """Per member: mean Re_tau and mean statistics over its snapshots, for the
    members that stayed turbulent."""
    re = data["re_tau"].mean(axis=1)
    keep = re >= min_re_tau
    return re[keep], data["stats"][keep].mean(axis=1)


# ---- the stored model --------------------------------------------------------
import os as _os

MODEL_DIR = _os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "models")
WEIGHTS = _os.path.join(MODEL_DIR, "initialiser_weights.npz")
TARGETS = _os.path.join(MODEL_DIR, "initialiser_targets.npz")


def save_weights(gen: Generator, path: str = WEIGHTS):
    """Parameters stored as BF16 (the precision the network computes in)."""
    p = gen.params.astype(np.float32)
    u = p.view(np.uint32).astype(np.uint64)
    b = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
    np.savez_compressed(path, params_bf16=b, **{k: np.asarray(v) for k, v in cfg_dict(gen.cfg).items()})


def load_weights(path: str = WEIGHTS, device: int = 0, batch: int = 1) -> Generator:
    d = np.load(path)
    cfg = config(nx=int(d["nx"]), ny=int(d["ny"]), nz=int(d["nz"]),
                 channels=[int(c) for c in d["channels"]],
                 latent_channels=int(d["latent_channels"]), batch=batch)
    g = Generator(cfg, device=device)
    g.params = (d["params_bf16"].astype(np.uint32) << 16).view(np.float32)
    return g


def _main(argv=None):
    """python -m powerllel_channel_sycl_b200.learned collect|train|evaluate"""
    import argparse
    import json
    ap = argparse.ArgumentParser(prog="python -m powerllel_channel_sycl_b200.learned")
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("collect", help="snapshot statistics from the batched DNS")
    c.add_argument("--members", type=int, default=16)
    c.add_argument("--spin", type=int, default=30000)
    c.add_argument("--snapshots", type=int, default=10)
    c.add_argument("--every", type=int, default=500)
    c.add_argument("--out", default=TARGETS)
    t = sub.add_parser("train", help="train the generator on collected targets")
    t.add_argument("--targets", default=TARGETS)
    t.add_argument("--iters", type=int, default=6000)
    t.add_argument("--lr", type=float, default=2e-3)
    t.add_argument("--out", default=WEIGHTS)
    e = sub.add_parser("evaluate", help="steps to stationarity: generator vs fallbacks")
    e.add_argument("--weights", default=WEIGHTS)
    e.add_argument("--re-tau", type=float, nargs="+", default=[180.0, 300.0, 395.0])
    e.add_argument("--max-steps", type=int, default=60000)
    e.add_argument("--json", default=None)
    a = ap.parse_args(argv)
    if a.cmd == "collect":
        gen = Generator(config(batch=1))
        data = collect(gen, member_specs(a.members), a.spin, a.every, a.snapshots)
        re, st = targets_from(data)
        np.savez_compressed(a.out, re_tau=re, stats=st, snapshot_re_tau=data["re_tau"],
                            grids=data["grids"], re=data["re"], spin=a.spin)
        print(f"{len(re)} targets, Re_tau {np.round(re, 1)} -> {a.out}")
    elif a.cmd == "train":
        d = np.load(a.targets)
        gen = Generator(config(batch=4, seed=1))
        gen.set_targets(d["re_tau"], d["stats"])
        t0 = time.perf_counter()
        hist = gen.train(a.iters, lr=a.lr, seed=1)
        print(f"{a.iters} iterations in {time.perf_counter() - t0:.1f} s, loss "
              f"{hist[:50].mean():.3g} -> {hist[-50:].mean():.3g}")
        save_weights(gen, a.out)
    else:
        from .channel import Channel
        gen = load_weights(a.weights)
        res = {}
        for rt in a.re_tau:
            spec = dict(nx=256, ny=192, nz=128, re=re_from_re_tau(rt))
            for method in ("generator", "vortices", "laminar_noise"):
                ch = Channel(channel_params_for(spec, vortices=0.15 if method == "vortices" else 0.0))
                ch.initFlow()
                t0 = time.perf_counter()
                if method == "generator":
                    gen.propose(ch, rt, seed=1)
                t_init = time.perf_counter() - t0
                r = spinup(ch, a.max_steps, min_re_tau=0.75 * rt)
                res[f"{rt:g}/{method}"] = {"steps": r["steps"], "steps_run": r["steps_run"],
                                           "wall_s": r["wall_s"] + t_init,
                                           "re_tau_end": float(r["re_tau"][-1])}
                print(f"Re_tau {rt:g} {method:13s} stationary after {r['steps']} steps "
                      f"({r['wall_s'] + t_init:.1f} s), Re_tau {r['re_tau'][-1]:.1f}", flush=True)
                ch.close()
        if a.json:
            with open(a.json, "w") as f:
                json.dump(res, f, indent=1)


if __name__ == "__main__":
    _main()
