"""Shared test helpers: build matching oracle / GPU cases on the same inputs."""
from __future__ import annotations

import numpy as np

import oracle

CONFIG0 = dict(nx=128, ny=64, nz=64, lx=4 * np.pi, ly=2 * np.pi, lz=2.0, dt=2e-3, re=2800.0,
               stretch_ratio=1.5)


def case_kwargs(nx, ny, nz, **kw):
    d = dict(nx=nx, ny=ny, nz=nz, lx=4 * np.pi, ly=2 * np.pi, lz=2.0, dt=2e-3, re=2800.0,
             mesh_type=1, stretch_func=0, stretch_ratio=1.5, u_crf=0.0,
             is_forced=(True, False, False), vel_force=(1.0, 0.0, 0.0))
    d.update(kw)
    return d


def oracle_case(**kw) -> oracle.Case:
    return oracle.Case(**kw)


def channel_params(**kw):
    from powerllel_channel_sycl_b200 import make_params
    mapping = dict(kw)
    return make_params(
        nx=mapping["nx"], ny=mapping["ny"], nz=mapping["nz"], lx=mapping["lx"], ly=mapping["ly"],
        lz=mapping["lz"], dt=mapping["dt"], re=mapping["re"], u_ref=1.0, l_ref=1.0,
        mesh_type=mapping["mesh_type"], stretch_func=mapping["stretch_func"],
        stretch_ratio=mapping["stretch_ratio"], u_crf=mapping["u_crf"],
        is_forced=[int(x) for x in mapping["is_forced"]], vel_force=list(mapping["vel_force"]),
        initial_field="poi", init_with_noise=1, noise_intensity=0.1)


def random_fields(case: oracle.Case, seed: int, n: int = 3, scale: float = 1.0):
    rng = np.random.default_rng(seed)
    return [rng.uniform(-scale, scale, case.shape) for _ in range(n)]


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.linalg.norm(b.ravel())
    if den == 0:
        return float(np.linalg.norm(a.ravel()))
    return float(np.linalg.norm((a - b).ravel()) / den)


def interior(a):
    return a[1:-1, 1:-1, 1:-1]


def demean(p):
    q = interior(p)
    return q - q.mean()
