"""The mixed-precision form (FP32 fields, stencils and FFTs; FP64 scalars,
reductions and tridiagonal sweep) against the FP64 oracle.

The mixed form has no counterpart in the reference; its error bars are the
ones stated for it: 10-step velocity rel L2 <= 1e-4 against FP64, and
plane-averaged mean profiles within 0.5 %.
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import case_kwargs, channel_params, demean, interior, oracle_case, rel_l2

pytestmark = pytest.mark.gpu

VEL_TOL = 1e-4        # 10-step velocity rel L2, mixed vs FP64
PROFILE_TOL = 5e-3    # mean-profile relative error
# Pressure (up to a constant) rel L2.  The pressure of these noisy fields is
# ill-conditioned: the FP64 oracle amplifies rounding of 1e-16 to ~1e-12
# (test_pressure_roundoff_floor), i.e. ~1e4, so FP32 rounding (6e-8) puts it
# near 1e-3.
P_TOL = 5e-3
DIV_TOL = 1e-3        # max |div u| after the projection, FP32 rounding level


def mixed_channel(nx, ny, nz, **kw):
    from powerllel_channel_sycl_b200 import Channel
    prm = channel_params(**case_kwargs(nx, ny, nz, **kw))
    prm.precision = 1
    return Channel(prm)


def fp64_pair(nx, ny, nz, **kw):
    from powerllel_channel_sycl_b200 import Channel
    kwargs = case_kwargs(nx, ny, nz, **kw)
    return oracle_case(**kwargs), Channel(channel_params(**kwargs))


def test_upload_download_rounds_to_fp32():
    ch = mixed_channel(32, 24, 16)
    assert ch.mixed
    rng = np.random.default_rng(7)
    a = rng.standard_normal(ch.shape)
    ch.upload("u", a)
    assert np.array_equal(ch.download("u"), a.astype(np.float32).astype(np.float64))
    s = rng.standard_normal(ch.spec_shape)
    ch.upload("spec", s)
    assert np.array_equal(ch.download("spec"), s.astype(np.float32).astype(np.float64))
    ptr, count, pitch = ch.ptr_f32("u")
    assert ptr and pitch % 4 == 0 and pitch >= 34
    assert count == pitch * (24 + 2) * (16 + 2)


def test_module_entry_points_refused():
    from powerllel_channel_sycl_b200 import PlcError
    ch = mixed_channel(32, 24, 16)
    with pytest.raises(PlcError) as e:
        ch.timeIntVelRK1()
    assert e.value.code == -8  # PLC_ERR_STATE
    with pytest.raises(PlcError):
        ch.execute_poisson_solver()


def test_init_flow_matches_fp64():
    """initFlow in the mixed form: the FP64 field rounded to FP32."""
    case, ref = fp64_pair(64, 48, 32)
    ch = mixed_channel(64, 48, 32)
    ref.initFlow()
    ch.initFlow()
    for name in "uvw":
        a, b = ch.download(name), ref.download(name)
        assert rel_l2(interior(a), interior(b)) < 1e-6, name


@pytest.mark.parametrize("nx,ny,nz,nsteps", [(32, 24, 16, 5), (128, 64, 64, 10)])
def test_step_vs_fp64_oracle(nx, ny, nz, nsteps):
    """nsteps of main.cc:116-154 in the mixed form vs the FP64 oracle."""
    case = oracle_case(**case_kwargs(nx, ny, nz))
    ch = mixed_channel(nx, ny, nz)
    u, v, w = case.init_flow("poi", noise_intensity=0.1)
    for name, a in zip("uvw", (u, v, w)):
        ch.upload(name, a)
    u1, v1, w1, p = case.zeros(), case.zeros(), case.zeros(), case.zeros()
    case.step(u, v, w, u1, v1, w1, p, nsteps=nsteps)
    ch.step(nsteps)
    for name, a in zip("uvw", (u, v, w)):
        e = rel_l2(interior(ch.download(name)), interior(a))
        assert e <= VEL_TOL, (name, e)
    e = rel_l2(demean(ch.download("p")), demean(p))
    assert e <= P_TOL, e
    ok, cfl, div = ch.check()
    assert ok
    assert div[0] < DIV_TOL, div
    # bulk velocity held at vel_force by the FP64 forcing sum
    ubar = (interior(ch.download("u")).mean(axis=(1, 2)) * case.dzflzi[1:-1]).sum()
    assert abs(ubar - 1.0) < 1e-5


def test_mean_profile_long_run():
    """200 steps: plane-averaged u(z) and u_rms(z) of the mixed form vs FP64."""
    _, ref = fp64_pair(64, 48, 48)
    ch = mixed_channel(64, 48, 48)
    ref.initFlow()
    ch.initFlow()
    ref.step(200)
    ch.step(200)
    a = interior(ch.download("u"))
    b = interior(ref.download("u"))
    ma, mb = a.mean(axis=(1, 2)), b.mean(axis=(1, 2))
    assert np.max(np.abs(ma - mb)) / np.max(np.abs(mb)) < PROFILE_TOL
    ra = np.sqrt(((a - ma[:, None, None]) ** 2).mean(axis=(1, 2)))
    rb = np.sqrt(((b - mb[:, None, None]) ** 2).mean(axis=(1, 2)))
    assert np.max(np.abs(ra - rb)) / np.max(rb) < 5e-2


def test_cfl_controlled_dt():
    from powerllel_channel_sycl_b200 import Channel
    prm = channel_params(**case_kwargs(64, 48, 32))
    prm.precision = 1
    prm.cfl_target = 0.5
    prm.nt_check = 5
    prm.cfl_limit = 1.0
    prm.div_limit = 1e-9  # scaled by 2^29 in the mixed form
    ch = Channel(prm)
    ch.initFlow()
    ch.step(20)
    ok, cfl, div = ch.check()
    assert ok
    assert 0.3 < cfl[0] < 0.6
    assert ch.dt > 0


def test_step_graph_kernel_count():
    """RK2 writes the bulk-mean partials, a one-block kernel turns them into
    the forcing and the correction applies it: no forcing pass over the field."""
    ch = mixed_channel(32, 24, 16)
    ch.initFlow()
    assert ch.kernels_per_step == 9


def test_profile_step_mixed():
    ch = mixed_channel(64, 48, 32)
    ch.initFlow()
    ms = ch.profile_step(2)
    assert len(ms) == 8 and all(t > 0 for t in ms.values())
    assert "correct+force+bound(u)" in ms


# line lengths of every FP32 transform plan: 3*2^a (two passes ending in a
# radix-24 butterfly, or one for 24), 2^a, and the 16/16/3 plan of 768
@pytest.mark.parametrize("nx,ny,nz", [(48, 32, 8), (96, 32, 8), (192, 32, 8), (384, 32, 8),
                                      (768, 16, 4), (32, 24, 8), (32, 48, 8), (32, 96, 8),
                                      (32, 192, 8), (16, 384, 8), (64, 256, 4)])
def test_fp32_transform_plans_project_like_fp64(nx, ny, nz):
    """The projection of one random field in both forms: the mixed form's
    velocity is divergence-free to FP32 rounding and within 1e-4 of the FP64
    form's, for transforms of every FP32 plan in x and in y."""
    from powerllel_channel_sycl_b200 import Channel
    rng = np.random.default_rng(nx * 1000 + ny)
    out = []
    for precision in (0, 1):
        prm = channel_params(**case_kwargs(nx, ny, nz))
        prm.precision = precision
        ch = Channel(prm)
        if precision == 0:
            fields = {q: rng.normal(size=ch.shape) for q in "uvw"}
        for q in "uvw":
            ch.upload(q, fields[q])
        ch.project()
        out.append(({q: interior(ch.download(q)) for q in "uvw"}, ch.check()[2][0]))
        ch.close()
    (ref, _), (mix, div) = out
    assert div < DIV_TOL, div
    for q in "uvw":
        assert rel_l2(mix[q], ref[q]) < VEL_TOL, (q, rel_l2(mix[q], ref[q]))
