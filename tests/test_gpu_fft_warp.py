"""The warp-line transforms (plan family 2) against the oracle.

Each warp transforms its own lines with no block barrier (first pass loaded
from global memory, passes exchanged through the warp's shared memory, last
inverse pass stored to global memory).  Pinned by PLC_FFT_PLANS=2,2 (FP64)
and PLC_FFT_PLANS_F32=2,2 (mixed form) on every length that has a plan:
each FFT direction within 1e-14 relative L2 of the oracle (as the other
families), the Poisson solve within 1e-12 on p - mean(p), the mixed form's
projection divergence-free to FP32 rounding, and 10 fused steps of the FP64
form within 1e-12 of the oracle.
"""
import numpy as np
import pytest

import oracle
from tests.helpers import case_kwargs, channel_params, demean, interior, random_fields, rel_l2

pytestmark = pytest.mark.gpu

# every length with a warp-line plan appears as an x and as a y length
SIZES = [(768, 384, 2), (384, 192, 4), (256, 192, 4), (128, 96, 8), (64, 48, 8), (96, 64, 8),
         (512, 32, 4), (192, 128, 4), (48, 64, 4), (96, 32, 4), (32, 256, 2)]


def make_pair(nx, ny, nz, **kw):
    from powerllel_channel_sycl_b200 import Channel
    kwargs = case_kwargs(nx, ny, nz, **kw)
    return oracle.Case(**kwargs), Channel(channel_params(**kwargs))


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_warp_fft_each_direction(monkeypatch, nx, ny, nz):
    monkeypatch.setenv("PLC_FFT_PLANS", "2,2")
    case, ch = make_pair(nx, ny, nz)
    t = ch.fft_tiles
    assert (t["plan_x"], t["plan_y"]) == (2, 2)
    (p,) = random_fields(case, 17, n=1)
    ch.upload("p", p)
    var = np.zeros(nx * ny * nz)
    case.fft_fwd_x(p, var)
    ch.execute_fft_fwd_xpen()
    gs = ch.download("spec").ravel()
    assert rel_l2(gs, var) < 1e-14
    case.fft_fwd_y(var)
    ch.upload("spec", gs.reshape(nz, ny, nx))
    ch.execute_fft_fwd_ypen()
    gs = ch.download("spec").ravel()
    assert rel_l2(gs, var) < 1e-14
    case.fft_bwd_y(var)
    ch.upload("spec", gs.reshape(nz, ny, nx))
    ch.execute_fft_bwd_ypen()
    gs = ch.download("spec").ravel()
    assert rel_l2(gs, var) < 1e-14
    q = case.zeros()
    case.fft_bwd_x(var, q)
    ch.upload("spec", gs.reshape(nz, ny, nx))
    ch.execute_fft_bwd_xpen()
    gq = ch.download("p")
    assert rel_l2(interior(gq), interior(q)) < 1e-14


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_warp_poisson_both_forms(monkeypatch, nx, ny, nz):
    monkeypatch.setenv("PLC_FFT_PLANS", "2,2")
    monkeypatch.setenv("PLC_FFT_PLANS_F32", "2,2")
    case, ch = make_pair(nx, ny, nz)
    u, v, w = random_fields(case, 19)
    case.update_bound_vel(u, v, w)
    p = case.zeros()
    case.calc_rhs(u, v, w, p)
    ch.upload("p", p)
    case.poisson(p)
    ch.execute_poisson_solver()
    assert rel_l2(demean(ch.download("p")), demean(p)) < 1e-12
    from powerllel_channel_sycl_b200 import Channel
    prm = channel_params(**case_kwargs(nx, ny, nz))
    prm.precision = 1
    m = Channel(prm)
    t = m.fft_tiles
    assert (t["plan_x"], t["plan_y"]) == (2, 2)
    for name, a in zip("uvw", (u, v, w)):
        m.upload(name, a)
    m.project()
    assert m.check()[2][0] < 1e-3


def test_warp_step_parity(monkeypatch):
    monkeypatch.setenv("PLC_FFT_PLANS", "2,2")
    case, ch = make_pair(128, 64, 64)
    u, v, w = case.init_flow("poi", noise_intensity=0.1)
    for name, a in zip("uvw", (u, v, w)):
        ch.upload(name, a)
    ch.upload("p", case.zeros())
    u1, v1, w1, p = case.zeros(), case.zeros(), case.zeros(), case.zeros()
    case.step(u, v, w, u1, v1, w1, p, nsteps=10)
    ch.step(10)
    for name, a in zip("uvw", (u, v, w)):
        assert rel_l2(ch.download(name), a) <= 1e-12, name
    assert rel_l2(demean(ch.download("p")), demean(p)) <= 2e-12
