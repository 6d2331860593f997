"""The two-pass transforms (plan family 3) against the oracle.

A line of length N = R1 * R2 is transformed by one radix-R1 pass loaded
straight from global memory into registers, one exchange through shared
memory and one radix-R2 pass, the two real spectra of each complex line
separated while storing (forward) or the result stored with its halos
(backward x).  Pinned by PLC_FFT_PLANS (FP64) and PLC_FFT_PLANS_F32 (mixed
form) on every x and y length that has a plan: each direction within 1e-14
relative L2 of the oracle (as the other families), the Poisson solve within
1e-12 on p - mean(p), the mixed form's projection divergence-free to FP32
rounding, and 10 fused steps of the FP64 form within 1e-12 of the oracle
(2e-12 in p - mean(p), its round-off floor).
"""
import numpy as np
import pytest

import oracle
from tests.helpers import case_kwargs, channel_params, demean, interior, random_fields, rel_l2

pytestmark = pytest.mark.gpu

# every y length with a two-pass plan; x lengths multiples of 32 columns
SIZES = [(64, 384, 2), (32, 256, 4), (64, 192, 4), (96, 128, 4), (32, 96, 8), (64, 64, 8),
         (32, 48, 8), (64, 32, 8)]


def make_pair(nx, ny, nz, **kw):
    from powerllel_channel_sycl_b200 import Channel
    kwargs = case_kwargs(nx, ny, nz, **kw)
    return oracle.Case(**kwargs), Channel(channel_params(**kwargs))


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_y2_each_direction(monkeypatch, nx, ny, nz):
    monkeypatch.setenv("PLC_FFT_PLANS", "0,3")
    case, ch = make_pair(nx, ny, nz)
    assert ch.fft_tiles["plan_y"] == 3
    rng = np.random.default_rng(ny)
    var = rng.standard_normal(nx * ny * nz)
    ch.upload("spec", var.reshape(nz, ny, nx))
    ref = var.copy()
    case.fft_fwd_y(ref)
    ch.execute_fft_fwd_ypen()
    assert rel_l2(ch.download("spec").ravel(), ref) < 1e-14
    ch.upload("spec", ref.reshape(nz, ny, nx))
    back = ref.copy()
    case.fft_bwd_y(back)
    ch.execute_fft_bwd_ypen()
    assert rel_l2(ch.download("spec").ravel(), back) < 1e-14


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_y2_poisson_both_forms(monkeypatch, nx, ny, nz):
    monkeypatch.setenv("PLC_FFT_PLANS", "0,3")
    monkeypatch.setenv("PLC_FFT_PLANS_F32", "0,3")
    case, ch = make_pair(nx, ny, nz)
    u, v, w = random_fields(case, 23)
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
    assert m.fft_tiles["plan_y"] == 3
    for name, a in zip("uvw", (u, v, w)):
        m.upload(name, a)
    m.project()
    assert m.check()[2][0] < 1e-3


# every x length with a two-pass plan, over whole blocks of rows
XSIZES = [(768, 16, 2), (512, 32, 2), (384, 32, 2), (256, 64, 2), (192, 32, 4), (128, 64, 4),
          (96, 32, 4), (64, 32, 8), (48, 64, 4), (32, 32, 8)]


@pytest.mark.parametrize("nx,ny,nz", XSIZES)
def test_x2_each_direction(monkeypatch, nx, ny, nz):
    monkeypatch.setenv("PLC_FFT_PLANS", "3,0")
    case, ch = make_pair(nx, ny, nz)
    t = ch.fft_tiles
    assert (t["plan_x"], t["plan_x_fwd"]) == (3, 3)
    (p,) = random_fields(case, nx, n=1)
    ch.upload("p", p)
    var = np.zeros(nx * ny * nz)
    case.fft_fwd_x(p, var)
    ch.execute_fft_fwd_xpen()
    assert rel_l2(ch.download("spec").ravel(), var) < 1e-14
    q = case.zeros()
    case.fft_bwd_x(var, q)
    ch.upload("spec", var.reshape(nz, ny, nx))
    ch.execute_fft_bwd_xpen()
    assert rel_l2(interior(ch.download("p")), interior(q)) < 1e-14


@pytest.mark.parametrize("nx,ny,nz", XSIZES)
def test_x2_poisson_both_forms(monkeypatch, nx, ny, nz):
    monkeypatch.setenv("PLC_FFT_PLANS", "3,0")
    monkeypatch.setenv("PLC_FFT_PLANS_F32", "3,0")
    case, ch = make_pair(nx, ny, nz)
    u, v, w = random_fields(case, 29)
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
    assert m.fft_tiles["plan_x"] == 3
    for name, a in zip("uvw", (u, v, w)):
        m.upload(name, a)
    m.project()
    assert m.check()[2][0] < 1e-3


@pytest.mark.parametrize("plans", ["0,3", "3,3"])
def test_two_pass_step_parity(monkeypatch, plans):
    monkeypatch.setenv("PLC_FFT_PLANS", plans)
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


def test_y2_pin_rejected_without_plan(monkeypatch):
    from powerllel_channel_sycl_b200 import Channel, PlcError
    monkeypatch.setenv("PLC_FFT_PLANS", "0,3")
    with pytest.raises(PlcError):
        Channel(channel_params(**case_kwargs(32, 24, 16)))  # no plan for 24
