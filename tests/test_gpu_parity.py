"""GPU parity: every entry point of libplc.so against the CPU oracle on the
same seeded inputs (FP64).

Tolerances: boundary rules, stencils (RK1, RK2, calcRHS, correctVel), the
bulk mean and the initial field are bit-exact (both sides evaluate the
reference expressions term by term without contraction, and sum in
double-double); FFT-based results agree to 1e-14 relative L2 (different FFT
algorithms); the 10-step run of the channel agrees to 1e-12 relative L2 in
u, v, w and in p - mean(p) (the reference's p carries an arbitrary constant
from the singular (0,0) mode).
"""
import numpy as np
import pytest

import oracle
from tests.helpers import case_kwargs, channel_params, demean, interior, random_fields, rel_l2

pytestmark = pytest.mark.gpu

SIZES = [(32, 24, 16), (48, 32, 8), (6, 4, 2), (16, 12, 6)]


def make_pair(nx, ny, nz, **kw):
    from powerllel_channel_sycl_b200 import Channel
    kwargs = case_kwargs(nx, ny, nz, **kw)
    case = oracle.Case(**kwargs)
    ch = Channel(channel_params(**kwargs))
    return case, ch


def bc_fields(case, seed):
    u, v, w = random_fields(case, seed)
    case.update_bound_vel(u, v, w)
    return u, v, w


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_mesh_identical(nx, ny, nz):
    case, ch = make_pair(nx, ny, nz)
    for name in ["dzf_global", "dzf", "dzf_inv", "dzc", "dzc_inv", "dzflzi", "zc_global"]:
        np.testing.assert_array_equal(ch.mesh(name), getattr(case, name))


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_update_bound_vel_exact(nx, ny, nz):
    case, ch = make_pair(nx, ny, nz, u_crf=0.25)
    u, v, w = random_fields(case, 1)
    for name, a in zip("uvw", (u, v, w)):
        ch.upload(name, a)
    case.update_bound_vel(u, v, w)
    ch.updateBoundVel(0.25)
    for name, a in zip("uvw", (u, v, w)):
        np.testing.assert_array_equal(ch.download(name), a)


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_update_bound_p_exact(nx, ny, nz):
    case, ch = make_pair(nx, ny, nz)
    (p,) = random_fields(case, 2, n=1)
    ch.upload("p", p)
    case.update_bound_p(p)
    ch.updateBoundP()
    np.testing.assert_array_equal(ch.download("p"), p)


@pytest.mark.parametrize("nx,ny,nz", SIZES)
@pytest.mark.parametrize("u_crf", [0.0, 0.3])
def test_rk1_rk2(nx, ny, nz, u_crf):
    case, ch = make_pair(nx, ny, nz, u_crf=u_crf)
    u, v, w = bc_fields(case, 3)
    for name, a in zip("uvw", (u, v, w)):
        ch.upload(name, a)
    u1, v1, w1 = case.zeros(), case.zeros(), case.zeros()
    case.rk1(u, v, w, u1, v1, w1)
    ch.timeIntVelRK1(u_crf)
    # stencils are evaluated term by term without contraction: bit-identical
    for name, a in zip(("u1", "v1", "w1"), (u1, v1, w1)):
        np.testing.assert_array_equal(interior(ch.download(name)), interior(a), err_msg=name)
    # RK2 from the same u1 (after its boundary update)
    case.update_bound_vel(u1, v1, w1)
    for name, a in zip(("u1", "v1", "w1"), (u1, v1, w1)):
        ch.upload(name, a)
    case.rk2(u, v, w, u1, v1, w1)
    ch.timeIntVelRK2(u_crf)
    for name, a in zip("uvw", (u, v, w)):
        np.testing.assert_array_equal(interior(ch.download(name)), interior(a), err_msg=name)


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_calc_rhs_and_correct(nx, ny, nz):
    case, ch = make_pair(nx, ny, nz)
    u, v, w = bc_fields(case, 4)
    for name, a in zip("uvw", (u, v, w)):
        ch.upload(name, a)
    p = case.zeros()
    case.calc_rhs(u, v, w, p)
    ch.calcRHS()
    np.testing.assert_array_equal(interior(ch.download("p")), interior(p))
    # correctVel on a random pressure with valid halos
    (q,) = random_fields(case, 5, n=1)
    case.update_bound_p(q)
    ch.upload("p", q)
    case.correct_vel(q, u, v, w)
    ch.correctVel()
    for name, a in zip("uvw", (u, v, w)):
        np.testing.assert_array_equal(interior(ch.download(name)), interior(a), err_msg=name)


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_mean_and_force(nx, ny, nz):
    case, ch = make_pair(nx, ny, nz)
    u, v, w = bc_fields(case, 6)
    for name, a in zip("uvw", (u, v, w)):
        ch.upload(name, a)
    # double-double accumulation on both sides: the same rounded sum
    assert ch.Mean(var="u") == case.mean(u)
    assert ch.Mean(17, 5, var="v") == case.mean(v, 17, 5)
    f_ref = case.force_vel(u, v, w)
    f_gpu = ch.forceVel()
    assert f_gpu[0] == f_ref[0]
    assert f_gpu[1] == 0.0 and f_gpu[2] == 0.0
    np.testing.assert_array_equal(interior(ch.download("u")), interior(u))


@pytest.mark.parametrize("nx,ny,nz", SIZES + [(128, 64, 8), (96, 48, 4), (768, 12, 2), (8, 384, 2),
                                      (512, 8, 2), (8, 256, 2), (192, 192, 2)])
def test_fft_each_direction(nx, ny, nz):
    case, ch = make_pair(nx, ny, nz)
    (p,) = random_fields(case, 7, n=1)
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
    # round trip returns the input
    assert rel_l2(interior(gq), interior(p)) < 1e-13


@pytest.mark.parametrize("nx,ny,nz", SIZES + [(64, 48, 64)])
def test_trid(nx, ny, nz):
    case, ch = make_pair(nx, ny, nz)
    rng = np.random.default_rng(8)
    var = rng.standard_normal(nx * ny * nz)
    ch.upload("spec", var.reshape(nz, ny, nx))
    ref = var.copy()
    case.trid(ref)
    ch.solve_trid()
    g = ch.download("spec").ravel()
    r3, g3 = ref.reshape(nz, ny, nx), g.reshape(nz, ny, nx)
    mask = np.ones((ny, nx), bool)
    mask[0, 0] = False
    assert rel_l2(g3[:, mask], r3[:, mask]) < 1e-13
    # the singular system agrees up to round-off of its (large) constant
    assert rel_l2(g3[:, 0, 0], r3[:, 0, 0]) < 1e-9


@pytest.mark.parametrize("nx,ny,nz", SIZES + [(128, 64, 64)])
def test_poisson_solve(nx, ny, nz):
    case, ch = make_pair(nx, ny, nz)
    u, v, w = bc_fields(case, 9)
    p = case.zeros()
    case.calc_rhs(u, v, w, p)
    ch.upload("p", p)
    case.poisson(p)
    ch.execute_poisson_solver()
    gp = ch.download("p")
    assert rel_l2(demean(gp), demean(p)) < 1e-12


@pytest.mark.parametrize("field,u_crf", [("poi", 0.0), ("log", 0.0), ("uni", 0.2)])
def test_init_flow(field, u_crf):
    from powerllel_channel_sycl_b200 import Channel
    kwargs = case_kwargs(32, 24, 16, u_crf=u_crf)
    case = oracle.Case(**kwargs)
    prm = channel_params(**kwargs)
    prm.initial_field = {"uni": 0, "poi": 1, "log": 2}[field]
    prm.u0 = 1.0
    ch = Channel(prm)
    ch.initFlow()
    u, v, w = case.init_flow(field, u0=1.0, noise_intensity=0.1)
    for name, a in zip("uvw", (u, v, w)):
        np.testing.assert_array_equal(ch.download(name), a, err_msg=name)


def test_checks():
    case, ch = make_pair(32, 24, 16)
    u, v, w = bc_fields(case, 10)
    for name, a in zip("uvw", (u, v, w)):
        ch.upload(name, a)
    assert ch.checkNaN("u")
    cfl = ch.calcMaxCFL()
    cref = case.max_cfl(u, v, w)
    assert cfl[1] == cref[1] and abs(cfl[0] - cref[0]) <= 1e-15 * cref[0]
    div = ch.calcMaxDiv()
    dref = case.max_div(u, v, w)
    assert div[1] == dref[1] and abs(div[0] - dref[0]) <= 1e-14 * dref[0]
    u2 = u.copy()
    u2[3, 4, 5] = np.nan
    ch.upload("u", u2)
    assert not ch.checkNaN("u")


# p tolerance per case.  p = Poisson(div(u*)/dt) amplifies round-off: the
# oracle itself, with 1e-16 relative noise injected after each Poisson solve
# (the size of FFT-algorithm rounding differences), drifts by 7-8e-13 in
# p - mean(p) after 5-10 steps at both sizes (tests/test_oracle_properties.py
# measures this floor), and 0.9-1.6e-12 at 32 x 24 x 16 after 10.  Which
# transform family the autotuner picks moves the GPU's p by as much
# (0.9-1.04e-12 seen at 128 x 64 x 64), so both cases hold p to about 2.5-4x
# the floor; u, v, w stay within 1e-12 (measured ~1e-15).
@pytest.mark.parametrize("nx,ny,nz,nsteps,p_tol", [(32, 24, 16, 5, 3e-12),
                                                    (128, 64, 64, 10, 2e-12)])
def test_step_parity(nx, ny, nz, nsteps, p_tol):
    """main.cc:116-154 for nsteps: fused GPU step vs the oracle loop."""
    case, ch = make_pair(nx, ny, nz)
    u, v, w = case.init_flow("poi", noise_intensity=0.1)
    for name, a in zip("uvw", (u, v, w)):
        ch.upload(name, a)
    ch.upload("p", case.zeros())
    u1, v1, w1, p = case.zeros(), case.zeros(), case.zeros(), case.zeros()
    case.step(u, v, w, u1, v1, w1, p, nsteps=nsteps)
    ch.step(nsteps)
    for name, a in zip("uvw", (u, v, w)):
        g = ch.download(name)
        e = rel_l2(g, a)
        assert e <= 1e-12, (name, e)
    gp = ch.download("p")
    e = rel_l2(demean(gp), demean(p))
    assert e <= p_tol, e
    div, _ = ch.calcMaxDiv()
    assert div < 1e-10
    # bulk velocity held at vel_force by the forcing
    assert abs(ch.Mean(var="u") - 1.0) < 1e-12


def test_step_matches_module_sequence(monkeypatch):
    """The fused graph step equals the reference's call sequence of entry
    points (the transform families pinned: the two contexts' autotuners could
    pick families whose results differ by rounding)."""
    from powerllel_channel_sycl_b200 import Channel
    monkeypatch.setenv("PLC_FFT_PLANS", "0,0")
    kwargs = case_kwargs(48, 32, 16)
    a = Channel(channel_params(**kwargs))
    b = Channel(channel_params(**kwargs))
    a.initFlow()
    b.initFlow()
    for _ in range(3):
        a.step(1)
        b.timeIntVelRK1()
        b.updateBoundVel(None, "u1", "v1", "w1")
        b.timeIntVelRK2()
        b.updateBoundVel()
        b.calcRHS()
        b.execute_poisson_solver()
        b.updateBoundP()
        b.correctVel()
        b.forceVel()
        b.updateBoundVel()
    for name in "uvw":
        assert rel_l2(a.download(name), b.download(name)) < 1e-13
    assert rel_l2(demean(a.download("p")), demean(b.download("p"))) < 1e-12


def test_step_forcing_read():
    """plc_step_forcing returns the forcing the fused step applied: forceVel's
    value in the reference's call sequence, mean + force = vel_force, and the
    mixed form's within FP32 rounding of the FP64 form's."""
    from powerllel_channel_sycl_b200 import Channel
    kwargs = case_kwargs(48, 32, 16)
    a = Channel(channel_params(**kwargs))
    b = Channel(channel_params(**kwargs))
    prm = channel_params(**kwargs)
    prm.precision = 1
    m32 = Channel(prm)
    for ch in (a, b, m32):
        ch.initFlow()
    for _ in range(3):
        a.step(1)
        m32.step(1)
        b.timeIntVelRK1()
        b.updateBoundVel(None, "u1", "v1", "w1")
        b.timeIntVelRK2()
        b.updateBoundVel()
        b.calcRHS()
        b.execute_poisson_solver()
        b.updateBoundP()
        b.correctVel()
        f_ref = b.forceVel()
        b.updateBoundVel()
        mean, force = a.step_forcing()
        assert abs(force[0] - f_ref[0]) <= 1e-12 * max(1.0, abs(f_ref[0])), (force, f_ref)
        assert mean[0] + force[0] == pytest.approx(kwargs["vel_force"][0], abs=1e-14)
        assert mean[1] == mean[2] == 0.0 and force[1] == force[2] == 0.0
        mean32, force32 = m32.step_forcing()
        assert abs(mean32[0] - mean[0]) < 1e-5 * abs(mean[0]), (mean32, mean)


def test_kernels_per_step():
    case, ch = make_pair(32, 24, 16)
    assert ch.kernels_per_step == 9


def test_fft_tiles_pinned_by_environment(monkeypatch):
    """PLC_FFT_TILES / PLC_FFT_TILES_F32 replace the tile autotuner."""
    from powerllel_channel_sycl_b200 import Channel, PlcError
    kw = case_kwargs(64, 48, 32)
    monkeypatch.setenv("PLC_FFT_TILES", "2,1,4")
    ch = Channel(channel_params(**kw))
    t = ch.fft_tiles
    assert (t["x_fwd"], t["x_bwd"], t["y"]) == (2, 1, 4)
    monkeypatch.setenv("PLC_FFT_TILES", "5,1,1")  # 5 does not divide ny/2 = 24
    with pytest.raises(PlcError):
        Channel(channel_params(**kw))
    monkeypatch.delenv("PLC_FFT_TILES")
    prm = channel_params(**kw)
    prm.precision = 1
    monkeypatch.setenv("PLC_FFT_TILES_F32", "3,3,3")  # odd y tiles are refused in FP32
    with pytest.raises(PlcError):
        Channel(prm)


@pytest.mark.parametrize("plans", ["0,0", "0,1", "1,0", "1,1"])
def test_fft_plan_families_pinned_by_environment(monkeypatch, plans):
    """PLC_FFT_PLANS / PLC_FFT_PLANS_F32 pin the radix plan families: the
    Poisson solve of every family matches the oracle in FP64, and the mixed
    form's projection is divergence-free with every family; a family a length
    does not have is refused."""
    from powerllel_channel_sycl_b200 import Channel, PlcError
    px, py = (int(x) for x in plans.split(","))
    nx, ny, nz = 96, 48, 8  # 96 = 4 x 24 and 48 = 2 x 24: both families in x and y
    monkeypatch.setenv("PLC_FFT_PLANS", plans)
    case, ch = make_pair(nx, ny, nz)
    t = ch.fft_tiles
    assert (t["plan_x"], t["plan_y"]) == (px, py)
    u, v, w = bc_fields(case, 9)
    p = case.zeros()
    case.calc_rhs(u, v, w, p)
    ch.upload("p", p)
    case.poisson(p)
    ch.execute_poisson_solver()
    assert rel_l2(demean(ch.download("p")), demean(p)) < 1e-12
    monkeypatch.setenv("PLC_FFT_PLANS_F32", plans)
    prm = channel_params(**case_kwargs(nx, ny, nz))
    prm.precision = 1
    m = Channel(prm)
    t = m.fft_tiles
    assert (t["plan_x"], t["plan_y"]) == (px, py)
    rng = np.random.default_rng(3)
    for q in "uvw":
        m.upload(q, rng.normal(size=m.shape))
    m.project()
    assert m.check()[2][0] < 1e-3
    monkeypatch.setenv("PLC_FFT_PLANS", "1,1")
    with pytest.raises(PlcError):  # 64 = 2^6 has no radix-24 family
        make_pair(64, 48, 8)


@pytest.mark.parametrize("vel_crf", [0.0, 0.35])
def test_transform2crf(vel_crf):
    """transform2CRF (mod_calcVel.cc:13-25): vel -= vel_crf on the interior
    only (halos untouched) and vel_force -= vel_crf, bit-identical to the
    oracle; a zero vel_crf leaves both as they are."""
    case, ch = make_pair(32, 24, 16)
    (u,) = random_fields(case, 11, n=1)
    ch.upload("u", u)
    vf_ref = oracle.C.c_double(1.25)
    oracle.lib().orc_transform2crf(case.gp, vel_crf, u, oracle.C.byref(vf_ref))
    vf = ch.transform2CRF(vel_crf, "u", 1.25)
    assert vf == vf_ref.value == 1.25 - vel_crf
    np.testing.assert_array_equal(ch.download("u"), u)
