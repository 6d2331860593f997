"""The oracle pinned to the reference's own code (CPU).

``oracle.reference_modules`` runs the reference's time-step modules,
compiled unmodified from its sources against host stand-ins for SYCL,
one-rank MPI, the oneMKL DFT and oneDPL (``oracle/reference_cpu``).  Every
function of the oracle restatement is checked against the reference's own
function on the same seeded inputs:

* bit-identical: mesh coefficients, eigenvalues, the boundary updates, RK1,
  RK2, calcRHS, correctVel, transform2CRF, the CFL and divergence maxima with
  their indices, the NaN check, the Thomas sweep, and the initial v and w;
* within the error bound of a sum in any order (Higham: n eps sum|terms|):
  the bulk mean and what depends on it (forceVel, the rescaled initial u) --
  the reference leaves the order of the sum to its SYCL reduction, the
  oracle sums in double-double;
* within 1e-14 relative L2: each FFT direction (the reference's DFT is
  oneMKL's, here the stand-in's mixed-radix FFT; the oracle has its own);
* within 1e-12 relative L2: the Poisson solve (p - mean(p)) and 10 full time
  steps of main.cc's loop (u, v, w; p - mean(p) within 2e-12, the pressure's
  round-off floor under FFT rounding differences).

The FFT is the one stage whose arithmetic is not the reference's own here:
oneMKL is closed source and absent, so its transforms are restated from
their documented definition in the stand-in.

Skipped when neither the reference build nor the reference sources exist
(a machine without them runs the other oracle tests only).
"""
import numpy as np
import pytest

import oracle
from oracle import reference_modules as refmod
from tests.helpers import case_kwargs, demean, interior, rel_l2

pytestmark = pytest.mark.skipif(not refmod.available(),
                                reason="the reference build and sources are absent")

SIZES = [(32, 24, 16), (48, 32, 8), (6, 4, 2)]


def pair(nx, ny, nz, **kw):
    kwargs = case_kwargs(nx, ny, nz, **kw)
    case = oracle.Case(**kwargs)
    ref = refmod.ReferenceModules(**{k: v for k, v in kwargs.items()})
    return case, ref


def seeded(case, seed, n=3):
    rng = np.random.default_rng(seed)
    return [rng.uniform(-1.0, 1.0, case.shape) for _ in range(n)]


def sum_bound(case, var, nxg=None, nyg=None):
    """Higham's bound for a recursive sum of the mean's n terms,
    n * eps * sum |var * dzflzi| / (nx_global * ny_global): how far a sum in
    any order may lie from the exact mean."""
    q = interior(var) * case.dzflzi[1:-1, None, None]
    n = q.size
    return n * np.finfo(np.float64).eps * np.abs(q).sum() / (nxg or case.nx) / (nyg or case.ny)


def ulps(a, b):
    a = np.atleast_1d(np.asarray(a, dtype=np.float64))
    b = np.atleast_1d(np.asarray(b, dtype=np.float64))
    scale = np.maximum(np.abs(a), np.abs(b))
    scale[scale == 0] = 1.0
    return float(np.max(np.abs(a - b) / (scale * np.finfo(np.float64).eps)))


@pytest.mark.parametrize("nx,ny,nz", SIZES)
@pytest.mark.parametrize("stretch", [1.5, 0.0])
def test_mesh(nx, ny, nz, stretch):
    case, ref = pair(nx, ny, nz, stretch_ratio=stretch)
    for name in ["dzf_global", "dzf", "dzf_inv", "dzc", "dzc_inv", "dzflzi", "zc_global"]:
        np.testing.assert_array_equal(ref.mesh(name), getattr(case, name), err_msg=name)
    dx, dy, dxi, dyi = ref.dxy()
    assert (dx, dy, dxi, dyi) == (case.g.dx, case.g.dy, case.g.dx_inv, case.g.dy_inv)
    np.testing.assert_array_equal(ref.eigen_values(nx), oracle.eigen_values(nx))
    ref.close()


@pytest.mark.parametrize("nx,ny,nz", SIZES)
@pytest.mark.parametrize("u_crf", [0.0, 0.25])
def test_update_bound(nx, ny, nz, u_crf):
    case, ref = pair(nx, ny, nz, u_crf=u_crf)
    u, v, w, p = seeded(case, 1, 4)
    for name, a in zip("uvw", (u, v, w)):
        ref.set(name, a)
    ref.set("p", p)
    case.update_bound_vel(u, v, w)
    case.update_bound_p(p)
    ref.update_bound_vel(0)
    ref.update_bound_p()
    for name, a in zip("uvwp", (u, v, w, p)):
        np.testing.assert_array_equal(ref.get(name), a, err_msg=name)
    ref.close()


@pytest.mark.parametrize("nx,ny,nz", SIZES)
@pytest.mark.parametrize("u_crf", [0.0, 0.3])
def test_rk1_rk2(nx, ny, nz, u_crf):
    case, ref = pair(nx, ny, nz, u_crf=u_crf)
    u, v, w = seeded(case, 2)
    case.update_bound_vel(u, v, w)
    for name, a in zip("uvw", (u, v, w)):
        ref.set(name, a)
    u1, v1, w1 = case.zeros(), case.zeros(), case.zeros()
    case.rk1(u, v, w, u1, v1, w1)
    ref.rk1()
    for name, a in zip(("u1", "v1", "w1"), (u1, v1, w1)):
        np.testing.assert_array_equal(interior(ref.get(name)), interior(a), err_msg=name)
    case.update_bound_vel(u1, v1, w1)
    ref.update_bound_vel(1)
    for name, a in zip(("u1", "v1", "w1"), (u1, v1, w1)):
        np.testing.assert_array_equal(ref.get(name), a, err_msg=name)
    case.rk2(u, v, w, u1, v1, w1)
    ref.rk2()
    for name, a in zip("uvw", (u, v, w)):
        np.testing.assert_array_equal(interior(ref.get(name)), interior(a), err_msg=name)
    ref.close()


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_calc_rhs_correct_force(nx, ny, nz):
    case, ref = pair(nx, ny, nz)
    u, v, w, q = seeded(case, 3, 4)
    case.update_bound_vel(u, v, w)
    for name, a in zip("uvw", (u, v, w)):
        ref.set(name, a)
    p = case.zeros()
    case.calc_rhs(u, v, w, p)
    ref.calc_rhs()
    np.testing.assert_array_equal(interior(ref.get("p")), interior(p))
    case.update_bound_p(q)
    ref.set("p", q)
    case.correct_vel(q, u, v, w)
    ref.correct_vel()
    for name, a in zip("uvw", (u, v, w)):
        np.testing.assert_array_equal(interior(ref.get(name)), interior(a), err_msg=name)
    # the bulk mean: the reference's SYCL reduction (summation order left to
    # the implementation) against the oracle's double-double sum, within the
    # error bound of a sum in any order
    bu = sum_bound(case, u)
    assert abs(ref.mean("u") - case.mean(u)) <= bu
    assert abs(ref.mean("v", 17, 5) - case.mean(v, 17, 5)) <= sum_bound(case, v, 17, 5)
    case.force_vel(u, v, w)
    ref.force_vel()
    assert np.max(np.abs(interior(ref.get("u")) - interior(u))) <= bu + 4e-16
    np.testing.assert_array_equal(ref.get("v"), v)
    np.testing.assert_array_equal(ref.get("w"), w)
    ref.close()


@pytest.mark.parametrize("vel_crf", [0.0, 0.35])
def test_transform2crf(vel_crf):
    case, ref = pair(32, 24, 16)
    (u,) = seeded(case, 4, 1)
    ref.set("u", u)
    f = ref.transform2crf("u", vel_crf, 1.25)
    vf = oracle.C.c_double(1.25)
    oracle.lib().orc_transform2crf(case.gp, vel_crf, u, oracle.C.byref(vf))
    assert f == vf.value
    np.testing.assert_array_equal(ref.get("u"), u)
    ref.close()


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_checks(nx, ny, nz):
    case, ref = pair(nx, ny, nz)
    u, v, w = seeded(case, 5)
    case.update_bound_vel(u, v, w)
    for name, a in zip("uvw", (u, v, w)):
        ref.set(name, a)
    assert ref.max_cfl() == case.max_cfl(u, v, w)
    assert ref.max_div() == case.max_div(u, v, w)
    assert ref.check_nan("u") and case.check_nan(u)
    u[2, 1, 3] = np.nan
    ref.set("u", u)
    assert not ref.check_nan("u") and not case.check_nan(u)
    ref.close()


@pytest.mark.parametrize("nx,ny,nz", SIZES + [(96, 48, 8), (64, 12, 4)])
def test_fft_and_trid(nx, ny, nz):
    case, ref = pair(nx, ny, nz)
    (p,) = seeded(case, 6, 1)
    ref.set("p", p)
    n = nx * ny * nz
    var_o, var_r = np.zeros(n), np.zeros(n)
    case.fft_fwd_x(p, var_o)
    ref.fft_fwd_x(var_r)
    assert rel_l2(var_r, var_o) < 1e-14
    case.fft_fwd_y(var_o)
    ref.fft_fwd_y(var_r)
    assert rel_l2(var_r, var_o) < 1e-14
    # the Thomas sweep on the same input: the same operations in the same order
    t_o, t_r = var_o.copy(), var_o.copy()
    case.trid(t_o)
    ref.trid(t_r)
    np.testing.assert_array_equal(t_r, t_o)
    case.fft_bwd_y(var_o)
    ref.fft_bwd_y(var_r)
    assert rel_l2(var_r, var_o) < 1e-14
    q = case.zeros()
    case.fft_bwd_x(var_o, q)
    ref.fft_bwd_x(var_r)
    assert rel_l2(interior(ref.get("p")), interior(q)) < 1e-14
    ref.close()


@pytest.mark.parametrize("nx,ny,nz", SIZES + [(128, 64, 64)])
def test_poisson(nx, ny, nz):
    case, ref = pair(nx, ny, nz)
    u, v, w = seeded(case, 7)
    case.update_bound_vel(u, v, w)
    p = case.zeros()
    case.calc_rhs(u, v, w, p)
    ref.set("p", p)
    case.poisson(p)
    ref.poisson()
    assert rel_l2(demean(ref.get("p")), demean(p)) < 1e-12
    ref.close()


@pytest.mark.parametrize("field,u_crf", [("poi", 0.0), ("log", 0.0), ("uni", 0.2)])
def test_init_flow(field, u_crf):
    case, ref = pair(32, 24, 16, u_crf=u_crf)
    u, v, w = case.init_flow(field, u0=1.0, noise_intensity=0.1)
    ru, rv, rw = ref.init_flow(field, u0=1.0, noise_intensity=0.1)
    np.testing.assert_array_equal(rv, v)
    np.testing.assert_array_equal(rw, w)
    # u of "poi"/"log" is rescaled by 1/Mean(u): the two means differ within
    # the error bound of their sums (4.5e-14 relative for these 12288 terms of
    # one sign), and the rescaled fields by as much
    if field != "uni":
        rel = np.max(np.abs(ru - u) / np.abs(u))
        assert rel <= 12288 * np.finfo(np.float64).eps + 4e-16, rel
    else:
        np.testing.assert_array_equal(ru, u)
    assert ref.vel_force(0) == 1.0 - u_crf
    ref.close()


# p tolerance per case: the oracle's own p - mean(p) moves by 0.9-1.6e-12
# (32x24x16) and 0.7e-12 (128x64x64) after 10 steps when each Poisson solve is
# perturbed by 1e-16 relative noise, the size of the rounding differences
# between two FFT implementations; the bars are 2.5-3x those floors
@pytest.mark.parametrize("nx,ny,nz,nsteps,p_tol", [(32, 24, 16, 10, 4e-12),
                                                    (128, 64, 64, 10, 2e-12)])
def test_steps(nx, ny, nz, nsteps, p_tol):
    """main.cc:116-154 for nsteps: the reference's modules against the oracle
    loop, from the same initial field."""
    case, ref = pair(nx, ny, nz)
    u, v, w = case.init_flow("poi", noise_intensity=0.1)
    for name, a in zip("uvw", (u, v, w)):
        ref.set(name, a)
    u1, v1, w1, p = case.zeros(), case.zeros(), case.zeros(), case.zeros()
    case.step(u, v, w, u1, v1, w1, p, nsteps=nsteps)
    ref.step(nsteps)
    errs = {name: rel_l2(ref.get(name), a) for name, a in zip("uvw", (u, v, w))}
    errs["p"] = rel_l2(demean(ref.get("p")), demean(p))
    print(f"{nx}x{ny}x{nz}, {nsteps} steps, reference modules vs oracle:", errs)
    for name in "uvw":
        assert errs[name] <= 1e-12, errs
    assert errs["p"] <= p_tol, errs
    ref.close()
