"""Known-answer and invariant tests of the oracle (CPU only).

They pin the oracle where the reference has no tests: a manufactured Poisson
solution, divergence after projection, bulk-flux forcing, the halo rules, the
laminar Poiseuille state and the round-off sensitivity of the pressure that
sets the parity tolerance of the GPU step tests.
"""
import numpy as np
import pytest

import oracle
from tests.helpers import demean, interior, rel_l2


def laplacian(case, phi):
    """The discrete operator of the Poisson solver (2nd-order, periodic x/y,
    Neumann z through the ghost rule p(0)=p(1), p(nz+1)=p(nz))."""
    p = phi.copy()
    case.update_bound_p(p)
    dx, dy = case.g.dx, case.g.dy
    dzf = case.dzf
    nz = case.nz
    out = np.zeros_like(p)
    c = p[1:-1, 1:-1, 1:-1]
    lap_xy = ((p[1:-1, 1:-1, 2:] - 2 * c + p[1:-1, 1:-1, :-2]) / dx**2 +
              (p[1:-1, 2:, 1:-1] - 2 * c + p[1:-1, :-2, 1:-1]) / dy**2)
    k = np.arange(1, nz + 1)
    a = 2.0 / (dzf[k] * (dzf[k - 1] + dzf[k]))
    cc = 2.0 / (dzf[k] * (dzf[k + 1] + dzf[k]))
    lap_z = (a[:, None, None] * (p[:-2, 1:-1, 1:-1] - c) + cc[:, None, None] * (p[2:, 1:-1, 1:-1] - c))
    out[1:-1, 1:-1, 1:-1] = lap_xy + lap_z
    return out


@pytest.mark.parametrize("nx,ny,nz", [(32, 24, 16), (48, 64, 32), (12, 6, 8)])
def test_poisson_manufactured(nx, ny, nz):
    case = oracle.Case(nx, ny, nz)
    x = (np.arange(nx) + 0.5) * case.g.dx
    y = (np.arange(ny) + 0.5) * case.g.dy
    z = case.zc_global[1:-1]
    phi = case.zeros()
    phi[1:-1, 1:-1, 1:-1] = (np.cos(2 * np.pi * x / case.lx)[None, None, :] *
                             np.sin(4 * np.pi * y / case.ly)[None, :, None] *
                             np.cos(np.pi * z / case.lz)[:, None, None] +
                             0.3 * np.cos(2 * np.pi * z / case.lz)[:, None, None])
    rhs = laplacian(case, phi)
    p = rhs.copy()
    case.poisson(p)
    assert rel_l2(demean(p), demean(phi)) < 1e-12


def test_divergence_after_projection_and_forcing():
    case = oracle.Case(64, 48, 32)
    u, v, w = case.init_flow("poi", noise_intensity=0.1)
    u1, v1, w1, p = case.zeros(), case.zeros(), case.zeros(), case.zeros()
    case.step(u, v, w, u1, v1, w1, p, nsteps=5)
    div, _ = case.max_div(u, v, w)
    assert div < 1e-11  # reference guard: div_limit 1e-9
    assert abs(case.mean(u) - 1.0) < 1e-13  # bulk velocity held at vel_force
    assert case.check_nan(u)


def test_init_bulk_rescale_quirk():
    """initFlow divides by Mean(nz, ny, ...) (mod_initFlow.cc:92): bulk = nz/nx."""
    case = oracle.Case(128, 64, 64)
    u, v, w = case.init_flow("poi", noise_intensity=0.1)
    assert abs(case.mean(u) - 64 / 128) < 1e-14


def test_halo_rules():
    case = oracle.Case(8, 6, 4, u_crf=0.2)
    rng = np.random.default_rng(0)
    u, v, w = (rng.standard_normal(case.shape) for _ in range(3))
    case.update_bound_vel(u, v, w)
    # periodic x and y (all rows, ghosts included)
    for q in (u, v, w):
        np.testing.assert_array_equal(q[:, :, 0], q[:, :, -2])
        np.testing.assert_array_equal(q[:, :, -1], q[:, :, 1])
        np.testing.assert_array_equal(q[:, 0, :], q[:, -2, :])
        np.testing.assert_array_equal(q[:, -1, :], q[:, 1, :])
    # no-slip: centred u (bc = -u_crf) and v, face w
    np.testing.assert_array_equal(u[0], 2.0 * (0.0 - 0.2) - u[1])
    np.testing.assert_array_equal(u[-1], 2.0 * (0.0 - 0.2) - u[-2])
    np.testing.assert_array_equal(v[0], -v[1])
    assert np.all(w[0] == 0.0) and np.all(w[-2] == 0.0) and np.all(w[-1] == 0.0)
    p = rng.standard_normal(case.shape)
    case.update_bound_p(p)
    np.testing.assert_array_equal(p[0], p[1])
    np.testing.assert_array_equal(p[-1], p[-2])


def test_laminar_poiseuille_near_stationary():
    """Without noise the laminar profile barely moves: the viscous term of a
    parabola is uniform and the bulk-preserving uniform forcing cancels it.
    nx == nz so that the initial bulk velocity is 1 (see the rescale quirk)."""
    case = oracle.Case(32, 12, 32, stretch_ratio=1.5)
    u, v, w = case.init_flow("poi", init_with_noise=False)
    u0 = u.copy()
    u1, v1, w1, p = case.zeros(), case.zeros(), case.zeros(), case.zeros()
    case.step(u, v, w, u1, v1, w1, p, nsteps=20)
    assert np.abs(v).max() < 1e-12 and np.abs(w).max() < 1e-12
    assert abs(case.mean(u) - 1.0) < 1e-13
    assert np.abs(interior(u) - interior(u0)).max() < 2e-3


def test_cfl_and_checks_known_values():
    case = oracle.Case(8, 6, 4)
    u, v, w = case.zeros(), case.zeros(), case.zeros()
    u[1:-1, 1:-1, 1:-1] = 1.0
    case.update_bound_vel(u, v, w)
    cfl, idx = case.max_cfl(u, v, w)
    assert abs(cfl - case.dt * 1.0 * case.g.dx_inv) < 1e-15
    assert idx == (1, 1, 1)  # first maximum of the k, j, i scan
    div, _ = case.max_div(u, v, w)
    assert div == 0.0
    u[3, 2, 4] = np.nan
    assert not case.check_nan(u)


def _run_with_noise(case, fields, nsteps, noise, seed):
    rng = np.random.default_rng(seed)
    u, v, w = (f.copy() for f in fields)
    u1, v1, w1, p = case.zeros(), case.zeros(), case.zeros(), case.zeros()
    for _ in range(nsteps):
        case.rk1(u, v, w, u1, v1, w1)
        case.update_bound_vel(u1, v1, w1)
        case.rk2(u, v, w, u1, v1, w1)
        case.update_bound_vel(u, v, w)
        case.calc_rhs(u, v, w, p)
        case.poisson(p)
        if noise:
            q = p[1:-1, 1:-1, 1:-1]
            q += np.std(q) * noise * rng.standard_normal(q.shape)
        case.update_bound_p(p)
        case.correct_vel(p, u, v, w)
        case.force_vel(u, v, w)
        case.update_bound_vel(u, v, w)
    return u, v, w, p


def test_pressure_roundoff_floor():
    """p - mean(p) after a few steps moves by ~1e-12 when each Poisson solve is
    perturbed at the 1e-16 level (FFT rounding): that floor, not the kernels,
    sets the p tolerance of the GPU step-parity tests, while the velocity
    stays within 1e-15."""
    case = oracle.Case(32, 24, 16)
    fields = case.init_flow("poi", noise_intensity=0.1)
    a = _run_with_noise(case, fields, 5, 0.0, 0)
    b = _run_with_noise(case, fields, 5, 1e-16, 1)
    floor_p = rel_l2(demean(b[3]), demean(a[3]))
    floor_u = rel_l2(b[0], a[0])
    assert 1e-13 < floor_p < 3e-12
    assert floor_u < 1e-15


def test_run_cfl_schedule():
    """orc_run_cfl: without a CFL target it is the fixed-dt loop; with one, dt
    is re-evaluated before step 1, after steps 1, 2, 4, 8 (below nt_check) and
    after every nt_check-th step, each time to cfl_target / rate, where
    rate * dt is calcMaxCFL's value."""
    case = oracle.Case(32, 24, 16)
    fields = case.init_flow("poi", noise_intensity=0.1)
    a = [f.copy() for f in fields] + [case.zeros() for _ in range(4)]
    b = [f.copy() for f in fields] + [case.zeros() for _ in range(4)]
    case.step(*a, nsteps=3)
    dts = case.run_cfl(*b, nsteps=3, nt_check=10, cfl_target=0.0)
    assert dts.tolist() == [case.dt] * 4
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    c = [f.copy() for f in fields] + [case.zeros() for _ in range(4)]
    rate0 = case.max_cfl(*c[:3])[0] / case.dt
    dts = case.run_cfl(*c, nsteps=12, nt_check=6, cfl_target=0.4)
    assert dts[0] == 0.4 / rate0
    # re-evaluated after steps 1, 2, 4 (below nt_check = 6) and 6, 12
    changes = [s for s in range(1, 13) if dts[s] != dts[s - 1]]
    assert set(changes) <= {1, 2, 4, 6, 12}, changes
    assert dts[3] == dts[2] and dts[5] == dts[4] and dts[7:12].tolist() == [dts[6]] * 5
    # the dt after the last step puts the final field at the target CFL
    rate = case.max_cfl(*c[:3])[0] / case.dt
    assert dts[12] == 0.4 / rate
