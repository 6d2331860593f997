"""The oracle's building blocks against the golden fixtures (CPU only).

The fixtures come from independent implementations (numpy FFT, scipy banded
solver, numpy-evaluated formulas); see tests/golden/make_golden.py.
"""
import os

import numpy as np
import pytest

import oracle

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLD, name))


@pytest.mark.parametrize("n", [2, 4, 6, 8, 12, 16, 24, 48, 64, 96, 128, 192, 256, 384, 768])
def test_packed_rfft_vs_numpy(n):
    g = load("fft_packed.npz")
    x, X = g[f"x{n}"], g[f"X{n}"]
    out = oracle.rfft_packed(x)
    assert np.abs(out - X).max() <= 1e-14 * max(1.0, np.abs(X).max())
    back = oracle.irfft_packed(out) / n
    assert np.abs(back - x).max() <= 1e-14 * max(1.0, np.abs(x).max())


@pytest.mark.parametrize("n", [2, 4, 6, 8, 12, 16, 24, 48, 64, 96, 128, 192, 256, 384, 768])
def test_eigen_values(n):
    g = load("eigen.npz")
    lam = oracle.eigen_values(n)
    np.testing.assert_allclose(lam, g[f"n{n}"], rtol=0, atol=1e-15)


@pytest.mark.parametrize("key", ["nz64_r1.5_f0", "nz128_r3.0_f0", "nz256_r1.8_f0", "nz48_r1.2_f1"])
def test_mesh(key):
    g = load("mesh.npz")
    nz = int(key.split("_")[0][2:])
    ratio = float(key.split("_")[1][1:])
    func = int(key.split("_")[2][1:])
    c = oracle.Case(8, 8, nz, lz=2.0, stretch_ratio=ratio, stretch_func=func)
    # dzf is a difference of face positions: numpy's and libm's tanh/sin may
    # differ by one ulp of zf (<= 2.2e-16 * lz), hence the absolute bound
    np.testing.assert_allclose(c.dzf_global, g[key], rtol=0, atol=1e-15)
    # the stretched mesh spans the channel height exactly
    assert abs(c.dzf_global[1:-1].sum() - 2.0) < 1e-13


def test_thomas_vs_banded_solve():
    """ssolve_trid on single systems against scipy.linalg.solve_banded."""
    g = load("trid.npz")
    dzf = g["dzf"]
    nz = dzf.size - 2
    for lam in [-1.0, -37.5, -4000.0]:
        # one (kx,ky) system with eigenvalue lam: a 2x2 grid whose packed
        # index (1,0) carries lam_x(n/2)/dx^2 + 0 = -4/dx^2 (nx = 2): choose dx
        nx, ny = 2, 2
        dx = np.sqrt(4.0 / -lam)
        c = oracle.Case(nx, ny, nz, lx=nx * dx, ly=ny * 1.0, lz=2.0, dzf_global=dzf)
        var = np.zeros((nz, ny, nx))
        var[:, 0, 1] = g[f"lam{lam}_rhs"]
        flat = var.ravel().copy()
        c.trid(flat)
        sol = flat.reshape(nz, ny, nx)[:, 0, 1]
        ref = g[f"lam{lam}_sol"]
        assert np.abs(sol - ref).max() <= 1e-12 * np.abs(ref).max()


def test_noise_generator():
    g = load("init_noise.npz")
    for seed in (123, 456, 789):
        for off, val in zip(g["offsets"], g[f"seed{seed}"]):
            assert oracle.lib().orc_noise_uniform(seed, int(off)) == val
