"""The Thomas sweep with its columns on chip (PLC_TRID=tile) against the
streaming sweep (PLC_TRID=stream) and the oracle.

The on-chip sweep copies 32 systems' columns into shared memory with bulk
copies and eliminates in place; it performs the streaming sweep's
operations in the same order, so both give bit-identical solutions in the
FP64 and the mixed form.  Against the oracle (ssolve_trid,
mod_poisson_solver.cc:317-357): within 1e-13 relative L2 on the regular
systems and 1e-9 on the singular (0,0) system, as the other solve tests.
Cases: nz from 2 to 256, including counts whose chunks of planes do
not divide them, and the lowest-wavenumber FP64 systems of the mixed form.
"""
import numpy as np
import pytest

import oracle
from tests.helpers import case_kwargs, channel_params, rel_l2

pytestmark = pytest.mark.gpu

SIZES = [(64, 48, 64), (32, 24, 16), (128, 64, 38), (96, 16, 2), (768, 8, 256), (64, 32, 6)]


def solve(monkeypatch, mode, nx, ny, nz, var, precision="fp64"):
    from powerllel_channel_sycl_b200 import Channel
    monkeypatch.setenv("PLC_TRID", mode)
    prm = channel_params(**case_kwargs(nx, ny, nz))
    if precision == "mixed":
        prm.precision = 1
    ch = Channel(prm)
    ch.upload("spec", var.reshape(nz, ny, nx))
    ch.solve_trid()
    out = ch.download("spec").ravel()
    ch.close()
    return out


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_tile_sweep_fp64(monkeypatch, nx, ny, nz):
    rng = np.random.default_rng(nz)
    var = rng.standard_normal(nx * ny * nz)
    tile = solve(monkeypatch, "tile", nx, ny, nz, var)
    stream = solve(monkeypatch, "stream", nx, ny, nz, var)
    np.testing.assert_array_equal(tile, stream)
    case = oracle.Case(**case_kwargs(nx, ny, nz))
    ref = var.copy()
    case.trid(ref)
    r3, g3 = ref.reshape(nz, ny, nx), tile.reshape(nz, ny, nx)
    mask = np.ones((ny, nx), bool)
    mask[0, 0] = False
    assert rel_l2(g3[:, mask], r3[:, mask]) < 1e-13
    assert rel_l2(g3[:, 0, 0], r3[:, 0, 0]) < 1e-9


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_tile_sweep_mixed(monkeypatch, nx, ny, nz):
    """The mixed form's projection (calcRHS, transforms, both sweeps of the
    Thomas solve with its FP64 low modes, correction) is bit-identical with
    the on-chip and the streaming sweep, the transform families pinned."""
    from powerllel_channel_sycl_b200 import Channel
    monkeypatch.setenv("PLC_FFT_PLANS_F32", "0,0")
    rng = np.random.default_rng(nz + 1)
    fields = [rng.uniform(-1, 1, (nz + 2, ny + 2, nx + 2)) for _ in range(3)]
    out = {}
    for mode in ("tile", "stream"):
        monkeypatch.setenv("PLC_TRID", mode)
        prm = channel_params(**case_kwargs(nx, ny, nz))
        prm.precision = 1
        m = Channel(prm)
        for name, a in zip("uvw", fields):
            m.upload(name, a)
        m.project()
        out[mode] = [m.download(name) for name in "uvwp"]
        m.close()
    for a, b in zip(out["tile"], out["stream"]):
        np.testing.assert_array_equal(a, b)


def test_trid_pin_rejected(monkeypatch):
    from powerllel_channel_sycl_b200 import Channel, PlcError
    monkeypatch.setenv("PLC_TRID", "onchip")
    with pytest.raises(PlcError):
        Channel(channel_params(**case_kwargs(32, 24, 16)))
