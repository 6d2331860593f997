"""The RK stages' z planes per block (autotuned among 8, 16, 24, 32; pinned
by PLC_RK_KCHUNK / PLC_RK_KCHUNK_F32) change which blocks compute which planes: three fused
steps of the FP64 form are bit-identical under every chunk, including one
that does not divide nz.  The mixed form's fused RK2 also sums the bulk
mean per block in FP32, so the chunk moves the forcing by FP32 rounding:
there the velocity agrees within 2e-6 relative L2 and the pressure, which
amplifies rounding about 1e4 times, within 5e-3 (the mixed form's bars)."""
import numpy as np
import pytest

from tests.helpers import case_kwargs, channel_params, demean, rel_l2

pytestmark = pytest.mark.gpu


def run(monkeypatch, kchunk, precision, nx=64, ny=48, nz=40):
    from powerllel_channel_sycl_b200 import Channel
    monkeypatch.setenv("PLC_FFT_PLANS", "0,0")
    monkeypatch.setenv("PLC_FFT_PLANS_F32", "0,0")
    var = "PLC_RK_KCHUNK_F32" if precision else "PLC_RK_KCHUNK"
    if kchunk is None:
        monkeypatch.delenv(var, raising=False)
    else:
        monkeypatch.setenv(var, str(kchunk))
    prm = channel_params(**case_kwargs(nx, ny, nz))
    prm.precision = precision
    ch = Channel(prm)
    k = ch.rk_kchunk
    ch.initFlow()
    ch.step(3)
    out = [ch.download(q) for q in "uvwp"]
    ch.close()
    return k, out


@pytest.mark.parametrize("precision", [0, 1])
def test_rk_chunk_changes_no_result(monkeypatch, precision):
    k_auto, ref = run(monkeypatch, None, precision)
    assert k_auto in (8, 16, 24, 32)
    for k in (8, 12, 32):
        got_k, out = run(monkeypatch, k, precision)
        assert got_k == k
        for q, a, b in zip("uvwp", out, ref):
            if precision == 0:
                np.testing.assert_array_equal(a, b)
            elif q != "p":
                assert rel_l2(a, b) <= 2e-6, (k, q)
            else:  # the pressure amplifies rounding ~1e4 (as the other mixed tests)
                assert rel_l2(demean(a), demean(b)) <= 5e-3, (k, q)


@pytest.mark.parametrize("value", ["0", "4", "33"])
def test_rk_chunk_pin_rejected(monkeypatch, value):
    """Pins outside 8..32 are refused (below 8 the mixed form's bulk-mean
    partials would not hold the blocks)."""
    from powerllel_channel_sycl_b200 import Channel, PlcError
    monkeypatch.setenv("PLC_RK_KCHUNK_F32", value)
    prm = channel_params(**case_kwargs(32, 24, 16))
    prm.precision = 1
    with pytest.raises(PlcError):
        Channel(prm)
