"""plc_mean_noalloc: the bulk mean for callers that cannot allocate device memory.

Such callers (an application that owns all GPU memory in its own pool, or a
time loop that must not take cudaMalloc's implicit synchronisation) pass
their own device buffers; the entry point keeps its partial sums in a static
array of the library.  This test calls it through the C ABI on buffers owned
by a context, twice in a row (the array keeps the previous call's contents),
and checks each result against plc_mean and the oracle to within a relative
2e-16 (both accumulate in double-double, over different reduction trees, so
the rounded totals agree to about an ulp).

The file name sorts last so that a run stopping at the first failure has run
every other test before this one.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from tests.helpers import case_kwargs, channel_params

pytestmark = pytest.mark.gpu


# the second shape is a thin channel: each plane is split over many blocks
@pytest.mark.parametrize("nx,ny,nz", [(48, 32, 24), (256, 192, 4)])
def test_mean_noalloc_matches_plc_mean(nx, ny, nz):
    from powerllel_channel_sycl_b200 import Channel
    from powerllel_channel_sycl_b200._lib import lib

    kw = case_kwargs(nx, ny, nz)
    case = oracle.Case(**kw)
    ch = Channel(channel_params(**kw))
    L = lib()
    rng = np.random.default_rng(31)
    # the caller's own device buffers: dzflzi and the output live in the
    # context's spectral array, the fields in the context's u and v
    spec = np.zeros((nz, ny, nx))
    flat = spec.reshape(-1)
    flat[: nz + 2] = case.dzflzi
    ch.upload("spec", spec)
    base = ch.ptr("spec")
    d_dzflzi = base
    d_out = base + 8 * (nz + 8)
    stream = ch.stream
    for call, field in enumerate(("u", "v")):
        q = rng.uniform(-1.0, 2.0, case.shape)
        ch.upload(field, q)
        expect = ch.Mean(var=field)
        rc = L.plc_mean_noalloc(ch.ptr(field), d_dzflzi, nx, ny, nz, nx, ny, d_out, stream)
        assert rc == 0, L.plc_last_error(None)
        got = ch.download("spec").reshape(-1)[nz + 8]
        assert abs(got - expect) <= 2e-16 * abs(expect), (call, got, expect)
        ref = case.mean(q)
        assert abs(got - ref) <= 2e-16 * abs(ref), (call, got, ref)


def test_mean_noalloc_rejects_bad_sizes():
    from powerllel_channel_sycl_b200._lib import lib
    L = lib()
    fake = 1 << 40  # never dereferenced: the size check comes first
    assert L.plc_mean_noalloc(fake, fake, 8, 8, 8193, 8, 8, fake, None) == -2
    assert b"8192" in L.plc_last_error(None)
    assert L.plc_mean_noalloc(None, fake, 8, 8, 8, 8, 8, fake, None) == -1
    assert L.plc_mean_noalloc(fake, fake, 0, 8, 8, 8, 8, fake, None) == -1
