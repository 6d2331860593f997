"""GPU parity against the reference's own modules (FP64 form).

The CUDA library through its C ABI against the reference's time-step
modules compiled unmodified from its sources for the CPU
(``oracle.reference_modules``; the oneMKL DFT is the one stand-in that
restates a library's documented transform).  Same tolerances as the parity
tests against the oracle: stencils, boundary updates, calcRHS, correctVel
and the initial field bit-identical; the bulk mean within the error bound of
a sum in any order; 10 full steps of 128 x 64 x 64 within 1e-12 relative L2
in u, v, w and 2e-12 in p - mean(p) (the pressure's round-off floor under
FFT rounding differences).

Skipped when the reference build is absent (it is made from the reference's
sources, which only the build machine has).
"""
import os

import numpy as np
import pytest

import oracle
from oracle import reference_modules as refmod
from tests.helpers import case_kwargs, channel_params, demean, interior, rel_l2

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(refmod.LIB_PATH),
                                 reason="the reference build is absent")]


def triple(nx, ny, nz, **kw):
    from powerllel_channel_sycl_b200 import Channel
    kwargs = case_kwargs(nx, ny, nz, **kw)
    case = oracle.Case(**kwargs)
    ref = refmod.ReferenceModules(**kwargs)
    ch = Channel(channel_params(**kwargs))
    return case, ref, ch


@pytest.mark.parametrize("u_crf", [0.0, 0.3])
def test_stencils_bit_identical(u_crf):
    case, ref, ch = triple(48, 32, 16, u_crf=u_crf)
    rng = np.random.default_rng(21)
    u, v, w = (rng.uniform(-1, 1, case.shape) for _ in range(3))
    for name, a in zip("uvw", (u, v, w)):
        ref.set(name, a)
        ch.upload(name, a)
    ref.update_bound_vel(0)
    ch.updateBoundVel(u_crf)
    for name in "uvw":
        np.testing.assert_array_equal(ch.download(name), ref.get(name), err_msg=name)
    ref.rk1()
    ch.timeIntVelRK1(u_crf)
    for name in ("u1", "v1", "w1"):
        np.testing.assert_array_equal(interior(ch.download(name)), interior(ref.get(name)))
    ref.update_bound_vel(1)
    ch.updateBoundVel(u_crf, "u1", "v1", "w1")
    ref.rk2()
    ch.timeIntVelRK2(u_crf)
    for name in "uvw":
        np.testing.assert_array_equal(interior(ch.download(name)), interior(ref.get(name)))
    ref.update_bound_vel(0)
    ch.updateBoundVel(u_crf)
    ref.calc_rhs()
    ch.calcRHS()
    np.testing.assert_array_equal(interior(ch.download("p")), interior(ref.get("p")))
    q = rng.uniform(-1, 1, case.shape)
    ref.set("p", q)
    ch.upload("p", q)
    ref.update_bound_p()
    ch.updateBoundP()
    np.testing.assert_array_equal(ch.download("p"), ref.get("p"))
    ref.correct_vel()
    ch.correctVel()
    for name in "uvw":
        np.testing.assert_array_equal(interior(ch.download(name)), interior(ref.get(name)))
    ref.close()


def test_init_flow_and_steps():
    case, ref, ch = triple(128, 64, 64)
    ru, rv, rw = ref.init_flow("poi", noise_intensity=0.1)
    ch.initFlow()
    np.testing.assert_array_equal(ch.download("v"), rv)
    np.testing.assert_array_equal(ch.download("w"), rw)
    # u is rescaled by 1/Mean: the two means lie within the sum's error bound
    gu = ch.download("u")
    assert np.max(np.abs(gu - ru) / np.maximum(np.abs(ru), 1e-300)) <= 1e-13
    # continue both from the reference's field
    ch.upload("u", ru)
    ch.upload("p", case.zeros())
    ref.set("p", case.zeros())
    ref.step(10)
    ch.step(10)
    errs = {name: rel_l2(ch.download(name), ref.get(name)) for name in "uvw"}
    errs["p"] = rel_l2(demean(ch.download("p")), demean(ref.get("p")))
    print("128x64x64, 10 steps, GPU vs the reference's modules:", errs)
    for name in "uvw":
        assert errs[name] <= 1e-12, errs
    assert errs["p"] <= 2e-12, errs
    ref.close()
