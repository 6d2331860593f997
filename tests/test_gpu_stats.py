"""Statistics (mod_statistics) and monitors (mod_monitor) on the device
against the oracle restatement, on the same FP64 fields."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import case_kwargs, channel_params, oracle_case, random_fields, rel_l2

pytestmark = pytest.mark.gpu

NAMES = ("u", "v", "w", "u2", "v2", "w2", "uv", "uw", "vw", "p", "p2")


def make_pair(nx, ny, nz, precision=0, which=(1,) * 11, nt_init_stat=0, sample_interval=1,
              **kw):
    from powerllel_channel_sycl_b200 import Channel
    kwargs = case_kwargs(nx, ny, nz, **kw)
    prm = channel_params(**kwargs)
    prm.precision = precision
    for q, on in enumerate(which):
        prm.stat_which_var[q] = int(on)
    prm.nt_init_stat = nt_init_stat
    prm.sample_interval = sample_interval
    return oracle_case(**kwargs), Channel(prm)


def upload_state(case, ch, seed):
    """A channel state after a few oracle steps, with a random p."""
    u, v, w = case.init_flow("poi", noise_intensity=0.1)
    u1, v1, w1, p = case.zeros(), case.zeros(), case.zeros(), case.zeros()
    case.step(u, v, w, u1, v1, w1, p, nsteps=2)
    (p,) = random_fields(case, seed, n=1)
    for name, a in zip("uvwp", (u, v, w, p)):
        ch.upload(name, a)
    return u, v, w, p


@pytest.mark.parametrize("u_crf", [0.0, 0.25])
def test_calc_stat_bit_identical(u_crf):
    """Three samples of calcStat: every running sum bit-identical to the oracle."""
    case, ch = make_pair(32, 24, 16, u_crf=u_crf)
    ch.initStat()
    assert ch.stat_info == {"nts": 1, "nte": 0, "nspl": 0}
    sums = [np.zeros((16, 24, 32)) for _ in NAMES]
    for s in range(3):
        u, v, w, p = upload_state(case, ch, seed=10 + s)
        ch.calcStat(nt=s + 1)
        case.calc_stat_sample(u, v, w, p, sums)
    assert ch.stat_info == {"nts": 1, "nte": 3, "nspl": 3}
    for q, name in enumerate(NAMES):
        assert np.array_equal(ch.stat(name), sums[q]), name
    # plane means of the sums / samples
    prof = ch.stat_profiles()
    for q, name in enumerate(NAMES):
        ref = sums[q].mean(axis=(1, 2)) / 3
        assert np.allclose(prof[name], ref, rtol=1e-13, atol=1e-15), name


def test_stat_sampling_rule_and_subset():
    """Samples only when (nt - nt_init_stat) % sample_interval == 0; only the
    enabled statistics are kept."""
    which = (1, 0, 0, 1, 0, 0, 0, 0, 0, 0, 1)
    case, ch = make_pair(16, 12, 8, which=which, nt_init_stat=10, sample_interval=3)
    ch.initStat()
    upload_state(case, ch, seed=3)
    for nt in range(11, 20):
        ch.calcStat(nt)
    # nt = 13, 16, 19 sample
    assert ch.stat_info == {"nts": 11, "nte": 19, "nspl": 3}
    from powerllel_channel_sycl_b200 import PlcError
    with pytest.raises(PlcError):
        ch.stat("v")
    u = ch.stat("u")
    assert np.any(u != 0)
    # upload restores the sums and the counters (restart of the statistics)
    ch.set_stat("u", 2 * u, nts=5, nte=40, nspl=12)
    assert np.array_equal(ch.stat("u"), 2 * u)
    assert ch.stat_info == {"nts": 5, "nte": 40, "nspl": 12}


@pytest.mark.parametrize("u_crf", [0.0, 0.2])
def test_monitors_match_oracle(u_crf):
    case, ch = make_pair(32, 24, 16, u_crf=u_crf)
    u, v, w, p = upload_state(case, ch, seed=5)
    # skin friction at both walls (double-double plane sums on both sides)
    for wall, k in ((0, 1), (1, 16)):
        tau = case.wall_tau(u, k)
        ut, cf = ch.monitor_skf(wall)
        assert ut == np.sqrt(tau)
        assert cf == tau / 0.5
    # probe point
    out = ch.monitor_probe(7, 5, 3)
    assert np.array_equal(out, [u[3, 5, 7] + u_crf, v[3, 5, 7], w[3, 5, 7], p[3, 5, 7]])
    # bulk velocity of the forced component
    fm = ch.monitor_forcing()
    assert fm[0] == case.mean(u) + u_crf and fm[1] == 0.0 and fm[2] == 0.0
    # region extracts, staggered components centred, clipped to the domain
    region = (3, 40, 2, 9, 0, 5)
    clip = (3, 32, 2, 9, 1, 5)
    st, sz = (clip[0], clip[2], clip[4]), (clip[1] - clip[0] + 1, clip[3] - clip[2] + 1,
                                           clip[5] - clip[4] + 1)
    for field, arr, d in (("u", u, 1), ("v", v, 2), ("w", w, 3), ("p", p, 0)):
        got = ch.extract_region(region, field)
        ref = case.extract_region(arr, d, st, sz) + (u_crf if field == "u" else 0.0)
        assert np.array_equal(got, ref), field


def test_re_tau_of_laminar_profile():
    """Laminar Poiseuille flow with bulk velocity 1: tau_w = nu * dU/dz at the
    wall, U = 1.5 (1 - z^2) on the half height 1 gives tau_w = 3 nu."""
    case, ch = make_pair(16, 12, 64, stretch_ratio=0.0)
    nu = 1.0 / 2800.0
    z = case.zc_global[1:-1] - 1.0
    u = case.zeros()
    u[1:-1, 1:-1, 1:-1] = (1.5 * (1 - z ** 2))[:, None, None]
    ch.upload("u", u)
    ut0, _ = ch.monitor_skf(0)
    # the discrete wall gradient of the first cell centre over dz/2
    dz = case.dzf[1]
    assert abs(ut0 ** 2 - nu * 1.5 * (1 - z[0] ** 2) / (0.5 * dz)) < 1e-15
    assert abs(ut0 ** 2 / (3 * nu) - 1) < 0.05
    assert abs(ch.re_tau() / (np.sqrt(3 * nu) / nu) - 1) < 0.03


def test_mixed_form_statistics():
    """The mixed form's sums are FP64 sums of its FP32 fields."""
    case, ch = make_pair(32, 24, 16, precision=1)
    ch.initStat()
    u, v, w, p = upload_state(case, ch, seed=7)
    ch.calcStat(1)
    f32 = [a.astype(np.float32).astype(np.float64) for a in (u, v, w, p)]
    sums = [np.zeros((16, 24, 32)) for _ in NAMES]
    case.calc_stat_sample(*f32, sums)
    for q, name in enumerate(NAMES):
        assert rel_l2(ch.stat(name), sums[q]) < 1e-15, name
    ut, cf = ch.monitor_skf(1)
    assert abs(ut ** 2 / case.wall_tau(f32[0], 16) - 1) < 1e-14
