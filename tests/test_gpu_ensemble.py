"""Batched ensembles on one GPU: every schedule, and the launches of several
steps per member branch between host events, give each member exactly the
fields it gets stepping alone; the autotuner restores the state it
advances; checks stay per member."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import case_kwargs, channel_params

pytestmark = pytest.mark.gpu

MEMBERS = [  # (nx, ny, nz, precision, re)
    (64, 48, 48, 0, 2800.0),
    (32, 24, 16, 1, 1800.0),
    (96, 64, 32, 1, 4000.0),
    (48, 32, 24, 0, 1000.0),
]


def member_params(nx, ny, nz, precision, re, **extra):
    prm = channel_params(**case_kwargs(nx, ny, nz, re=re))
    prm.precision = precision
    for k, v in extra.items():
        setattr(prm, k, v)
    return prm


def standalone(spec, nsteps, **extra):
    from powerllel_channel_sycl_b200 import Channel
    ch = Channel(member_params(*spec, **extra))
    ch.initFlow()
    ch.step(nsteps)
    return {q: ch.download(q) for q in "uvwp"}


@pytest.fixture(scope="module", autouse=True)
def pinned_fft_families():
    """The transform families pinned for the whole module: the autotuner of
    each context may pick different families (whose results differ by
    rounding) for a member and for the same channel alone."""
    with pytest.MonkeyPatch.context() as mp:
        mp.setenv("PLC_FFT_PLANS", "0,0")
        mp.setenv("PLC_FFT_PLANS_F32", "0,0")
        yield


@pytest.fixture(scope="module")
def alone(pinned_fft_families):
    return [standalone(s, 6, nt_check=3, cfl_limit=10.0, div_limit=1e-8) for s in MEMBERS]


@pytest.mark.parametrize("schedule", ["concurrent", "proportional", "two_groups", "sequential"])
def test_members_match_standalone(alone, schedule):
    from powerllel_channel_sycl_b200 import Ensemble
    ens = Ensemble([member_params(*s, nt_check=3, cfl_limit=10.0, div_limit=1e-8)
                    for s in MEMBERS])
    ens.set_schedule(schedule)
    name, groups, budgets = ens.schedule()
    assert name == schedule
    if schedule == "sequential":
        assert sorted(groups) == list(range(len(MEMBERS)))
    if schedule == "proportional":
        assert sum(budgets) <= 148 + len(MEMBERS) and min(budgets) >= 1
    ens.initFlow()
    ens.step(4)
    ens.step(2)
    for m, ref in zip(ens.members, alone):
        assert m.step_count == 6
        for q in "uvwp":
            assert np.array_equal(m.download(q), ref[q]), (schedule, q)
    ens.close()


def test_autotune_restores_state(alone):
    from powerllel_channel_sycl_b200 import Ensemble
    ens = Ensemble([member_params(*s, nt_check=3, cfl_limit=10.0, div_limit=1e-8)
                    for s in MEMBERS])
    ens.initFlow()
    ens.step(3)
    before = [{q: m.download(q) for q in "uvwp"} for m in ens.members]
    times = ens.autotune(steps=3)
    assert set(times) == {"concurrent", "proportional", "two_groups", "sequential"}
    assert all(t is not None and t > 0 for t in times.values())
    best = min(times, key=times.get)
    assert ens.schedule()[0] == best
    for m, b in zip(ens.members, before):
        assert m.step_count == 3
        for q in "uvwp":
            assert np.array_equal(m.download(q), b[q]), q
    ens.step(3)  # and the run continues exactly as without the tuning
    for m, ref in zip(ens.members, alone):
        for q in "uvw":
            assert np.array_equal(m.download(q), ref[q]), q


def test_member_check_failure_names_the_member():
    from powerllel_channel_sycl_b200 import Ensemble, PlcError
    prms = [member_params(*MEMBERS[0], nt_check=2, cfl_limit=10.0, div_limit=1e-8),
            member_params(*MEMBERS[3], nt_check=2, cfl_limit=10.0, div_limit=1e-300)]
    ens = Ensemble(prms)
    ens.initFlow()
    with pytest.raises(PlcError) as e:
        ens.step(4)
    assert e.value.code == -5 and "member 1" in str(e.value) and "checkDiv" in str(e.value)


def test_ensemble_cfl_controlled_dt():
    from powerllel_channel_sycl_b200 import Ensemble
    prms = [member_params(*s, nt_check=4, cfl_limit=1.0, div_limit=1e-3, cfl_target=0.4)
            for s in MEMBERS[:3]]
    ens = Ensemble(prms)
    ens.initFlow()
    ens.step(12)
    for m in ens.members:
        ok, cfl, div = m.check()
        assert ok and 0.2 < cfl[0] < 0.5


def test_ensemble_timed_and_throughput():
    """16 uneven channels: one graph launch per ensemble step beats stepping
    the members one after another."""
    from powerllel_channel_sycl_b200 import Ensemble
    rng = np.random.default_rng(1)
    specs = []
    for _ in range(16):
        nx = int(rng.choice([64, 96, 128]))
        ny = int(rng.choice([48, 64, 96]))
        nz = int(rng.choice([48, 64]))
        re_tau = rng.uniform(120, 400)
        specs.append((nx, ny, nz, 1, 0.5 * (re_tau / 0.09) ** (1 / 0.88)))
    ens = Ensemble([member_params(*s, dt=1e-4) for s in specs])
    ens.initFlow()
    times = ens.autotune(steps=5)
    assert times["concurrent"] < times["sequential"] or times["proportional"] < times["sequential"]
    ms = ens.step_timed(10) / 10
    assert ms > 0
