"""Batched ensembles on one GPU: every schedule -- the members as graph
branches, or (batched) each stage of the mixed-form members' step as one
launch over all of them -- and the launches of several steps between host
events, give each member exactly the fields it gets stepping alone; a member
stepped in an ensemble matches the oracle; the autotuner restores the state
it advances; checks stay per member."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from helpers import case_kwargs, channel_params, demean, rel_l2

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
    """The transform families and the RK stages' z chunk pinned for the whole
    module: the autotuner of each context may pick different families (whose
    results differ by rounding) or, in the mixed form, chunks (which change
    the FP32 rounding of the bulk-mean partials) for a member and for the
    same channel alone."""
    with pytest.MonkeyPatch.context() as mp:
        mp.setenv("PLC_FFT_PLANS", "0,0")
        mp.setenv("PLC_FFT_PLANS_F32", "0,0")
        mp.setenv("PLC_RK_KCHUNK", "8")
        mp.setenv("PLC_RK_KCHUNK_F32", "8")
        yield


@pytest.fixture(scope="module")
def alone(pinned_fft_families):
    return [standalone(s, 6, nt_check=3, cfl_limit=10.0, div_limit=1e-8) for s in MEMBERS]


@pytest.mark.parametrize("schedule", ["concurrent", "proportional", "two_groups", "sequential",
                                      "batched"])
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
    assert set(times) == {"concurrent", "proportional", "two_groups", "sequential", "batched"}
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


# mixed-form members for the batched launches: lengths shared by several
# members (one launch each), lengths without a compiled plan (36, 24: the
# runtime plan), and x lengths that are not multiples of the 32-column RK tile
MIXED = [(64, 48, 48), (64, 64, 32), (96, 48, 32), (32, 24, 16), (36, 24, 16), (48, 32, 24)]


@pytest.fixture(scope="module")
def mixed_alone(pinned_fft_families):
    specs = [(nx, ny, nz, 1, 1000.0 + 400.0 * q) for q, (nx, ny, nz) in enumerate(MIXED)]
    kw = dict(nt_check=3, cfl_limit=10.0, div_limit=1e-8)
    return specs, kw, [standalone(s, 7, **kw) for s in specs]


@pytest.mark.parametrize("chains", [1, 2])
@pytest.mark.parametrize("pdl", [False, True])
def test_batched_mixed_members_match_standalone(mixed_alone, chains, pdl):
    """With one or two chains, with or without programmatic dependent
    launch of the batched kernels: each member as alone."""
    from powerllel_channel_sycl_b200 import Ensemble
    specs, kw, ref = mixed_alone
    ens = Ensemble([member_params(*s, **kw) for s in specs])
    ens.set_schedule("batched")
    ens.set_batch_chains(chains)
    ens.set_batch_pdl(pdl)
    assert ens.batch_choice()["chains"] == chains
    assert ens.batch_choice()["pdl"] == pdl
    ens.initFlow()
    ens.step(5)
    ens.step(2)
    for q, (m, r) in enumerate(zip(ens.members, ref)):
        assert m.step_count == 7
        for f in "uvwp":
            assert np.array_equal(m.download(f), r[f]), (specs[q], f)
    ens.close()


def test_batched_two_pass_y_transforms(monkeypatch):
    """The batched schedule's y transforms in the two-pass family (pinned as
    the members' own): each member as alone."""
    from powerllel_channel_sycl_b200 import Ensemble
    monkeypatch.setenv("PLC_FFT_PLANS_F32", "0,3")
    specs = [(64, 48, 48, 1, 1500.0), (64, 64, 32, 1, 2000.0), (96, 48, 32, 1, 2500.0),
             (32, 96, 16, 1, 1800.0)]
    kw = dict(nt_check=3, cfl_limit=10.0, div_limit=1e-8)
    ref = [standalone(s, 5, **kw) for s in specs]
    ens = Ensemble([member_params(*s, **kw) for s in specs])
    assert all(m.fft_tiles["plan_y"] == 3 for m in ens.members)
    ens.set_schedule("batched")
    ens.initFlow()
    ens.step(5)
    for m, r, spec in zip(ens.members, ref, specs):
        for f in "uvwp":
            assert np.array_equal(m.download(f), r[f]), (spec, f)
    ens.close()


def test_batched_more_members_than_one_launch_holds():
    """40 mixed-form members: the batched stages take two launches each (32
    members' arguments per launch); every member still steps as alone."""
    from powerllel_channel_sycl_b200 import Ensemble
    kw = dict(nt_check=3, cfl_limit=10.0, div_limit=1e-8)
    specs = [(32, 24, 16, 1, 1000.0 + 50.0 * q) for q in range(40)]
    ref = {q: standalone(specs[q], 4, **kw) for q in (0, 31, 32, 39)}
    ens = Ensemble([member_params(*s, **kw) for s in specs])
    ens.set_schedule("batched")
    ens.initFlow()
    ens.step(4)
    for q, r in ref.items():
        for f in "uvwp":
            assert np.array_equal(ens.members[q].download(f), r[f]), (q, f)
    ens.close()


@pytest.mark.parametrize("trid", ["tile", "stream"])
def test_batched_thomas_sweeps(monkeypatch, trid):
    """The batched schedule's Thomas sweep, on chip or streamed (pinned by
    PLC_TRID as the channels' own), after the batch autotuner: each member as
    alone with the same sweep."""
    from powerllel_channel_sycl_b200 import Ensemble
    monkeypatch.setenv("PLC_TRID", trid)
    specs = [(64, 48, 48, 1, 1500.0), (96, 64, 32, 1, 2500.0), (32, 24, 16, 1, 1800.0)]
    kw = dict(nt_check=3, cfl_limit=10.0, div_limit=1e-8)
    ref = [standalone(s, 5, **kw) for s in specs]
    ens = Ensemble([member_params(*s, **kw) for s in specs])
    ens.initFlow()
    ens.autotune(steps=2)
    ens.set_schedule("batched")
    ens.step(5)
    for m, r, spec in zip(ens.members, ref, specs):
        for f in "uvwp":
            assert np.array_equal(m.download(f), r[f]), (trid, spec, f)
    ens.close()


@pytest.mark.parametrize("schedule", ["concurrent", "batched"])
def test_member_matches_oracle(schedule):
    """The smallest FP64 member, stepped 5 times inside an ensemble (beside a
    mixed-form member), against the oracle: the FP64 parity bar (1e-12 in
    u, v, w; p - mean(p) within its round-off floor at this size)."""
    from powerllel_channel_sycl_b200 import Ensemble
    spec = (32, 24, 16, 0, 2800.0)
    case = oracle.Case(**case_kwargs(32, 24, 16, re=2800.0))
    u, v, w = case.init_flow("poi", noise_intensity=0.1)
    p = case.zeros()
    ens = Ensemble([member_params(*spec), member_params(64, 48, 48, 1, 2000.0)])
    ens.set_schedule(schedule)
    ens.initFlow()
    m = ens.members[0]
    for name, a in zip("uvwp", (u, v, w, p)):
        m.upload(name, a)
    ens.step(5)
    case.step(u, v, w, case.zeros(), case.zeros(), case.zeros(), p, nsteps=5)
    for name, a in zip("uvw", (u, v, w)):
        assert rel_l2(m.download(name), a) <= 1e-12, name
    assert rel_l2(demean(m.download("p")), demean(p)) <= 4e-12
    ens.close()


def test_member_check_failure_names_the_member():
    from powerllel_channel_sycl_b200 import Ensemble, PlcError
    prms = [member_params(*MEMBERS[0], nt_check=2, cfl_limit=10.0, div_limit=1e-8),
            member_params(*MEMBERS[3], nt_check=2, cfl_limit=10.0, div_limit=1e-300)]
    ens = Ensemble(prms)
    ens.initFlow()
    with pytest.raises(PlcError) as e:
        ens.step(4)
    assert e.value.code == -5 and "member 1" in str(e.value) and "checkDiv" in str(e.value)


@pytest.mark.parametrize("pdl", [False, True])
def test_batched_check_failure_names_the_member(pdl):
    """The batched schedule's checks (one launch for the mixed-form members,
    inside the graph) report a failing member by its index."""
    from powerllel_channel_sycl_b200 import Ensemble, PlcError
    prms = [member_params(64, 48, 48, 1, 1500.0, nt_check=2, cfl_limit=10.0, div_limit=1e-8),
            member_params(96, 64, 32, 1, 2500.0, nt_check=2, cfl_limit=10.0, div_limit=1e-300)]
    ens = Ensemble(prms)
    ens.set_schedule("batched")
    ens.set_batch_pdl(pdl)
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


@pytest.mark.parametrize("schedule", ["concurrent", "batched", "batched_pdl"])
def test_cfl_controlled_members_match_standalone(schedule):
    """Under CFL control the checks every nt_check steps run inside the
    ensemble's graph, which sets each member's new dt on the device: the same
    division as the host's, so each member still steps exactly as alone."""
    from powerllel_channel_sycl_b200 import Ensemble
    kw = dict(nt_check=4, cfl_limit=1.0, div_limit=1e-3, cfl_target=0.4)
    specs = [MEMBERS[0], MIXED[1] + (1, 1500.0), MEMBERS[2]]
    ref = [standalone(s, 14, **kw) for s in specs]
    ens = Ensemble([member_params(*s, **kw) for s in specs])
    ens.set_schedule(schedule.replace("_pdl", ""))
    ens.set_batch_pdl(schedule.endswith("_pdl"))
    ens.initFlow()
    ens.step(14)
    for m, r, spec in zip(ens.members, ref, specs):
        assert m.step_count == 14
        for f in "uvwp":
            assert np.array_equal(m.download(f), r[f]), (schedule, spec, f)
    ens.close()


@pytest.mark.parametrize("schedule", ["concurrent", "batched"])
def test_check_period_above_block_cap_matches_standalone(schedule):
    """A check period above the multi-step block's cap (nt_check 40: blocks
    of 20 steps, every second one carrying the checks and the new dt in the
    graph) under CFL control: each member steps exactly as alone."""
    from powerllel_channel_sycl_b200 import Ensemble
    kw = dict(nt_check=40, cfl_limit=1.0, div_limit=1e-3, cfl_target=0.4)
    specs = [MEMBERS[0], MIXED[1] + (1, 1500.0), MEMBERS[2]]
    ref = [standalone(s, 85, **kw) for s in specs]
    ens = Ensemble([member_params(*s, **kw) for s in specs])
    ens.set_schedule(schedule)
    ens.initFlow()
    ens.step(85)
    for m, r, spec in zip(ens.members, ref, specs):
        assert m.step_count == 85
        for f in "uvwp":
            assert np.array_equal(m.download(f), r[f]), (schedule, spec, f)
    ens.close()


def test_long_check_period_keeps_blocks_short():
    """A check period far above the multi-step block's cap (nt_check 100000)
    steps in blocks of at most 32 steps: the captured graphs stay small."""
    from powerllel_channel_sycl_b200 import Ensemble
    import time
    ens = Ensemble([member_params(*s, nt_check=100000) for s in MEMBERS[:2]])
    ens.initFlow()
    t0 = time.perf_counter()
    ens.step(20)
    assert time.perf_counter() - t0 < 30.0
    assert all(m.step_count == 20 for m in ens.members)
    ens.close()


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
