"""Batched ensembles of independent channels over the C ABI (plc_ensemble_*).

No counterpart in the reference (one channel per run).  Each member has its
own parameters; ``members[i]`` is a :class:`Channel` view of member i for the
usual entry points (upload, download, statistics, I/O).
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from ._lib import PlcError, PlcParams, lib
from .channel import Channel

SCHEDULES = ("concurrent", "proportional", "two_groups", "sequential", "batched")


def _check(rc: int, ens=None) -> None:
    if rc != 0:
        msg = lib().plc_ensemble_last_error(ens)
        raise PlcError(rc, msg.decode() if msg else "")


class Ensemble:
    def __init__(self, params: Sequence[PlcParams], device: int = 0, dzf_globals=None):
        n = len(params)
        arr = (PlcParams * n)(*params)
        self.params = list(params)
        dz = None
        self._dzf = None
        if dzf_globals is not None:
            self._dzf = [None if d is None else np.ascontiguousarray(d, dtype=np.float64)
                         for d in dzf_globals]
            dz = (C.c_void_p * n)(*[None if d is None else d.ctypes.data for d in self._dzf])
        ens = C.c_void_p()
        _check(lib().plc_ensemble_create(n, arr, dz, device, C.byref(ens)))
        self._ens = ens
        self.members = []
        for i in range(n):
            ctx = C.c_void_p()
            self._check(lib().plc_ensemble_member(self._ens, i, C.byref(ctx)))
            self.members.append(Channel._wrap(ctx, self.params[i], self))

    def _check(self, rc):
        _check(rc, self._ens)

    def close(self):
        if getattr(self, "_ens", None):
            for m in self.members:
                m.close()
            lib().plc_ensemble_destroy(self._ens)
            self._ens = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return len(self.members)

    def initFlow(self):
        self._check(lib().plc_ensemble_init_flow(self._ens))

    def step(self, nsteps: int = 1):
        self._check(lib().plc_ensemble_step(self._ens, int(nsteps)))

    def step_timed(self, nsteps: int) -> float:
        ms = C.c_double()
        self._check(lib().plc_ensemble_step_timed(self._ens, int(nsteps), C.byref(ms)))
        return ms.value

    def set_schedule(self, name):
        q = SCHEDULES.index(name) if isinstance(name, str) else int(name)
        self._check(lib().plc_ensemble_set_schedule(self._ens, q))

    def schedule(self):
        n = len(self.members)
        s = C.c_int()
        groups = (C.c_int * n)()
        budgets = (C.c_int * n)()
        self._check(lib().plc_ensemble_schedule(self._ens, C.byref(s), groups, budgets))
        return SCHEDULES[s.value], list(groups), list(budgets)

    def set_batch_chains(self, chains: int):
        """The batched schedule's concurrent chains of mixed-form members (1 or 2)."""
        self._check(lib().plc_ensemble_set_batch_chains(self._ens, int(chains)))

    def set_batch_pdl(self, on: bool):
        """Programmatic dependent launch of the batched schedule's kernels
        (each stage's blocks become resident while the previous stage drains;
        results are the same either way)."""
        self._check(lib().plc_ensemble_set_batch_pdl(self._ens, 1 if on else 0))

    def batch_choice(self):
        """The batched schedule's tuned choices: the concurrent chains of
        mixed-form members, the RK z planes per block (0: each member's own),
        resident blocks per SM of the RK kernels, the number of tuned
        line-length groups of the forward x, backward x and y transforms, and
        whether the kernels use programmatic dependent launch."""
        ch, kc, mb, pdl = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        groups = (C.c_int * 3)()
        self._check(lib().plc_ensemble_batch_choice(self._ens, C.byref(ch), C.byref(kc),
                                                    C.byref(mb), groups))
        self._check(lib().plc_ensemble_batch_pdl(self._ens, C.byref(pdl)))
        return {"chains": ch.value, "rk_kchunk": kc.value, "rk_blocks_per_sm": mb.value,
                "fft_groups": list(groups), "pdl": bool(pdl.value)}

    def autotune(self, steps: int = 5) -> dict:
        """Times every schedule (ms per ensemble step) and keeps the fastest."""
        out = (C.c_float * len(SCHEDULES))()
        self._check(lib().plc_ensemble_autotune(self._ens, int(steps), out))
        return {name: (t if t >= 0 else None) for name, t in zip(SCHEDULES, out)}

    @property
    def points(self) -> int:
        return sum(p.nx * p.ny * p.nz for p in self.params)


def partition(costs, n_gpus: int) -> list:
    """Placement of members on GPUs, longest processing time first."""
    n = len(costs)
    c = (C.c_double * n)(*costs)
    out = (C.c_int * n)()
    _check(lib().plc_ensemble_partition(n, c, int(n_gpus), out))
    return list(out)


def members_of_rank(costs, rank: int, world: int) -> list:
    """The members one rank of a world_size-GPU job runs (one process per GPU)."""
    gpu_of = partition(costs, world)
    return [i for i, g in enumerate(gpu_of) if g == rank]
