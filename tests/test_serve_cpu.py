"""Scheduling of the serving loop, checked on the host with a fake batch:
admission in arrival order under the HBM budget, retirement exactly at each
request's step count, requests that arrive while others run join the batch
(continuous batching), and an over-budget request waits instead of failing."""
import numpy as np
import pytest

from lh_b200.capi import LH_ENOMEM, Desc, LHError
from lh_b200.serve import Request, serve


class FakeBatch:
    instances = []

    def __init__(self, budget):
        self.budget, self.used = budget, 0
        self.live = {}
        self.log = []
        FakeBatch.instances.append(self)

    def add(self, desc, *state):
        need = desc.points()
        if self.budget and self.used + need > self.budget:
            raise LHError(LH_ENOMEM, "budget")
        slot = next(k for k in range(1000) if k not in self.live)
        self.live[slot] = [desc, 0]
        self.used += need
        self.log.append(("add", slot, len(self.live)))
        return slot

    def step(self, k):
        for v in self.live.values():
            v[1] += k
        self.log.append(("step", k, len(self.live)))

    def synchronize(self):
        pass

    def download(self, slot):
        return {"steps": self.live[slot][1]}

    def remove(self, slot):
        self.used -= self.live[slot][0].points()
        del self.live[slot]

    def close(self):
        pass


def _reqs():
    small = Desc(Nx=8, Nz=8, ny=17)
    big = Desc(Nx=16, Nz=16, ny=33)
    return [Request(0, small, 1, 7, 0.0), Request(1, big, 2, 3, 0.0), Request(2, small, 3, 12, 0.0),
            Request(3, big, 4, 5, 0.0), Request(4, small, 5, 2, 0.0)]


def test_every_request_runs_exactly_its_steps():
    FakeBatch.instances.clear()
    reqs = _reqs()
    st = serve(reqs, hbm_budget=0, max_chunk=4, batch_factory=FakeBatch, state_fn=lambda r: (), prefetch=0)
    assert st.requests == 5
    for r in reqs:
        assert r.result["steps"] == r.nsteps
        assert r.finished >= r.admitted
    log = FakeBatch.instances[-1].log
    assert max(n for op, _, n in log if op == "step") == 5  # all five ran together
    assert all(k <= 4 for op, k, _ in log if op == "step")


def test_budget_defers_admission_until_memory_frees():
    FakeBatch.instances.clear()
    reqs = _reqs()
    budget = Desc(Nx=16, Nz=16, ny=33).points() + Desc(Nx=8, Nz=8, ny=17).points()
    st = serve(reqs, hbm_budget=budget, max_chunk=50, batch_factory=FakeBatch, state_fn=lambda r: (), prefetch=0)
    for r in reqs:
        assert r.result["steps"] == r.nsteps
    log = FakeBatch.instances[-1].log
    assert max(n for op, _, n in log) <= 2  # never more than the budget allows
    assert st.max_live <= 2


def test_late_arrivals_join_while_others_run():
    FakeBatch.instances.clear()
    d = Desc(Nx=8, Nz=8, ny=17)
    t = {"now": 0.0}

    def clock():
        t["now"] += 0.01
        return t["now"]

    reqs = [Request(0, d, 1, 40, 0.0), Request(1, d, 2, 5, 0.05)]
    serve(reqs, hbm_budget=0, max_chunk=2, batch_factory=FakeBatch, state_fn=lambda r: (), clock=clock, prefetch=0)
    log = FakeBatch.instances[-1].log
    adds = [i for i, e in enumerate(log) if e[0] == "add"]
    steps = [i for i, e in enumerate(log) if e[0] == "step"]
    assert adds[1] > steps[0]          # the second request joined after stepping began
    assert reqs[0].result["steps"] == 40 and reqs[1].result["steps"] == 5
    assert reqs[1].finished < reqs[0].finished


def test_non_budget_errors_propagate():
    class Broken(FakeBatch):
        def add(self, desc, *state):
            raise LHError(-1, "bad size")
    with pytest.raises(LHError):
        serve(_reqs(), hbm_budget=0, batch_factory=Broken, state_fn=lambda r: (), prefetch=0)


def test_prefetched_states_run_exactly_their_steps():
    """With initial states built ahead by the worker thread the admissions may
    fall into later rounds, but every request still runs exactly its steps,
    with the state its own request produced."""
    FakeBatch.instances.clear()
    reqs = _reqs()
    seen = []

    def state_fn(r):
        seen.append(r.rid)
        return (r.rid,)

    st = serve(reqs, hbm_budget=0, max_chunk=3, batch_factory=FakeBatch, state_fn=state_fn, prefetch=2)
    assert st.requests == 5 and sorted(seen) == [0, 1, 2, 3, 4]
    for r in reqs:
        assert r.result["steps"] == r.nsteps
        assert r.finished >= r.admitted
