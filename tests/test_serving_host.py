"""Admission, retire and refill logic of the serving loop, on a fake engine (no GPU)."""
import types

import numpy as np

from pyheartsim_b200 import serving


class FakeEngine:
    """Advances instances by whole launches; records admission order and occupancy."""

    def __init__(self):
        self.inst = {}
        self.step = {}
        self.next = 0
        self.max_active = 0
        self.order = []

    def set_profile(self, on):
        pass

    def add(self, inst):
        s = self.next
        self.next += 1
        self.inst[s] = inst
        self.step[s] = 0
        self.order.append(inst.rid)
        self.max_active = max(self.max_active, len(self.inst))
        return s

    def advance(self, n, stream=None, sync=True):
        for s in self.inst:
            self.step[s] = min(self.inst[s].n_steps, self.step[s] + n)

    def rebalance(self):
        pass

    def info(self, s):
        return {"step": self.step[s], "n_steps": self.inst[s].n_steps, "status": 0,
                "samples": self.step[s] // 10}

    def history(self, s, count=None):
        return np.zeros((count or 0, self.inst[s].n_voxel), np.float32)

    def remove(self, s):
        del self.inst[s]

    def close(self):
        pass


def _inst(rid, n, steps):
    return types.SimpleNamespace(rid=rid, n_voxel=n, n_steps=steps, n_samples=steps // 10, restart=20, save_h=0)


def test_fifo_admission_respects_budget_and_refills():
    reqs = serving.poisson_requests(12, rate_per_s=1000.0, n_min=1000, n_max=5000, seed=3)
    for r in reqs:
        r.arrival_s = 0.0                            # all waiting at once
    eng = FakeEngine()
    built = {r.rid: _inst(r.rid, r.n_target, 200 + 50 * (r.rid % 3)) for r in reqs}
    srv = serving.Server(hbm_budget_bytes=3, steps_per_launch=50, engine=eng, build_threads=0,
                         builder=lambda r: built[r.rid], footprint=lambda inst: 1)
    done, totals = srv.run(reqs)
    srv.close()
    assert len(done) == 12
    assert eng.order == sorted(eng.order)            # FIFO: never overtaken
    assert eng.max_active == 3                       # budget of 3 units, one unit each
    assert all(r.done_s >= r.admit_s >= 0 for r in done)
    summary = serving.summarize(done, totals, reqs)
    assert summary["requests"] == 12 and summary["p99_latency_s"] >= summary["p50_latency_s"]


def test_oversized_request_runs_alone():
    reqs = serving.poisson_requests(3, rate_per_s=1000.0, seed=1)
    eng = FakeEngine()
    srv = serving.Server(hbm_budget_bytes=10, steps_per_launch=100, engine=eng, build_threads=0,
                         builder=lambda r: _inst(r.rid, 100, 300), footprint=lambda inst: 50)
    done, _ = srv.run(reqs)
    srv.close()
    assert len(done) == 3 and eng.max_active == 1    # each one too big to share, admitted alone


def test_poisson_requests_are_seeded():
    a = serving.poisson_requests(20, seed=5)
    b = serving.poisson_requests(20, seed=5)
    assert [(r.arrival_s, r.n_target, r.model) for r in a] == [(r.arrival_s, r.n_target, r.model) for r in b]
    assert all(20_000 <= r.n_target <= 1_000_000 for r in a)
    assert all(200 <= r.duration_ms <= 2000 for r in a)
