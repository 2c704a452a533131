"""Host logic of the continuous-batching server, on a fake backend (no GPU)."""
import numpy as np

from mrm_b200 import _lib
from mrm_b200.serve import Server, coercivity
from mrm_b200.workloads import Request, served_requests


class FakeRun:
    def __init__(self, medium, steps):
        self.medium = medium
        self.budget = steps
        self.done = 0


class FakeBackend:
    def __init__(self, budget_bytes):
        self.t = 0.0
        self.free = budget_bytes
        self.runs = []
        self.max_used = 0
        self.used = 0
        self.calls = []

    def memory(self):
        return self.free, self.free

    def footprint(self, medium):
        return medium.n_grains * 300

    def add(self, medium, dt, steps, seed, tmpl):
        r = FakeRun(medium, steps)
        self.runs.append(r)
        self.used += self.footprint(medium)
        self.max_used = max(self.max_used, self.used)
        return r

    def make_template(self, run):
        return object()

    def hdir(self, run):
        return np.array([0.0, 0.0, 1.0])

    def remove(self, run):
        self.runs.remove(run)
        self.used -= self.footprint(run.medium)

    def step(self, k):
        rem = [r.budget - r.done for r in self.runs]
        assert k <= min(rem), "a call must not run past a budget"
        self.calls.append((k, len(self.runs)))
        for r in self.runs:
            r.done += k
        self.t += 1e-4 * k

    def stats(self, runs):
        st = np.zeros(len(runs), _lib.STATS_DTYPE)
        for i, r in enumerate(runs):
            st[i]["t"] = r.done * 1e-13
            st[i]["step"] = r.done
            st[i]["mms_l"][0] = [0.0, 0.0, 1.0 - 2.0 * r.done / r.budget]
            st[i]["mave"] = [0.0, 0.0, 1.0 - 2.0 * r.done / r.budget]
        return st

    def clock(self):
        return self.t

    def sleep(self, s):
        self.t += max(s, 1e-6)


def _small_requests(n=40, seed=3):
    reqs = served_requests(n=n, rate=2000.0, seed=seed, lo=1024, hi=16384, steps_lo=200, steps_hi=900)
    return reqs


def test_all_requests_complete_with_exact_step_counts():
    be = FakeBackend(budget_bytes=10**12)
    srv = Server(backend=be, chunk=128, clock=be.clock, sleep=be.sleep)
    reqs = _small_requests()
    out = srv.run(reqs)
    assert len(out["results"]) == len(reqs)
    for r, q in zip(out["results"], sorted(reqs, key=lambda x: x.rid)):
        assert r["rid"] == q.rid and r["step"] == q.steps
        assert r["latency"] >= 0 and r["finished"] >= q.arrival
    assert out["grain_steps"] == sum(q.grains * q.steps for q in reqs)


def test_admission_respects_the_memory_budget():
    reqs = _small_requests(60)
    biggest = max(q.grains for q in reqs) * 300
    be = FakeBackend(budget_bytes=3 * biggest)
    srv = Server(backend=be, hbm_budget=3 * biggest, chunk=100, clock=be.clock, sleep=be.sleep)
    out = srv.run(reqs)
    assert len(out["results"]) == len(reqs)
    assert be.max_used <= 3 * biggest
    # requests overlap on the device (continuous batching, not a serial queue)
    assert max(n for _, n in be.calls) > 1


def test_late_arrivals_join_running_batch():
    reqs = [Request(0, 0.0, "mh", 32, 300.0, 1000, 1), Request(1, 0.0, "mh", 32, 300.0, 1000, 2),
            Request(2, 0.02, "write", 64, 300.0, 400, 3)]
    be = FakeBackend(budget_bytes=10**12)
    srv = Server(backend=be, chunk=100, clock=be.clock, sleep=be.sleep)
    out = srv.run(reqs)
    res = {r["rid"]: r for r in out["results"]}
    # request 2 arrived while 0 and 1 were running and finished before them
    assert res[2]["admitted"] > 0 and res[2]["finished"] < res[0]["finished"]
    assert any(n == 3 for _, n in be.calls)


def test_coercivity_interpolation():
    h = np.linspace(20000, -20000, 41)
    mh = np.tanh((h + 9000.0) / 1500.0)
    hc, mr = coercivity(h, mh)
    assert abs(hc - 9000.0) < 60.0
    assert abs(mr - np.tanh(9000.0 / 1500.0)) < 1e-3
