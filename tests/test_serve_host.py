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
        self.idle = 0


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

    def delay(self, run, idle):
        assert run.done == 0 and run.idle == 0 and 0 < idle
        run.idle = idle

    def hdir(self, run):
        return np.array([0.0, 0.0, 1.0])

    def remove(self, run):
        self.runs.remove(run)
        self.used -= self.footprint(run.medium)

    def step(self, k):
        # every budget ends on a call boundary: no run stops inside a call
        for r in self.runs:
            assert r.idle + (r.budget - r.done) >= k, "a call must not run past a budget"
        self.calls.append((k, len(self.runs)))
        for r in self.runs:
            r.done += k - r.idle
            r.idle = 0
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


def test_timeouts_retire_queued_and_running_requests():
    """A request whose timeout passes is dropped at the next call boundary,
    whether it still waits for memory or is on the device; the others finish
    with their exact step counts and the memory of the dropped ones is freed."""
    reqs = [Request(0, 0.0, "mh", 64, 300.0, 4000, 1, timeout=0.05),   # running when it times out
            Request(1, 0.0, "mh", 64, 300.0, 600, 2),
            Request(2, 0.0, "mh", 64, 300.0, 600, 3, timeout=0.01),    # still queued (no memory yet)
            Request(3, 0.001, "write", 32, 300.0, 300, 4, timeout=10.0)]
    be = FakeBackend(budget_bytes=10**12)
    fp = 64 * 64 * 300
    srv = Server(backend=be, hbm_budget=2 * fp, chunk=100, clock=be.clock, sleep=be.sleep)
    out = srv.run(reqs)
    res = {r["rid"]: r for r in out["results"]}
    assert len(res) == 4
    assert res[0]["status"] == "timeout" and 0 < res[0]["steps_done"] < 4000
    assert res[0]["finished"] - res[0]["arrival"] >= 0.05
    assert res[2]["status"] == "timeout" and res[2]["admitted"] is None and res[2]["steps_done"] == 0
    for rid in (1, 3):
        assert res[rid]["status"] == "done" and res[rid]["step"] == reqs[rid].steps
    assert out["timed_out"] == 2 and out["completed"] == 2
    assert be.used == 0 and not be.runs  # every run left the device
    assert out["grain_steps"] == sum(r["grains"] * r["steps_done"] for r in out["results"])


def test_cancellation_from_another_thread():
    """Server.cancel from another thread (here: from inside a launch) drops the
    request at the next call boundary; a cancelled request that has not
    arrived yet never runs."""
    reqs = [Request(0, 0.0, "mh", 64, 300.0, 3000, 1), Request(1, 0.0, "mh", 32, 300.0, 900, 2),
            Request(2, 5.0, "mh", 32, 300.0, 900, 3)]
    be = FakeBackend(budget_bytes=10**12)
    srv = Server(backend=be, chunk=100, clock=be.clock, sleep=be.sleep)
    step = be.step

    def step_and_cancel(k):
        step(k)
        if len(be.calls) == 3:
            import threading
            t = threading.Thread(target=lambda: (srv.cancel(0), srv.cancel(2)))
            t.start()
            t.join()

    be.step = step_and_cancel
    out = srv.run(reqs)
    res = {r["rid"]: r for r in out["results"]}
    # 3000 steps are a multiple of the chunk: no idle prefix, three calls done
    assert res[0]["status"] == "cancelled" and res[0]["steps_done"] == 300
    assert res[2]["status"] == "cancelled" and res[2]["steps_done"] == 0 and res[2]["admitted"] is None
    assert res[1]["status"] == "done" and res[1]["step"] == 900
    assert out["cancelled"] == 2 and not be.runs


def test_every_call_has_the_full_chunk():
    """Aligned starts: budgets that are not multiples of the chunk idle through
    the head of their first call, so every call runs the full chunk and each
    request still executes exactly its own step count."""
    reqs = [Request(0, 0.0, "mh", 32, 300.0, 1000, 1), Request(1, 0.0, "mh", 32, 300.0, 130, 2),
            Request(2, 0.0, "write", 32, 300.0, 777, 3), Request(3, 0.0, "mh", 32, 300.0, 256, 4)]
    be = FakeBackend(budget_bytes=10**12)
    srv = Server(backend=be, chunk=128, clock=be.clock, sleep=be.sleep)
    out = srv.run(reqs)
    assert {k for k, _ in be.calls} == {128}
    assert len(be.calls) == -(-1000 // 128)
    res = {r["rid"]: r for r in out["results"]}
    for q in reqs:
        assert res[q.rid]["status"] == "done" and res[q.rid]["step"] == q.steps
        assert res[q.rid]["steps_done"] == q.steps
    # a request finishes after as many calls as its steps need
    assert res[1]["finished"] < res[2]["finished"] < res[0]["finished"]
