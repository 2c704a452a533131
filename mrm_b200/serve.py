"""Served form: continuous batching of M(H)-loop and write-pattern requests.

Requests arrive over time (`Request.arrival`, seconds after the stream
start).  The server keeps one Batch resident on the GPU and loops:

1. move requests whose arrival time has passed into the admission queue;
2. admit queued requests first-come-first-served while their device
   footprint (state, parameters, spectra, tensor) fits the HBM budget; a
   request's tensor spectrum is copied device-to-device from a per-geometry
   template instead of being rebuilt.  The GPU backend sets admitted runs up
   in a second (staging) batch, whose uploads wait only for its own stream,
   and moves them into the serving batch (mrm_batch_adopt, no copy) right
   before its next call;
3. advance every active run by K = chunk Heun steps in one launch sequence,
   enqueued before step 2's admissions so that their host work overlaps it.
   A request of S steps is admitted with an aligned start: it idles through
   the first K - S mod K steps of its first call (mrm_batch_delay_run), so
   its budget ends on a call boundary and its reductions at the end of
   every call describe its own last step, while every call keeps the full
   chunk length (a run's trajectory is the same as without the delay);
4. record each run's M(H) sample (time, applied field, m.h), retire finished
   runs (result + latency = finish - arrival) and free their memory (the
   frees themselves run while the next call is on the GPU).

A request's medium (its grains, parameters and exchange lists, built on the
host) is prepared by a worker thread as soon as the request arrives, while
the GPU runs the current call (the launch releases the interpreter lock), so
admission only uploads it.  Requests that arrive while others are on the
GPU are admitted as soon as memory frees up and join the next launch; a run's trajectory does not depend
on its neighbours (each run's kernels read only its own data), which the
tests check bit for bit against the same request run alone.

A request can carry a timeout (seconds after its arrival) and can be
cancelled (Server.cancel, from any thread).  At each call boundary the loop
retires such requests -- queued or running -- with status "timeout" or
"cancelled" and the samples taken so far, and frees their memory; the other
runs continue unchanged.  Finished requests have status "done".
"""
from __future__ import annotations

import collections
import concurrent.futures
import threading
import time
from typing import Callable, Dict, List, Optional

import numpy as np

from . import _lib
from .workloads import DT, Request


class _Active:
    __slots__ = ("req", "run", "fp", "admitted", "remaining", "samples")

    def __init__(self, req, run, fp, admitted, idle):
        self.req = req
        self.run = run
        self.fp = fp
        self.admitted = admitted
        self.remaining = req.steps + idle  # steps of the calls left, idle prefix included
        self.samples = []

    @property
    def steps_done(self) -> int:
        return max(0, self.req.steps - self.remaining)


def applied_field(req: Request, t: float) -> float:
    """Signed magnitude of the request's uniform field along its direction."""
    if req.kind == "mh":
        u = min(1.0, max(0.0, t / (req.steps * DT)))
        return 20000.0 - 40000.0 * u
    return 12000.0  # write: STE amplitude; the sign follows the square wave


def coercivity(h, mh):
    h, mh = np.asarray(h, float), np.asarray(mh, float)
    hc = mr = None
    for k in range(1, len(h)):
        if hc is None and mh[k - 1] > 0 >= mh[k]:
            hc = -(h[k - 1] + (h[k] - h[k - 1]) * mh[k - 1] / (mh[k - 1] - mh[k]))
        if mr is None and h[k - 1] > 0 >= h[k]:
            mr = mh[k - 1] + (mh[k] - mh[k - 1]) * h[k - 1] / (h[k - 1] - h[k])
    return hc, mr


class Server:
    """Continuous-batching scheduler over a Batch-like backend.

    backend: object with add(medium, dt, steps, thermal_seed, tensor_from) ->
    run, delay(run, idle_steps), remove(run), step(k) (or enqueue(k), which
    returns at once), stats(runs) (waits for the call), footprint(medium) ->
    bytes, memory() -> (free, total); defaults to the GPU Batch.
    """

    def __init__(self, backend=None, precision: int = _lib.FP32, device: int = 0,
                 hbm_fraction: float = 0.8, hbm_budget: Optional[int] = None, chunk: int = 500,
                 max_active: int = 4096, keep_state: bool = False,
                 clock: Callable[[], float] = time.perf_counter,
                 sleep: Callable[[float], None] = time.sleep):
        if backend is None:
            backend = GpuBackend(precision, device)
        self.be = backend
        free, total = backend.memory()
        self.budget = hbm_budget if hbm_budget is not None else int(free * hbm_fraction)
        self.chunk = int(chunk)
        self.max_active = int(max_active)
        self.keep_state = keep_state
        self.clock = clock
        self.sleep = sleep
        self.used = 0
        self.templates: Dict[tuple, object] = {}
        self._cancel_lock = threading.Lock()
        self._cancelled: set = set()

    def cancel(self, rid: int):
        """Asks the serving loop to drop request `rid` at its next call
        boundary (queued or running); thread-safe."""
        with self._cancel_lock:
            self._cancelled.add(int(rid))

    def _enqueue(self, k: int):
        """Starts a call of k steps (the backend's asynchronous launch when it
        has one; stats() then waits for it)."""
        launch = getattr(self.be, "enqueue", None)
        (launch or self.be.step)(k)

    def _take_cancelled(self) -> set:
        with self._cancel_lock:
            c, self._cancelled = self._cancelled, set()
        return c

    def _admit(self, req: Request, med, fp: int, now: float):
        key = (req.side, req.side)
        tmpl = self.templates.get(key)
        run = self.be.add(med, DT, req.steps, req.seed, tmpl)
        if tmpl is None:
            self.templates[key] = self.be.make_template(run)
        idle = (-req.steps) % self.chunk
        if idle:
            self.be.delay(run, idle)
        return _Active(req, run, fp, now, idle)

    def _retire(self, a: Optional[_Active], req: Request, status: str, now: float, s=None) -> dict:
        """Result record of a request that leaves the server (a: its run, or
        None when it never left the queue)."""
        samples = a.samples if a is not None else []
        res = {"rid": req.rid, "kind": req.kind, "grains": req.grains, "steps": req.steps,
               "arrival": req.arrival, "admitted": a.admitted if a is not None else None,
               "finished": now, "latency": now - req.arrival, "status": status,
               "steps_done": a.steps_done if a is not None else 0,
               "samples": len(samples)}
        if s is not None:
            res["final_mave"] = np.asarray(s["mave"]).tolist()
            res["step"] = int(s["step"])
        if status == "done" and req.kind == "mh":
            ts = np.array(samples)
            res["hc"], res["mr"] = coercivity(ts[:, 1], ts[:, 2])
        if a is not None:
            if self.keep_state and status == "done":
                res["m"] = self.be.get_state(a.run)
            self.be.remove(a.run)
            self.used -= a.fp
        return res

    def run(self, requests: List[Request]) -> dict:
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        queue = collections.deque()
        active: List[_Active] = []
        results = []
        t0 = self.clock()
        calls = 0
        # media of arrived requests, built on a worker thread (rid -> future)
        prep = concurrent.futures.ThreadPoolExecutor(max_workers=1)
        media = {}
        try:
            return self._loop(pending, queue, active, results, t0, calls, prep, media)
        finally:
            for f in media.values():
                f.cancel()
            prep.shutdown(wait=True)

    def _loop(self, pending, queue, active, results, t0, calls, prep, media) -> dict:
        while pending or queue or active:
            now = self.clock() - t0
            while pending and pending[0].arrival <= now:
                q = pending.popleft()
                queue.append(q)
                media[q.rid] = prep.submit(q.medium)
            # cancellations and timeouts, at a call boundary: queued or running
            cancelled = self._take_cancelled()
            for rid in cancelled:
                for q in [p for p in pending if p.rid == rid]:
                    pending.remove(q)
                    results.append(self._retire(None, q, "cancelled", now))
            expired = lambda r: r.timeout is not None and now - r.arrival >= r.timeout  # noqa: E731
            for q in [q for q in queue if q.rid in cancelled or expired(q)]:
                queue.remove(q)
                media.pop(q.rid).cancel()
                results.append(self._retire(None, q, "cancelled" if q.rid in cancelled else "timeout", now))
            for a in [a for a in active if a.req.rid in cancelled or expired(a.req)]:
                active.remove(a)
                results.append(self._retire(a, a.req, "cancelled" if a.req.rid in cancelled else "timeout", now))
            # one launch sequence of the full chunk for the runs already on the
            # device (every budget ends on a call boundary: aligned starts),
            # enqueued before the admissions below, whose host work (uploads,
            # the next requests' set-up) then overlaps it; runs admitted now
            # join the next call
            running = list(active)
            k = self.chunk
            if running:
                self._enqueue(k)
                calls += 1
            # admission, first come first served, by device footprint
            while queue and len(active) < self.max_active:
                req = queue[0]
                med = media[req.rid].result()
                fp = self.be.footprint(med)
                if active and self.used + fp > self.budget:
                    break
                queue.popleft()
                del media[req.rid]
                a = self._admit(req, med, fp, self.clock() - t0)
                self.used += a.fp
                active.append(a)
            if not running:
                if not active and pending:
                    self.sleep(max(0.0, min(pending[0].arrival - (self.clock() - t0), 0.01)))
                continue
            st = self.be.stats([a.run for a in running])
            done_t = self.clock() - t0
            finished = []
            for a, s in zip(running, st):
                a.remaining -= k
                mh = float(np.asarray(s["mms_l"][0]) @ self.be.hdir(a.run))
                a.samples.append((float(s["t"]), applied_field(a.req, float(s["t"])), mh,
                                  float(s["mave"][2])))
                if a.remaining <= 0:
                    finished.append((a, s))
            for a, s in finished:
                active.remove(a)
                results.append(self._retire(a, a.req, "done", done_t, s))
        wall = self.clock() - t0
        done = [r for r in results if r["status"] == "done"]
        lat = np.array([r["latency"] for r in done]) if done else np.zeros(1)
        gs = sum(r["grains"] * r["steps_done"] for r in results)
        return {"results": sorted(results, key=lambda r: r["rid"]), "wall_s": wall,
                "grain_steps": gs, "grain_steps_per_s": gs / wall if wall > 0 else 0.0,
                "p50_latency_s": float(np.percentile(lat, 50)),
                "p99_latency_s": float(np.percentile(lat, 99)), "calls": calls,
                "completed": len(done), "timed_out": sum(r["status"] == "timeout" for r in results),
                "cancelled": sum(r["status"] == "cancelled" for r in results)}


class GpuBackend:
    """The GPU Batch behind the server."""

    def __init__(self, precision: int, device: int):
        from .batch import Batch, device_memory, footprint
        self._Batch = Batch
        self._fp = footprint
        self._mem = device_memory
        self.precision = precision
        self.device = device
        self.batch = Batch(precision, device)
        self.lib_batch = Batch(precision, device)  # per-geometry tensor templates (never stepped)
        # arriving runs are set up here (uploads, tensor copies or builds on
        # this batch's stream, overlapping the serving batch's call in
        # flight) and move into the serving batch before its next call
        self.stage = Batch(precision, device)
        self._staged = []

    def memory(self):
        return self._mem(self.device)

    def footprint(self, medium) -> int:
        return self._fp(medium, self.precision)

    def add(self, medium, dt, steps, seed, template):
        run = self.stage.add(medium, dt=dt, steps=steps, thermal_seed=seed, tensor_from=template)
        run._hdir = np.array(medium.layers[0].hdir, float)
        self._staged.append(run)
        return run

    def _adopt(self):
        for run in self._staged:
            self.batch.adopt(run)
        self._staged = []

    def delay(self, run, idle_steps):
        run.delay(idle_steps)

    def make_template(self, run):
        t = self.lib_batch.add(run.medium, dt=DT, steps=0, demag=True, tensor_from=run)
        t.set_run(DT, 0, active=False)
        return t

    def hdir(self, run):
        return run._hdir

    def remove(self, run):
        if run in self._staged:
            self._staged.remove(run)
            self.stage.remove(run)
            self.stage.stats([])  # the staging batch never steps: release now
        else:
            self.batch.remove(run)

    def step(self, k: int):
        self._adopt()
        self.batch.step(k)

    def enqueue(self, k: int):
        self._adopt()
        self.batch.enqueue(k)

    def stats(self, runs):
        return self.batch.stats(runs)

    def get_state(self, run):
        return run.get_state(0)

    def close(self):
        self.batch.close()
        self.stage.close()
        self.lib_batch.close()
