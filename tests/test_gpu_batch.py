"""Batched and served forms against the plain single-run path (bitwise)."""
import math

import numpy as np
import pytest

from mrm_b200 import FP32, FP64, GpuSim, media
from mrm_b200.batch import Batch
from mrm_b200.serve import Server
from mrm_b200.workloads import Request

pytestmark = pytest.mark.gpu


def _media():
    a = media.mh_medium(16, seed=21, temperature=0.0, ramp_s=1e-10)
    b = media.mh_medium(32, seed=22, temperature=300.0, ramp_s=1e-10)
    c = media.mh_medium(24, seed=23, temperature=250.0)
    lay = c.layers[0]
    lay.func, lay.amp, lay.fgamma, lay.param, lay.scale = 4, 12000.0, 2e-11, 1e-12, 1.0
    lay.hdir = (math.sin(0.3), 0.0, -math.cos(0.3))
    return [a, b, c]


@pytest.mark.parametrize("precision", [FP64, FP32])
def test_batch_matches_alone(gpulib, precision):
    meds = _media()
    n = 150
    alone = []
    for i, m in enumerate(meds):
        g = GpuSim(m, precision=precision, thermal_seed=5 + i)
        s = g.step(n, 1e-13)
        alone.append((g.get_state(0), s))
        g.close()
    b = Batch(precision)
    runs = [b.add(m, dt=1e-13, steps=n, thermal_seed=5 + i) for i, m in enumerate(meds)]
    b.step(n)
    st = b.stats(runs)
    for r, s, (m_alone, s_alone) in zip(runs, st, alone):
        assert np.array_equal(r.get_state(0), m_alone)
        assert s["step"] == n and np.array_equal(s["mave"], s_alone["mave"])
    b.close()


def test_batch_step_budgets(gpulib):
    meds = _media()
    budgets = [40, 100, 64]
    b = Batch(FP64)
    runs = [b.add(m, dt=1e-13, steps=k, thermal_seed=9) for m, k in zip(meds, budgets)]
    b.step(100)
    for r, m, k in zip(runs, meds, budgets):
        g = GpuSim(m, precision=FP64, thermal_seed=9)
        g.step(k, 1e-13)
        assert np.array_equal(r.get_state(0), g.get_state(0))
        assert r.get_time()[1] == k
        g.close()
    b.close()


def test_batch_aligned_start(gpulib):
    """A run delayed by K - S mod K idles through the head of its first call
    and ends its S-step budget on the call boundary: state, time and the
    call's reductions equal the run stepped alone; an undelayed neighbour is
    unaffected."""
    meds = _media()[:2]
    b = Batch(FP64)
    r0 = b.add(meds[0], dt=1e-13, steps=70, thermal_seed=9)
    r1 = b.add(meds[1], dt=1e-13, steps=200, thermal_seed=9)
    r0.delay(30)
    b.step(100)
    st = b.stats([r0, r1])
    assert st[0]["step"] == 70 and st[1]["step"] == 100
    b.step(100)
    st2 = b.stats([r0, r1])
    assert st2[0]["step"] == 70 and np.array_equal(st2[0]["mave"], st[0]["mave"])
    for r, m, k, s in ((r0, meds[0], 70, st[0]), (r1, meds[1], 200, st2[1])):
        g = GpuSim(m, precision=FP64, thermal_seed=9)
        sg = g.step(k, 1e-13)
        assert np.array_equal(r.get_state(0), g.get_state(0))
        assert r.get_time()[1] == k
        assert s["t"] == sg["t"] and np.array_equal(s["mave"], sg["mave"])
        g.close()
    b.close()


def test_adopted_run_matches_alone(gpulib):
    """A run set up (uploads, tensor) in a second batch and moved into a
    stepping batch between two of its calls, next to a run removed at the same
    boundary, advances exactly like the run alone; the removed run's device
    memory comes back at the batch's next stats."""
    from mrm_b200.batch import device_memory
    meds = _media()
    b, stage = Batch(FP64), Batch(FP64)
    r0 = b.add(meds[0], dt=1e-13, steps=60, thermal_seed=9)
    r1 = b.add(meds[1], dt=1e-13, steps=120, thermal_seed=9)
    b.step(60)
    r2 = stage.add(meds[2], dt=1e-13, steps=60, thermal_seed=9)
    assert stage.runs == [r2]
    b.remove(r0)
    b.adopt(r2)
    assert stage.runs == [] and b.runs == [r1, r2] and r2.batch is b
    b.step(60)
    st = b.stats([r1, r2])
    for r, m, k, s in ((r1, meds[1], 120, st[0]), (r2, meds[2], 60, st[1])):
        g = GpuSim(m, precision=FP64, thermal_seed=9)
        sg = g.step(k, 1e-13)
        assert np.array_equal(r.get_state(0), g.get_state(0))
        assert s["step"] == k and np.array_equal(s["mave"], sg["mave"])
        g.close()
    # a large run removed between calls: its memory is back after the next stats
    big = b.add(media.mh_medium(512, seed=5), dt=1e-13, steps=16)
    b.step(16)
    free0, _ = device_memory(0)
    b.remove(big)
    b.stats([r1])
    free1, _ = device_memory(0)
    assert free1 - free0 > 48 * 1024 * 1024, (free0, free1)
    stage.close()
    b.close()


def test_adopt_refuses_other_precision(gpulib):
    """A run moves only between batches of one precision and device; a refused
    move leaves it where it was, still stepping."""
    from mrm_b200 import MrmError
    m = media.mh_medium(16, seed=36)
    b32, b64 = Batch(FP32), Batch(FP64)
    r = b64.add(m, dt=1e-13, steps=8)
    with pytest.raises(MrmError):
        b32.adopt(r)
    assert b64.runs == [r] and b32.runs == [] and r.batch is b64
    b64.step(8)
    assert r.get_time()[1] == 8
    b32.close()
    b64.close()


def test_packed_short_rows_match_alone(gpulib):
    """FP32 runs whose rows are shorter than the batch's longest get several
    rows per row task (2 to 8 here, next to a 128-grain-wide run); every run,
    a two-layer one and one with the STE time function among them, still
    steps bit for bit as it does alone (where it has the longest rows)."""
    from tests.helpers import two_layer
    big = media.mh_medium(128, seed=31, temperature=300.0)
    meds = [big, media.mh_medium(16, seed=32, temperature=300.0), media.mh_medium(32, seed=33, temperature=300.0),
            two_layer(32, 16, seed=34, temperature=300.0), media.mh_medium(64, seed=35, temperature=300.0)]
    lay = meds[4].layers[0]
    lay.func, lay.amp, lay.fgamma, lay.param, lay.scale = 4, 12000.0, 2e-11, 1e-12, 1.0
    b = Batch(FP32)
    runs = [b.add(m, dt=1e-13, steps=64, thermal_seed=40 + i) for i, m in enumerate(meds)]
    b.step(64)
    st = b.stats(runs)
    for i, (r, m) in enumerate(zip(runs, meds)):
        g = GpuSim(m, precision=FP32, thermal_seed=40 + i)
        sg = g.step(64, 1e-13)
        for l in range(m.n_lay):
            assert np.array_equal(r.get_state(l), g.get_state(l)), (i, l)
        assert np.array_equal(st[i]["mave"], sg["mave"]), i
        g.close()
    b.close()


def test_tensor_copy_matches_build(gpulib):
    m = media.mh_medium(32, seed=4)
    b = Batch(FP32)
    r1 = b.add(m, steps=50)
    r2 = b.add(m, steps=50, tensor_from=r1)
    b.step(50)
    assert np.array_equal(r1.get_state(0), r2.get_state(0))
    b.close()


def test_shared_tensor_copy_on_write(gpulib):
    """Runs whose tensor is copied from another run of the same geometry share
    its buffer; a later upload on the source gives the source a buffer of its
    own and leaves the copies' tensor as it was."""
    m = media.mh_medium(32, seed=4)
    b = Batch(FP32)
    r1 = b.add(m, steps=40)
    r2 = b.add(m, steps=40, tensor_from=r1)
    n2d = r1.download_tensor()
    r1.upload_tensor(2.0 * n2d)  # the source's tensor changes; r2 keeps the original
    b.step(40)
    g = GpuSim(m, precision=FP32, tensor=n2d)
    g.step(40, 1e-13)
    assert np.array_equal(r2.get_state(0), g.get_state(0))
    assert not np.array_equal(r1.get_state(0), r2.get_state(0))
    g.close()
    b.close()


def test_served_results_equal_alone(gpulib):
    reqs = [Request(0, 0.0, "mh", 32, 300.0, 300, 31), Request(1, 0.0, "write", 64, 260.0, 500, 32),
            Request(2, 0.0, "mh", 32, 340.0, 700, 33), Request(3, 0.05, "mh", 64, 300.0, 200, 34),
            Request(4, 0.05, "write", 32, 290.0, 450, 35)]
    srv = Server(precision=FP32, chunk=128, keep_state=True)
    out = srv.run(reqs)
    assert len(out["results"]) == len(reqs)
    for r in out["results"]:
        q = reqs[r["rid"]]
        g = GpuSim(q.medium(), precision=FP32, thermal_seed=q.seed)
        g.step(q.steps, 1e-13)
        assert np.array_equal(r["m"], g.get_state(0)), q
        g.close()
    srv.be.close()
