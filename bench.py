"""Benchmark of the per-timestep grain dynamics on B200.

Headline workload (one GPU): the batched form over B (default 32) independent
realisations of the 65,536-grain medium -- 256 x 256 grains-as-nodes at 8 nm
pitch, 10 nm thick, Ms 700 emu/cc, Hk 15 kOe sigma 5 %, easy axes within 3 deg,
nearest-neighbour exchange 0.5 kOe, alpha 0.1, T = 300 K Philox thermal field
(one seed per realisation), FP32 state/field/FFT with FP64 tensor and FP64
reductions, demag as a 512 x 512 zero-padded FFT convolution, uniform field
ramped +20 kOe -> -20 kOe at 10 deg off normal over 2 ns, Heun dt = 0.1 ps --
advanced by one graph-captured launch sequence per Heun stage.  Synthetic
media (seeded).  One bench step = HEUN_PER_STEP (100) Heun steps of every
realisation; K = 200 timed bench steps = the full 20,000-step, 2 ns run.

Beside the headline (sub-objects of the same JSON line):
  plain    the same medium as one plain single run (the drop-in; the
           denominator of the batched/plain ratio), full 2 ns ramp, L2 flushed
           between timed chunks; its coercivity against an FP64 run of the
           same medium and seed;
  mix      64 realisations with grain counts log-uniform in [1,024, 65,536],
           Hk sigma in [3 %, 10 %], 5,000 Heun steps each, one batch;
  write    the two-layer 1,024 x 256 recording write by the moving Karlqvist
           head (PRBS pattern), a bounded 2,000-step sample;
  served   the first 200 requests of the Poisson request stream (200 req/s,
           M(H) and write requests of 1,024..262,144 grains, 2,000..20,000
           steps): aggregate grain-steps/s and p50/p99 latency.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--gpus N > 1 runs under torch.distributed.run: one replica of the headline
batch per GPU (the path does not shard: independent media realisations),
value = grain-steps of all ranks / max rank time; the sub-objects run on rank
0 only.  --impl reference times the CPU port of the reference algorithm
(oracle/, OpenMP, all host cores) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "grain-steps/s (1 B200) batched/served vs plain GPU at <=1% Hc err; p50/p99 latency"
UNIT = "grain-steps/s"
HEUN_PER_STEP = 100
SIDE = 256
DT = 1e-13
RAMP_STEPS = 20000  # 2 ns at 0.1 ps
WORKLOAD = ("batched {b} x 65,536-grain M(H) ramp realisations, T=300 K, FP32, "
            "512x512 zero-padded FFT demag, Heun 0.1 ps")

# DRAM traffic per launch of each kernel in bytes per grain of the launch:
# dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture of the
# headline batch (32 x 65,536 grains, row shape 1, the register column kernel
# {128 threads, 4 blocks/SM}, one column per task), divided by its grains; a
# kernel change calls for a new capture
NCU_TRAFFIC_BYTES_PER_GRAIN = {"row_pred": 141.0, "col": 35.7, "row_corr": 164.4}


def algorithmic_bytes(nx: int, ny: int, px: int, py: int, nl: int = 1, fp: int = 4, runs: int = 1,
                      tensors: int = 1) -> dict:
    """Bytes each kernel must move at minimum with this path's data layout, for
    `runs` runs of one geometry that read `tensors` tensor copies (runs whose
    tensor comes from another run of the same geometry share its buffer).

    row predictor: H^ rows in + M^ rows out (2 * 3 ny (px/2+1) complex), per grain
      m, pa, pb (3 x 16 B), exchange CSR (4 B index + 4 x (4 B nbr + 4 B coef)),
      writes m*, d (2 x 16 B)                     -> 116 B/grain
    row corrector: same spectra, per grain m, m*, d, pa, pb (5 x 16 B),
      CSR 36 B, writes m (16 B)                    -> 132 B/grain
    column: M^ columns in + H^ out (2 * 3 ny (px/2+1) complex) per run, plus
      the tensor: one layer, the symmetric tensor's six components at every
      k_y of the (px/2+1) columns (the register column kernel's layout:
      6 py reals per column); more layers, nine components per layer pair at
      0 <= k_y <= py/2
    """
    c = 2 * fp
    spec = 3 * nl * ny * (px // 2 + 1) * c
    n = nx * ny * nl
    row_pred = 2 * spec + n * (3 * 16 + 36 + 2 * 16)
    row_corr = 2 * spec + n * (5 * 16 + 36 + 16)
    tensor = ((px // 2 + 1) * 6 * py * fp if nl == 1 else (px // 2 + 1) * nl * nl * 9 * (py // 2 + 1) * fp)
    col = runs * 2 * spec + tensors * tensor
    return {"row_pred": runs * row_pred, "col": col, "row_corr": runs * row_corr}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.proc = None
        self.gpu = gpu_index
        self.path = os.path.join("/tmp", f"mrm_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def make_medium(seed: int = 1):
    from mrm_b200 import media
    return media.mh_medium(SIDE, boundary=1, temperature=300.0, seed=seed)


def applied(t: float) -> float:
    return 20000.0 - 40000.0 * min(1.0, max(0.0, t / (RAMP_STEPS * DT)))


def coercivity(h, mh):
    """Hc, Mr from a descending M(H) branch by linear interpolation of the sign changes."""
    h, mh = np.asarray(h), np.asarray(mh)
    hc = mr = None
    for k in range(1, len(h)):
        if mh[k - 1] > 0 >= mh[k] and hc is None:
            hc = -(h[k - 1] + (h[k] - h[k - 1]) * mh[k - 1] / (mh[k - 1] - mh[k]))
        if h[k - 1] > 0 >= h[k] and mr is None:
            mr = mh[k - 1] + (mh[k] - mh[k - 1]) * h[k - 1] / (h[k - 1] - h[k])
    return hc, mr


def cpu_model() -> str:
    try:
        for line in subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout.splitlines():
            if line.startswith("Model name:"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def oracle_rate(threads: int, fft_bits: int, min_s: float, chunk: int = 10, max_steps: int = 2000) -> float:
    """Grain-steps/s of the CPU port (oracle/) on one 65,536-grain realisation of
    the headline medium: `threads` OpenMP threads, FP32 or FP64 FFT grids
    (the reference's default single-precision FFTW build or its FFTD=1
    build; state and fields FP64 in both), timed after 2 warm-up steps."""
    from oracle import pyoracle
    pyoracle.build()
    pyoracle.set_threads(threads)
    med = make_medium()
    sim = pyoracle.OracleSim(med, rng_mode=1, seed=1, fft_bits=fft_bits)
    sim.step(2, DT)
    done, t0 = 0, time.perf_counter()
    while done < max_steps:
        sim.step(chunk, DT)
        done += chunk
        if time.perf_counter() - t0 >= min_s:
            break
    el = time.perf_counter() - t0
    sim.close()
    return med.n_grains * done / el


def cpu_baseline_sample(threads: int, reps: int = 3, min_s: float = 3.0):
    """The CPU port on the host cores: FP32 grids on all threads (median of
    `reps` samples; the like-precision baseline of the FP32 GPU path), FP64 on
    all threads, FP32 on 4 threads (the reference's own openmp setting) and on
    1 thread.  About 20 s of CPU work."""
    from oracle import pyoracle
    f32 = sorted(oracle_rate(threads, 32, min_s) for _ in range(reps))
    variants = {
        f"fp32_{threads}t_median_of_{reps}": f32[len(f32) // 2],
        f"fp64_{threads}t": oracle_rate(threads, 64, min_s),
        "fp32_4t": oracle_rate(min(4, threads), 32, min_s),
        "fp32_1t": oracle_rate(1, 32, min_s),
    }
    # the write leg's readback call on the oracle (initial state of the same medium)
    from mrm_b200 import media
    pyoracle.set_threads(threads)
    wsim = pyoracle.OracleSim(media.head_write_medium(1024, 256, seed=1, prbs_seed=1, temperature=300.0),
                              rng_mode=1, seed=1, demag=False)
    t0 = time.perf_counter()
    wsim.off_field(**READBACK)
    off_ms = (time.perf_counter() - t0) * 1e3
    wsim.close()
    return {"value": f32[len(f32) // 2], "unit": UNIT, "cores": threads, "kind": "port",
            "cpu": cpu_model(), "nproc": os.cpu_count(),
            "sample": f"Heun steps of one 65,536-grain realisation for {min_s:.0f} s per sample after 2 warm-up "
                      f"steps (oracle port, OpenMP, FP32 FFT grids with FP64 state and fields; tensor build "
                      f"excluded); value: median of {reps} samples on {threads} threads",
            "variants": variants, "readback_ms_per_call": off_ms}


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    from oracle import pyoracle
    pyoracle.build()
    pyoracle.set_threads(threads)
    med = make_medium()
    # FP32 FFT grids, as the reference's default single-precision FFTW build
    sim = pyoracle.OracleSim(med, rng_mode=1, seed=1, fft_bits=32)
    per = 4  # Heun steps of one realisation per bench step: a bounded sample
    for _ in range(args.warmup):
        sim.step(per, DT)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sim.step(per, DT)
    el = time.perf_counter() - t0
    n = med.n_grains
    value = n * per * args.steps / el
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded media)",
        "config": {"workload": WORKLOAD.format(b=args.batch) +
                   f"; CPU sample: {per} Heun steps of one realisation per bench step",
                   "grains": n, "heun_steps_per_bench_step": per,
                   "precision": "FP32 FFT grids, FP64 state and fields (the reference's default build)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "cpu": cpu_model(),
                         "sample": f"{per} Heun steps x {args.steps} bench steps of one {n}-grain realisation"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def max_over_ranks(value: float, dist, device) -> float:
    """Largest value over the ranks (a timed region's duration: the job ends
    with its slowest replica); the value itself on a single process."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank: float, world: int, seconds: float) -> float:
    """Whole-job throughput of `world` replicas that each processed
    units_per_rank within `seconds` (the max over ranks)."""
    return world * units_per_rank / seconds


def launches_per_bench_step(heun: int, stats: bool = True) -> int:
    """Kernels per call of `heun` Heun steps: 4 per step, one advance per graph of
    <= 16 steps, one stats finalisation per call."""
    return 4 * heun + math.ceil(heun / 16) + (1 if stats else 0)


def batched_leg(args, torch, local, rank, dist):
    """Headline: B realisations of the 65,536-grain medium in one batch."""
    from mrm_b200 import FP32, STATS_DTYPE
    from mrm_b200.batch import Batch

    b = Batch(FP32, local)
    meds = [make_medium(seed=1 + rank * args.batch + i) for i in range(args.batch)]
    runs = []
    for i, med in enumerate(meds):
        runs.append(b.add(med, dt=DT, thermal_seed=1 + rank * args.batch + i,
                          tensor_from=runs[0] if runs else None))
    if args.shape:
        runs[0].set_shape(*[int(x) for x in args.shape.split(",")])
    n = meds[0].n_grains
    ext = torch.cuda.ExternalStream(b.stream(), device=local)
    hdirs = [np.array(m.layers[0].hdir) for m in meds]

    def reset():
        for r, med in zip(runs, meds):
            r.set_state(0, med.m0[0])
            r.set_time(0.0, 0)

    for _ in range(args.warmup):
        b.step(args.heun)
    reset()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    hs, mhs = [], []
    for k in range(args.steps):
        ev[k][0].record(ext)
        b.enqueue(args.heun)
        ev[k][1].record(ext)
        st = b.stats(runs)  # waits; outside the event pair
        hs.append(applied(float(st[0]["t"])))
        mhs.append([float(st[i]["mms_l"][0] @ hdirs[i]) for i in range(len(runs))])
    torch.cuda.synchronize()
    clk = clocks.stop()
    dev_ms = sum(a.elapsed_time(c) for a, c in ev)
    dev_ms = max_over_ranks(dev_ms, dist, f"cuda:{local}")
    mh = np.array(mhs)
    hcs = [coercivity(hs, mh[:, i])[0] for i in range(len(runs))]
    hcs = [h for h in hcs if h is not None]

    # end to end through the public API with host buffers: each bench step uploads
    # every realisation's m, advances the batch and reads back its stats and m
    reset()
    m_host = [torch.from_numpy(np.ascontiguousarray(med.m0[0])).pin_memory().numpy() for med in meds]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    k_e2e = max(1, min(args.steps, args.e2e_steps))
    t0 = time.perf_counter()
    for k in range(k_e2e):
        for r, m in zip(runs, m_host):
            r.set_state(0, m)
        b.step(args.heun)
        st = b.stats(runs)
        for i, r in enumerate(runs):
            r.get_state(0, out=m_host[i])
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, dist, f"cuda:{local}")
    h2d = sum(m.nbytes for m in m_host)
    d2h = sum(m.nbytes for m in m_host) + len(runs) * STATS_DTYPE.itemsize

    # per-kernel CUDA-event timing on the batch's stream
    prof = b.profile(20)
    px, py = runs[0].fft_grid()
    occ = b.occupancy()
    shape = runs[0].get_shape()
    b.close()
    return {"n": n, "runs": len(runs), "dev_ms": dev_ms, "clocks": clk, "hcs": hcs,
            "e2e_s": e2e_s, "k_e2e": k_e2e, "h2d": h2d, "d2h": d2h, "prof": prof, "fft": (px, py),
            "occupancy": occ, "shape": shape, "samples": len(hs)}


GOLDEN_C2 = os.path.join(ROOT, "tests", "golden", "c2_mh.npz")


def physics_leg(local):
    """The Hc/Mr gate on the headline medium: the FP32 batched path over the
    full 20,000-step ramp, one realisation per seed of the committed oracle
    ensemble (tests/golden/c2_mh.npz, FP64 oracle, same medium and ramp), and
    the relative error of the ensemble means of coercivity and remanence."""
    from mrm_b200 import FP32
    from mrm_b200.batch import Batch
    if not os.path.exists(GOLDEN_C2):
        return {"oracle_ensemble": "absent"}
    g = np.load(GOLDEN_C2)
    seeds = [int(x) for x in g["seeds"]]
    b = Batch(FP32, local)
    runs = []
    for sd in seeds:
        runs.append(b.add(make_medium(seed=1), dt=DT, thermal_seed=sd, tensor_from=runs[0] if runs else None))
    hdir = np.array(make_medium(seed=1).layers[0].hdir)
    hs, mhs = [], []
    for _ in range(RAMP_STEPS // HEUN_PER_STEP):
        b.step(HEUN_PER_STEP)
        st = b.stats(runs)
        hs.append(applied(float(st[0]["t"])))
        mhs.append([float(x["mms_l"][0] @ hdir) for x in st])
    b.close()
    mh = np.array(mhs)
    hm = [coercivity(hs, mh[:, i]) for i in range(len(seeds))]
    hc = np.array([x[0] for x in hm], float)
    mr = np.array([x[1] for x in hm], float)
    return {"workload": f"{len(seeds)} realisations of the 65,536-grain medium (seeds {seeds}), full 2 ns ramp, "
                        "FP32 batched path",
            "hc_mean_oe": float(hc.mean()), "mr_mean": float(mr.mean()),
            "oracle_hc_mean_oe": float(g["hc"].mean()), "oracle_mr_mean": float(g["mr"].mean()),
            "hc_rel_err_vs_oracle_ensemble": float(hc.mean() / g["hc"].mean() - 1.0),
            "mr_rel_err_vs_oracle_ensemble": float(mr.mean() / g["mr"].mean() - 1.0),
            "oracle_hc_seed_spread_oe": float(np.std(g["hc"])),
            "gate": "|rel err| <= 1 % for Hc and Mr"}


def plain_leg(torch, local, precision, heun_chunk=100, total=RAMP_STEPS, flush_l2=True):
    """One plain single run of the 65,536-grain medium over the full ramp."""
    from mrm_b200 import GpuSim
    med = make_medium(seed=1)
    sim = GpuSim(med, precision=precision, device=local, thermal_seed=1)
    ext = torch.cuda.ExternalStream(sim.stream(), device=local)
    sim.step(3 * heun_chunk, DT, stats=False)  # warm-up: graphs, clocks
    sim.set_time(0.0, 0)
    sim.set_state(0, med.m0[0])
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    hdir = np.array(med.layers[0].hdir)
    nchunks = total // heun_chunk
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(nchunks)]
    hs, mhs = [], []
    torch.cuda.synchronize()
    for k in range(nchunks):
        if flush_l2:
            flush.fill_(float(k))  # 256 MB > 126 MB L2
            torch.cuda.synchronize()
        ev[k][0].record(ext)
        sim.enqueue(heun_chunk, DT)
        ev[k][1].record(ext)
        st = sim.stats()
        hs.append(applied(float(st["t"])))
        mhs.append(float(st["mms_l"][0] @ hdir))
    torch.cuda.synchronize()
    dev_ms = sum(a.elapsed_time(c) for a, c in ev)
    prof = sim.profile(50, DT)
    sim.close()
    del flush
    hc, mr = coercivity(hs, mhs)
    n = med.n_grains
    return {"value": n * nchunks * heun_chunk / (dev_ms * 1e-3), "us_per_heun_step":
            1e3 * dev_ms / (nchunks * heun_chunk), "hc_oe": hc, "mr": mr, "prof": prof}


# readback slab 1 nm above the media, 1 nm thick, no images (lengths in cm)
READBACK = dict(zoff=1e-7, dzobs=1e-7, num_images=0)
READBACK_TEXT = "(slab 1 nm above the media, 1 nm thick, FP64 tensor, FFTs and products on the device)"


def write_leg(torch, local, steps=2000):
    """The two-layer recording write (1,024 x 256 grains per layer, 7 nm pitch,
    Karlqvist head at 20 m/s writing a 64-bit PRBS at 15 nm bits, T = 300 K,
    FP32, Heun) as one plain run: a bounded sample of the 480,000-step write."""
    from mrm_b200 import FP32, GpuSim, media
    med = media.head_write_medium(1024, 256, seed=1, prbs_seed=1, temperature=300.0)
    sim = GpuSim(med, precision=FP32, device=local, thermal_seed=1)
    ext = torch.cuda.ExternalStream(sim.stream(), device=local)
    sim.step(48, DT, stats=False)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    sim.enqueue(steps, DT)
    e1.record(ext)
    st = sim.stats()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    px, py = sim.fft_grid()
    # readback field of the written track (plot_off_field): one synchronous call
    # through the public API, the field copied back to host memory
    sim.off_field(**READBACK)
    t0 = time.perf_counter()
    for _ in range(3):
        hr = sim.off_field(**READBACK)
    off_ms = (time.perf_counter() - t0) / 3 * 1e3
    sim.close()
    grains = 2 * 1024 * 256
    return {"workload": f"two-layer 1024x256x2 head write (gap 25 nm, fly 6 nm, 12 kOe, 20 m/s, 64-bit PRBS "
                        f"at 15 nm), T=300 K, FP32, {px}x{py} padded FFT, {steps} Heun steps of the 480,000",
            "grains": grains, "value": grains * steps / (ms * 1e-3), "unit": UNIT, "device_ms": ms,
            "us_per_heun_step": 1e3 * ms / steps, "mave_top": np.asarray(st["mave_l"][0]).tolist(),
            "readback": {"call": "off_field " + READBACK_TEXT, "grid": [1024, 256], "ms_per_call": off_ms,
                         "hz_rms_oe": float(np.sqrt(np.mean(hr[2] ** 2)))},
            "tabulated": table_write_leg(torch, local, steps),
            "windowed": window_write_leg(torch, local, steps)}


def window_write_leg(torch, local, steps):
    """A longer track (2048 x 256 grains x 2 layers) written by the tabulated
    head with a moving demag window of 512 x 256 cells centred on it (nxfft <
    nx): only the window's grains are evaluated and pushed, the FFT covers the
    window.  Value: grain-steps/s of the pushed (windowed) grains."""
    from mrm_b200 import FP32, GpuSim, media
    med = media.table_write_medium(2048, 256, seed=1, temperature=300.0)
    med.window = dict(nx=512, ny=256, v=(2000.0, 0.0), offset=(-0.5 * 2048 * med.dx, 0.0))
    sim = GpuSim(med, precision=FP32, device=local, thermal_seed=1)
    ext = torch.cuda.ExternalStream(sim.stream(), device=local)
    sim.set_time(3.6e-7, 0)  # the head 7.2 um (1,029 cells) down the track, the window centred on it
    sim.step(48, DT, stats=False)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    sim.enqueue(steps, DT)
    e1.record(ext)
    sim.stats()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    px, py = sim.fft_grid()
    win = sim.get_window()
    sim.close()
    active = 2 * 512 * 256
    return {"workload": f"two-layer 2048x256x2 track, tabulated head at 20 m/s, 512x256 demag window following "
                        f"it ({px}x{py} FFT), T=300 K, FP32, {steps} Heun steps",
            "value": active * steps / (ms * 1e-3), "unit": UNIT, "us_per_heun_step": 1e3 * ms / steps,
            "window_origin": list(win[2:])}


def table_write_leg(torch, local, steps):
    """The same write driven by a tabulated head-field profile per layer (97 x 33
    nodes, bilinear per cell, the way the reference drives writes) instead of
    the analytic head: the field-table path's cost in the stepping kernels."""
    from mrm_b200 import FP32, GpuSim, media
    med = media.table_write_medium(1024, 256, seed=1, temperature=300.0)
    sim = GpuSim(med, precision=FP32, device=local, thermal_seed=1)
    ext = torch.cuda.ExternalStream(sim.stream(), device=local)
    sim.step(48, DT, stats=False)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    sim.enqueue(steps, DT)
    e1.record(ext)
    sim.stats()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    sim.close()
    grains = 2 * 1024 * 256
    return {"workload": f"two-layer 1024x256x2 write, tabulated head profile (97 x 33 nodes) at 20 m/s, "
                        f"STE polarity, T=300 K, FP32, {steps} Heun steps",
            "value": grains * steps / (ms * 1e-3), "unit": UNIT, "us_per_heun_step": 1e3 * ms / steps}


def llb_leg(torch, local, steps=2000):
    """The heat-assisted LLB workload (f3): a 256 x 256-grain FePt-like layer at
    T = 600 K below a distributed Tc ~ 700 K with thermal noise and a reversing
    field, push_llb's Heun branch with |m| per grain, FP32 state (the push in
    FP64 arithmetic), one plain run."""
    from mrm_b200 import FP32, GpuSim, media
    med = media.llb_medium(256, seed=1)
    sim = GpuSim(med, precision=FP32, device=local, thermal_seed=1)
    ext = torch.cuda.ExternalStream(sim.stream(), device=local)
    sim.step(48, 1e-14, stats=False)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    sim.enqueue(steps, 1e-14)
    e1.record(ext)
    st = sim.stats()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    mag = float(np.mean(sim.get_mag(0)))
    sim.close()
    n = med.n_grains
    return {"workload": f"LLB heat-assisted layer 256x256 (T 600 K, Tc ~ 700 K +- 3 %, S = 1/2, 8 kOe reversing), "
                        f"FP32, {steps} Heun steps of 10 fs",
            "value": n * steps / (ms * 1e-3), "unit": UNIT, "us_per_heun_step": 1e3 * ms / steps,
            "mean_abs_m": mag, "mave_z": float(st["mave"][2])}


def mix_leg(torch, local, steps=5000, nreal=64):
    from mrm_b200 import FP32
    from mrm_b200.batch import Batch
    from mrm_b200.workloads import batched_media
    meds = batched_media(nreal, steps=steps)
    b = Batch(FP32, local)
    for i, med in enumerate(meds):
        b.add(med, dt=DT, steps=steps, thermal_seed=100 + i)
    ext = torch.cuda.ExternalStream(b.stream(), device=local)
    b.step(16)  # warm-up: task tables, attributes, first graph
    for r, med in zip(b.runs, meds):
        r.set_state(0, med.m0[0])
        r.set_time(0.0, 0)
        r.set_run(DT, steps)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    b.enqueue(steps)
    e1.record(ext)
    b.stats()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    grains = sum(m.n_grains for m in meds)
    b.close()
    return {"workload": f"{nreal} realisations, grain counts log-uniform 1,024..65,536 (side a multiple "
                        f"of 32), Hk sigma 3..10 %, T=300 K, FP32, {steps} Heun steps each",
            "grains": grains, "value": grains * steps / (ms * 1e-3), "unit": UNIT, "device_ms": ms}


def served_leg(local, nreq):
    from mrm_b200 import FP32
    from mrm_b200.serve import GpuBackend, Server
    from mrm_b200.workloads import served_requests
    reqs = served_requests(nreq)
    be = GpuBackend(FP32, local)
    srv = Server(backend=be)
    out = srv.run(reqs)
    be.close()
    return {"workload": f"first {nreq} requests of the seeded Poisson stream (200 req/s, M(H) and STE "
                        "write requests, 1,024..262,144 grains, T 250..350 K, 2,000..20,000 Heun steps)",
            "requests": nreq, "completed": out["completed"], "value": out["grain_steps_per_s"], "unit": UNIT,
            "p50_latency_s": out["p50_latency_s"], "p99_latency_s": out["p99_latency_s"],
            "latency_over": f"the {out['completed']} completed requests, arrival to result",
            "wall_s": out["wall_s"], "launch_calls": out["calls"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=RAMP_STEPS // HEUN_PER_STEP)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=32, help="realisations in the headline batch")
    ap.add_argument("--heun", type=int, default=HEUN_PER_STEP, help="Heun steps per bench step")
    ap.add_argument("--e2e-steps", type=int, default=50, help="bench steps of the end-to-end leg")
    ap.add_argument("--served", type=int, default=200, help="requests of the served sample (0: skip)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--shape", default="",
                    help="row,column,columns-per-task kernel shapes of the batch (default: autotuned)")
    ap.add_argument("--headline-only", action="store_true",
                    help="only the headline batch (profiling runs)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    dist = None
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from mrm_b200 import FP32, FP64, build
    build.build()

    B = batched_leg(args, torch, local, rank, dist)
    if dist:
        dist.destroy_process_group()  # the sub-objects run on rank 0 alone
    if rank != 0:
        return
    n, nb = B["n"], B["runs"]
    value = job_throughput(nb * n * args.heun * args.steps, world, B["dev_ms"] * 1e-3)
    e2e_value = job_throughput(nb * n * args.heun * B["k_e2e"], world, B["e2e_s"])
    px, py = B["fft"]
    # every run of the batch shares the first run's tensor (same geometry)
    ab = algorithmic_bytes(SIDE, SIDE, px, py, runs=nb, tensors=1)
    prof = B["prof"]
    per_kernel = {"row_pred": prof[0], "col": 0.5 * (prof[1] + prof[3]), "row_corr": prof[2]}
    launches_per_heun = {"row_pred": 1, "col": 2, "row_corr": 1}
    # dominant kernel: the largest share of a Heun step's device time
    dom = max(per_kernel, key=lambda k: per_kernel[k] * launches_per_heun[k])
    peak, peak_kind = measured_peaks()
    achieved = ab[dom] / (per_kernel[dom] * 1e-3) / 1e9
    hc_mean = float(np.mean(B["hcs"])) if B["hcs"] else None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": B["dev_ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded media, random-init grain properties)",
        "config": {"workload": WORKLOAD.format(b=nb), "realisations_per_gpu": nb, "grains_per_realisation": n,
                   "fft_grid": [px, py], "heun_steps_per_bench_step": args.heun,
                   "form": "batched: one launch sequence per Heun stage over every realisation",
                   "parallelism": f"replicas x{world}",
                   "l2": f"inputs larger than L2 ({nb} realisations, ~{nb * 17} MB resident)"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": B["h2d"], "d2h_bytes_per_step": B["d2h"],
                "bench_steps": B["k_e2e"]},
        "gpu_launches": args.steps * launches_per_bench_step(args.heun),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                     "algorithmic_bytes": ab[dom], "avg_launch_ms": per_kernel[dom],
                     "traffic": (NCU_TRAFFIC_BYTES_PER_GRAIN[dom] * nb * n
                                 if dom in NCU_TRAFFIC_BYTES_PER_GRAIN else None),
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch, 32 x 65,536 "
                                       "grains, row shape 1, register column kernel 128 x 4, 1 column per task",
                     "per_kernel_ms": per_kernel, "launches_per_heun_step": launches_per_heun,
                     "per_kernel_frac": {k: ab[k] / (v * 1e-3) / 1e9 / peak for k, v in per_kernel.items()},
                     "occupancy_blocks_per_sm": {"row": B["occupancy"][0], "col": B["occupancy"][1]},
                     "kernel_shapes": {"row": B["shape"][0], "col": B["shape"][1], "cols_per_task": B["shape"][2]}},
        "physics": {"hc_mean_oe": hc_mean,
                    "hc_std_oe": float(np.std(B["hcs"])) if B["hcs"] else None,
                    "hc_realisations": len(B["hcs"]), "m_h_samples": B["samples"]},
    }
    if B["clocks"]:
        line["clocks"] = B["clocks"]
    if not args.headline_only:
        p32 = plain_leg(torch, local, FP32)
        p64 = plain_leg(torch, local, FP64, flush_l2=False)
        hc_err = (abs(p32["hc_oe"] - p64["hc_oe"]) / abs(p64["hc_oe"])
                  if p32["hc_oe"] and p64["hc_oe"] else None)
        line["plain"] = {"workload": "one 65,536-grain realisation (seed 1), full 2 ns ramp, FP32",
                         "value": p32["value"], "unit": UNIT, "us_per_heun_step": p32["us_per_heun_step"],
                         "batched_over_plain": value / world / p32["value"],
                         "per_kernel_ms": {"row_pred": p32["prof"][0], "col": 0.5 * (p32["prof"][1] + p32["prof"][3]),
                                           "row_corr": p32["prof"][2]},
                         "l2": "flushed (256 MB write) between timed 100-step chunks"}
        line["physics"].update({"hc_fp32_oe": p32["hc_oe"], "hc_fp64_oe": p64["hc_oe"], "hc_rel_err_fp32_vs_fp64": hc_err,
                                "mr_fp32": p32["mr"], "mr_fp64": p64["mr"],
                                "fp64_us_per_heun_step": p64["us_per_heun_step"]})
        line["physics"]["vs_oracle"] = physics_leg(local)
        line["mix"] = mix_leg(torch, local)
        line["write"] = write_leg(torch, local)
        line["llb"] = llb_leg(torch, local)
        if args.served > 0:
            line["served"] = served_leg(local, args.served)
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_sample(os.cpu_count() or 1)
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
