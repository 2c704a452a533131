"""Benchmark of the per-timestep grain dynamics on B200.

Workload (one GPU): the 65,536-grain medium -- 256 x 256 grains-as-nodes at
8 nm pitch, 10 nm thick, Ms 700 emu/cc, Hk 15 kOe sigma 5 %, easy axes within
3 deg, nearest-neighbour exchange 0.5 kOe, alpha 0.1, T = 300 K Philox thermal
field, FP32 state/field/FFT with FP64 tensor and FP64 reductions, demag as a
512 x 512 zero-padded FFT convolution, uniform field ramped +20 kOe -> -20 kOe
at 10 deg off normal over 2 ns, Heun dt = 0.1 ps.  Synthetic media (seeded).

One bench step = HEUN_PER_STEP (1,000) Heun steps of that run; K timed bench
steps = K * 1,000 Heun steps (K = 20 is the full 20,000-step run).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--gpus N > 1 runs under torch.distributed.run: one replica per GPU (the path
does not shard: independent media realisations), value = sum of grain-steps
over ranks / max rank time.  --impl reference times the CPU port of the
reference algorithm (oracle/, OpenMP, all host cores) on a bounded sample.
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
HEUN_PER_STEP = 1000
SIDE = 256
DT = 1e-13
WORKLOAD = "65,536-grain M(H) ramp, T=300 K, FP32, 512x512 zero-padded FFT demag, Heun 0.1 ps"

# DRAM traffic per launch of the dominant kernel from the ncu capture summarised
# in profiles/ (None until a capture exists for the current kernel version).
NCU_TRAFFIC_BYTES = None


def algorithmic_bytes(nx: int, ny: int, px: int, py: int, nl: int = 1, fp: int = 4) -> dict:
    """Bytes each kernel must move at minimum with this path's data layout.

    row predictor: H^ rows in + M^ rows out (2 * 3 ny (px/2+1) complex), per grain
      m, pa, pb (3 x 16 B), exchange CSR (4 B index + 4 x (4 B nbr + 4 B coef)),
      writes m*, d (2 x 16 B)                     -> 116 B/grain
    row corrector: same spectra, per grain m, m*, d, pa, pb (5 x 16 B),
      CSR 36 B, writes m (16 B)                    -> 132 B/grain
    column: M^ columns in + H^ out (2 * 3 ny (px/2+1) complex) + tensor
      (px/2+1) * 9 * (py/2+1) reals (nl^2 pairs)
    """
    c = 2 * fp
    spec = 3 * nl * ny * (px // 2 + 1) * c
    n = nx * ny * nl
    row_pred = 2 * spec + n * (3 * 16 + 36 + 2 * 16)
    row_corr = 2 * spec + n * (5 * 16 + 36 + 16)
    col = 2 * spec + (px // 2 + 1) * nl * nl * 9 * (py // 2 + 1) * fp
    return {"row_pred": row_pred, "col": col, "row_corr": row_corr}


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


def cpu_baseline_sample(threads: int, nsteps: int = 12, warm: int = 2):
    """Oracle port (FP64, OpenMP) timed on a bounded sample of the same workload."""
    from oracle import pyoracle
    pyoracle.set_threads(threads)
    med = make_medium()
    sim = pyoracle.OracleSim(med, rng_mode=1, seed=1)
    sim.step(warm, DT)
    t0 = time.perf_counter()
    sim.step(nsteps, DT)
    el = time.perf_counter() - t0
    n = med.n_grains
    return {"value": n * nsteps / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{nsteps} Heun steps of the {n}-grain workload (FP64 oracle, OpenMP, after {warm} warm-up steps; tensor build excluded)"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    from oracle import pyoracle
    pyoracle.build()
    pyoracle.set_threads(threads)
    med = make_medium()
    sim = pyoracle.OracleSim(med, rng_mode=1, seed=1)
    per = 4  # Heun steps per bench step: bounded sample
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
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded media)",
        "config": {"workload": WORKLOAD + f"; CPU sample of {per} Heun steps per bench step",
                   "grains": n, "heun_steps_per_bench_step": per},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{per} Heun steps x {args.steps} bench steps of the {n}-grain workload"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    global HEUN_PER_STEP
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--heun", type=int, default=HEUN_PER_STEP,
                    help="Heun steps per bench step (profiling runs use a small value)")
    ap.add_argument("--timing-only", action="store_true",
                    help="skip the e2e and per-kernel legs (profiling runs)")
    args = ap.parse_args()
    HEUN_PER_STEP = args.heun

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)

    from mrm_b200 import FP32, GpuSim, build
    build.build()

    med = make_medium(seed=1 + rank)
    n = med.n_grains
    sim = GpuSim(med, precision=FP32, device=local, thermal_seed=1 + rank)
    px, py = sim.fft_grid()
    ext = torch.cuda.ExternalStream(sim.stream(), device=local)

    # warm-up (untimed), then restart the run from t = 0 for the timed region
    for _ in range(args.warmup):
        sim.step(HEUN_PER_STEP, DT, stats=False)
    sim.set_time(0.0, 0)
    sim.set_state(0, med.m0[0])
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    hs, mhs = [], []
    hdir = np.array(med.layers[0].hdir)
    for k in range(args.steps):
        flush.fill_(float(k))  # L2 flush between timed iterations (256 MB > 126 MB L2)
        torch.cuda.synchronize()
        ev[k][0].record(ext)
        sim.enqueue(HEUN_PER_STEP, DT)
        ev[k][1].record(ext)
        st = sim.stats()  # waits; outside the event pair
        t = st["t"]
        hs.append(20000.0 - 40000.0 * min(1.0, t / 2e-9))
        mhs.append(float(st["mms_l"][0] @ hdir))
    torch.cuda.synchronize()
    clk = clocks.stop()
    dev_ms = sum(a.elapsed_time(b) for a, b in ev)
    if dist:
        tt = torch.tensor([dev_ms], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        dev_ms = float(tt.item())
    heun_total = HEUN_PER_STEP * args.steps
    value = world * n * heun_total / (dev_ms * 1e-3)

    if args.timing_only:
        if rank == 0:
            print(json.dumps({"timing_only": True, "value": value, "ms_per_step": dev_ms / args.steps}))
        sim.close()
        if dist:
            dist.destroy_process_group()
        return

    # end-to-end through the C ABI with host buffers: upload m, step, read stats + m
    m_host = torch.from_numpy(np.ascontiguousarray(med.m0[0])).pin_memory()
    m_out = np.zeros_like(med.m0[0])
    sim.set_time(0.0, 0)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(args.steps):
        sim.set_state(0, m_host.numpy())
        sim.step(HEUN_PER_STEP, DT, stats=True)
        m_out[:] = sim.get_state(0)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if dist:
        tt = torch.tensor([e2e_s], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    e2e_value = world * n * heun_total / e2e_s
    h2d = m_host.numel() * 8
    d2h = m_out.size * 8 + np.dtype(__import__("mrm_b200").STATS_DTYPE).itemsize

    # per-kernel CUDA-event timing on the launching stream (roofline of the dominant kernel)
    prof = sim.profile(50, DT)
    names = ["row_pred", "col", "row_corr", "col"]
    ab = algorithmic_bytes(med.nx, med.ny, px, py)
    per_kernel = {"row_pred": prof[0], "col": 0.5 * (prof[1] + prof[3]), "row_corr": prof[2]}
    dom = max(per_kernel, key=per_kernel.get)
    peak, peak_kind = measured_peaks()
    achieved = ab[dom] / (per_kernel[dom] * 1e-3) / 1e9
    sim.close()

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    hc, mr = coercivity(hs, mhs)
    n_chunks = math.ceil(HEUN_PER_STEP / 16)
    launches = args.steps * (4 * HEUN_PER_STEP + 2 * n_chunks)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded media, random-init grain properties)",
        "config": {"workload": WORKLOAD, "grains": n, "fft_grid": [px, py],
                   "heun_steps_per_bench_step": HEUN_PER_STEP, "form": "plain single run per GPU",
                   "parallelism": f"replicas x{world}",
                   "l2": "flushed (256 MB write) between timed bench steps"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                     "algorithmic_bytes": ab[dom], "avg_launch_ms": per_kernel[dom],
                     "traffic": NCU_TRAFFIC_BYTES,
                     "per_kernel_ms": per_kernel},
        "physics": {"Hc_Oe": hc, "Mr": mr, "m_h_samples": len(hs)},
    }
    if clk:
        line["clocks"] = clk
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample(os.cpu_count() or 1)
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
