"""Seeded synthetic workloads of the batched and served forms.

* batched: 64 independent realisations, grain counts log-uniform in
  [1,024, 65,536] with the square-lattice side rounded to a multiple of 32,
  Hk sigma uniform in [3 %, 10 %], T = 300 K, 5,000 Heun steps each, the
  M(H) ramp compressed into the run;
* served: Poisson arrivals (mean rate 200/s) of M(H)-loop and write-pattern
  requests, grain counts log-uniform in [1,024, 262,144] (side a multiple of
  32), T uniform in [250, 350] K, step counts uniform in [2,000, 20,000].
  Write requests drive the medium with the reference's STE time function (a
  trapezoidal square-wave field, applied.f90:363-377) of a 1.5 ns period.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

from . import media

DT = 1e-13


def side_of(n_grains: float) -> int:
    return max(32, int(round(math.sqrt(n_grains) / 32.0)) * 32)


def batched_media(n: int = 64, seed: int = 11, steps: int = 5000, lo: int = 1024, hi: int = 65536):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        ng = math.exp(rng.uniform(math.log(lo), math.log(hi)))
        side = side_of(ng)
        sigma = rng.uniform(0.03, 0.10)
        m = media.mh_medium(side, k_sigma=-sigma, temperature=300.0, seed=1000 + i,
                            ramp_s=steps * DT)
        out.append(m)
    return out


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float        # s after the stream start
    kind: str             # "mh" or "write"
    side: int
    temperature: float
    steps: int
    seed: int
    timeout: Optional[float] = None  # s after arrival; the server gives up on the request then

    @property
    def grains(self) -> int:
        return self.side * self.side

    def medium(self):
        if self.kind == "mh":
            return media.mh_medium(self.side, temperature=self.temperature, seed=self.seed,
                                   ramp_s=self.steps * DT)
        m = media.mh_medium(self.side, temperature=self.temperature, seed=self.seed)
        lay = m.layers[0]
        # write pattern: +-12 kOe square wave (STE) at 20 deg, 1.5 ns period, 50 ps rise
        a = math.radians(20.0)
        lay.hdir = (math.sin(a), 0.0, -math.cos(a))
        lay.func, lay.amp, lay.fgamma, lay.param, lay.dc, lay.scale = 4, 12000.0, 1.5e-9, 5e-11, 0.0, 1.0
        return m


def served_requests(n: int = 1000, rate: float = 200.0, seed: int = 7, lo: int = 1024,
                    hi: int = 262144, steps_lo: int = 2000, steps_hi: int = 20000) -> List[Request]:
    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        ng = math.exp(rng.uniform(math.log(lo), math.log(hi)))
        reqs.append(Request(rid=i, arrival=t, kind="mh" if rng.random() < 0.5 else "write",
                            side=side_of(ng), temperature=float(rng.uniform(250.0, 350.0)),
                            steps=int(rng.integers(steps_lo, steps_hi + 1)), seed=10000 + i))
    return reqs
