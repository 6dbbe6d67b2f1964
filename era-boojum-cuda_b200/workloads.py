"""Seeded synthetic workloads of the LDE path (no public dataset exists for it).

* uneven_batch: jobs of mixed size for the single-launch batch path --
  log_n uniform in {12..22}, column count log-uniform in [1, 256], blowup
  uniform in {2, 4, 8}.
* serving_stream: Poisson arrivals of LDE requests -- log_n uniform in
  {14..22}, columns log-uniform in [8, 512], blowup in {2, 4}.

Every job also carries a per-job seed for its input words (uniform in [0, p)).
"""
from __future__ import annotations

import math
import random
from dataclasses import dataclass

P = 0xFFFFFFFF00000001


@dataclass
class LdeSpec:
    log_n: int
    cols: int
    log_blowup: int
    seed: int
    arrival_s: float = 0.0

    @property
    def n(self) -> int:
        return 1 << self.log_n

    @property
    def in_words(self) -> int:
        return self.cols << self.log_n

    @property
    def out_words(self) -> int:
        return (self.cols << self.log_n) << self.log_blowup

    @property
    def bytes(self) -> int:
        return 8 * (self.in_words + self.out_words)


def _log_uniform_int(rng: random.Random, lo: int, hi: int) -> int:
    return max(lo, min(hi, int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))))


def uneven_batch(n_jobs: int = 96, seed: int = 42, log_n_range=(12, 22), cols_range=(1, 256),
                 log_blowups=(1, 2, 3), max_total_bytes: int | None = None) -> list[LdeSpec]:
    """The uneven batch; with max_total_bytes, jobs are drawn until the next one would not fit."""
    rng = random.Random(seed)
    jobs, total = [], 0
    for i in range(n_jobs):
        j = LdeSpec(rng.randint(*log_n_range), _log_uniform_int(rng, *cols_range), rng.choice(log_blowups),
                    seed * 1000 + i)
        if max_total_bytes is not None and total + j.bytes > max_total_bytes:
            continue
        jobs.append(j)
        total += j.bytes
    return jobs


def serving_stream(n_requests: int = 200, rate_per_s: float = 50.0, seed: int = 7, log_n_range=(14, 22),
                   cols_range=(8, 512), log_blowups=(1, 2)) -> list[LdeSpec]:
    rng = random.Random(seed)
    t, out = 0.0, []
    for i in range(n_requests):
        t += rng.expovariate(rate_per_s)
        out.append(LdeSpec(rng.randint(*log_n_range), _log_uniform_int(rng, *cols_range), rng.choice(log_blowups),
                           seed * 100000 + i, arrival_s=t))
    return out
