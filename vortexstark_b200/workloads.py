"""Proof workloads over the slot engine: plain (one job at a time), batched (a
job list submitted at once) and served (seeded Poisson arrivals, continuous
admission). Job mixes follow the benchmark definitions:

* plain:   Fibonacci proofs, a0 = 1, a1 seeded, fixed log_n (65,536 rows by default);
* batched: 64 jobs, log_n uniform in 16..22, each either a Fibonacci proof
           (a1 seeded) or a commitment of 1..34 seeded uniform-M31 columns;
* served:  arrivals with exponential gaps (mean 5 ms, 200 jobs/s); half
           Fibonacci proofs at log_n 16/20/24 with weights 0.5/0.3/0.2, half
           34-column commitments at log_n 18/20/22; HBM budget 150 GB.
"""
from __future__ import annotations

import math
import statistics
import threading
import time

from .api import COMMIT, FIB, Engine, commit_job, commit_seeded, fib_job, prove_fib

P = 0x7FFFFFFF


class SplitMix64:
    M = (1 << 64) - 1

    def __init__(self, seed: int):
        self.s = seed & self.M

    def next(self) -> int:
        self.s = (self.s + 0x9E3779B97F4A7C15) & self.M
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & self.M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & self.M
        return z ^ (z >> 31)

    def m31(self) -> int:
        while True:
            v = self.next() >> 33
            if v != P:
                return v

    def uniform(self) -> float:  # [0, 1)
        return (self.next() >> 11) / float(1 << 53)

    def below(self, k: int) -> int:
        return self.next() % k


def plain_jobs(n: int, log_n: int = 16, seed: int = 0x56530000):
    g = SplitMix64(seed)
    return [fib_job(log_n, 1, g.m31()) for _ in range(n)]


def batched_jobs(n: int = 64, seed: int = 0x56530003):
    g = SplitMix64(seed)
    jobs = []
    for _ in range(n):
        log_n = 16 + g.below(7)
        if g.below(2) == 0:
            jobs.append(fib_job(log_n, 1, g.m31()))
        else:
            jobs.append(commit_job(log_n, 1 + g.below(34), g.next()))
    return jobs


def served_arrivals(n: int, seed: int = 0x56530004, rate: float = 200.0):
    """[(arrival_offset_s, job, size_class)]"""
    g = SplitMix64(seed)
    t, out = 0.0, []
    for _ in range(n):
        t += -math.log(1.0 - g.uniform()) / rate
        if g.below(2) == 0:
            u = g.uniform()
            log_n = 16 if u < 0.5 else (20 if u < 0.8 else 24)
            out.append((t, fib_job(log_n, 1, g.m31()), f"fib{log_n}"))
        else:
            log_n = (18, 20, 22)[g.below(3)]
            out.append((t, commit_job(log_n, 34, g.next()), f"commit34x{log_n}"))
    return out


def shapes(jobs):
    seen, out = set(), []
    for j in jobs:
        key = (j.kind, j.log_n)
        if key not in seen:
            seen.add(key)
            out.append(j)
    return out


def run_list(engine: Engine, jobs, sequential: bool):
    """Runs jobs; sequential waits for each before submitting the next. Returns
    (makespan_s, results). The makespan ends when every job is done, its result
    (KRAK proof or root) serialised in host memory inside the engine; copying the
    results out to Python objects comes after."""
    t0 = engine.now()
    res = []
    if sequential:
        for j in jobs:
            res.append(engine.wait(engine.submit(j)))
        return engine.now() - t0, res
    tickets = engine.submit_many(jobs)
    engine.drain()
    t = engine.now() - t0
    return t, [engine.wait(x) for x in tickets]


def run_plain(jobs):
    """The plain single-job GPU path: each job through the drop-in entry points
    (vs_prove_fib / vs_commit_columns), one after another. Returns (seconds, results)."""
    import torch

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = []
    for j in jobs:
        if j.kind == FIB:
            res.append(prove_fib(j.a, j.b, j.log_n))
        else:
            res.append(commit_seeded(j.log_n, j.n_cols, j.seed))
    torch.cuda.synchronize()
    return time.perf_counter() - t0, res


def percentile(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    k = (len(xs) - 1) * q
    lo, hi = math.floor(k), math.ceil(k)
    return xs[lo] + (xs[hi] - xs[lo]) * (k - lo)


def run_served(engine: Engine, arrivals):
    """Submits each job at its arrival time from a submitter thread; returns per-job records."""
    tickets = [None] * len(arrivals)
    start = time.perf_counter()

    def submitter():
        for i, (t, job, _) in enumerate(arrivals):
            delay = start + t - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            tickets[i] = engine.submit(job)

    th = threading.Thread(target=submitter)
    th.start()
    records = []
    for i, (_, job, cls) in enumerate(arrivals):
        while tickets[i] is None:
            time.sleep(0.0002)
        out, ts, tb, te = engine.wait(tickets[i])
        records.append({"class": cls, "kind": job.kind, "t_submit": ts, "t_start": tb, "t_end": te,
                        "latency_ms": (te - ts) * 1e3, "bytes": out})
    th.join()
    return records


def summarize_served(records):
    by, wait, run = {}, {}, {}
    for r in records:
        by.setdefault(r["class"], []).append(r["latency_ms"])
        wait.setdefault(r["class"], []).append((r["t_start"] - r["t_submit"]) * 1e3)
        run.setdefault(r["class"], []).append((r["t_end"] - r["t_start"]) * 1e3)
    span = max(r["t_end"] for r in records) - min(r["t_submit"] for r in records)
    n_fib = sum(1 for r in records if r["kind"] == FIB)
    return {"jobs": len(records), "seconds": span, "jobs_per_s": len(records) / span, "proofs_per_s": n_fib / span,
            "p50_ms": percentile([r["latency_ms"] for r in records], 0.5),
            "p99_ms": percentile([r["latency_ms"] for r in records], 0.99),
            "per_class": {c: {"n": len(v), "p50_ms": percentile(v, 0.5), "p99_ms": percentile(v, 0.99),
                              "mean_ms": statistics.mean(v),
                              "queue_p50_ms": percentile(wait[c], 0.5), "queue_p99_ms": percentile(wait[c], 0.99),
                              "run_p50_ms": percentile(run[c], 0.5), "run_p99_ms": percentile(run[c], 0.99)}
                          for c, v in sorted(by.items())}}
