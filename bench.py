#!/usr/bin/env python3
"""Commitment-layer benchmark on B200: committed M31 elements/s.

Workload (one step): 34 columns x 2^24 rows of seeded uniform M31 values, treated
as bit-reversed canonic evaluations, go through circle interpolation, x4
low-degree extension (CanonicCoset(26), bit-reversed output) and a row-packed
Blake2s-256 Merkle root; then one seeded uniform QM31 vector of 2^26 values is
folded by FRI (circle fold, then line folds down to 8 values) with seeded fold
challenges, committing every folded layer.

Committed elements per step = 34 * 2^26 (trace LDE leaves) + 4 * (2^26 - 8)
(the FRI layers' SoA4 leaves).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl vstark|reference]

N > 1 runs one independent replica per GPU (weak scaling, no collective on the
data path); rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
# The slot engine keeps up to 24 streams busy at once (8 slots x 3 priorities).
# With the default 8 hardware queues, streams share queues and a small job can
# wait behind a large job's kernels; 32 gives every stream its own queue. Read by
# CUDA at context creation, so it is set before torch touches the GPU.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

SEED = 0x56530001
P = 0x7FFFFFFF
METRIC = "committed M31 elems/s & proofs/s batched vs plain on 1 B200; p50/p99 latency"
UNIT = "committed M31 elements/s"


def hbm_peak() -> tuple[float, str]:
    """HBM copy bandwidth the roofline fractions divide by (GB/s) and where it came
    from: the pool's measured copy bandwidth when that file is present, else an
    earlier copy measurement on the same B200s (6.65 TB/s)."""
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        v = json.loads(f.read_text()).get("hbm_gbs")
        if v:
            return float(v), "MEASURED_PEAKS.json hbm_gbs (measured)"
    return 6650.0, "fallback: 6650 GB/s, an earlier copy measurement on this B200 type"


def splitmix_m31(seed: int, offset: int, n: int) -> list[int]:
    """Same stream as vs_fill_uniform_m31 (host side, for the few fold challenges)."""
    P, M = 0x7FFFFFFF, (1 << 64) - 1

    def at(c):
        z = (seed + 0x9E3779B97F4A7C15 * c) & M
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        return z ^ (z >> 31)

    out = []
    for k in range(offset, offset + n):
        v = at(k + 1) >> 33
        if v == P:
            v = at(k + 2) >> 33
            v = 0 if v == P else v
        out.append(v)
    return out


def workload(args):
    n_cols, log_n, blow, fri_log = args.cols, args.log_n, 2, args.fri_log
    N = 1 << (log_n + blow)
    committed = n_cols * N + 4 * ((1 << (fri_log - 1)) * 2 - 8)
    return n_cols, log_n, blow, fri_log, N, committed


def config_json(args):
    n_cols, log_n, blow, fri_log, N, _ = workload(args)
    cols_gb, lde_gb, fri_gb = n_cols * 4 * (1 << log_n) / 1e9, n_cols * 4 * N / 1e9, 16 * (1 << fri_log) / 1e9
    l2_gb = 0.126
    big = cols_gb > l2_gb and fri_gb > l2_gb
    return {"workload": f"commitment layer: {n_cols} cols x 2^{log_n} rows, stwo LDE x{1 << blow} + row-packed "
                        f"Blake2s root, then FRI fold+commit of 2^{fri_log} QM31",
            "n_cols": n_cols, "log_n": log_n, "blowup": 1 << blow, "fri_log_n": fri_log,
            "l2": (f"inputs larger than L2 ({cols_gb:.2f} GB columns, {lde_gb:.2f} GB LDE, {fri_gb:.2f} GB QM31 "
                   f"vector; no flush between steps)" if big else
                   f"inputs not all larger than the 126 MB L2 ({cols_gb:.3f} GB columns, {fri_gb:.3f} GB QM31 vector)"),
            "seed": hex(SEED)}


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index, self.lines, self.proc = index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- CPU (oracle) baseline
def cpu_sample(args, threads: int):
    """The oracle's CPU pipeline on a bounded sample of the same workload."""
    import numpy as np
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_lib as O
    n_cols, _, blow, _, _, _ = workload(args)
    s_log, f_log = args.cpu_log_n, args.cpu_log_n + blow
    cols = O.seeded_m31(SEED, n_cols << s_log).reshape(n_cols, -1)
    root = np.zeros(8, np.uint32)
    t_commit = O.lib().oracle_bench_commit(O.ptr(cols), n_cols, s_log, blow, threads, O.ptr(root))
    src = O.seeded_m31(SEED + 1, 4 << f_log).reshape(4, -1)
    alphas = np.array(splitmix_m31(SEED + 2, 0, 4 * (f_log - 3)), np.uint32)
    roots = np.zeros((f_log - 3, 8), np.uint32)
    last = np.zeros((8, 4), np.uint32)
    t_fri = O.lib().oracle_bench_fri(O.ptr_array(list(src)), f_log, O.ptr(alphas), threads, O.ptr(roots), O.ptr(last))
    elems = n_cols * (1 << f_log) + 4 * ((1 << f_log) - 8)
    secs = t_commit + t_fri
    return {"value": elems / secs, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n_cols} cols x 2^{s_log} rows (LDE 2^{f_log}) + FRI of 2^{f_log} QM31, "
                      f"{secs:.2f} s on {threads} threads"}


def cpu_proofs(threads: int, n_proofs: int = 4, log_n: int = 16):
    """Config 0 on the host: full Fibonacci prove + verify at log_n = 16 (a0 = 1, a1
    seeded), the oracle's prover on `threads` threads (the reference's equivalent
    is prove_lean, timed by src/bin/full_benchmark.rs:30-59)."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_lib as O
    from vortexstark_b200.workloads import SplitMix64
    g = SplitMix64(0x56530000)
    jobs = [(1, g.m31()) for _ in range(n_proofs)]
    O.prove(1, 1, log_n, threads=threads)  # warm-up
    t0 = time.perf_counter()
    ok = True
    for a, b in jobs:
        rc, _ = O.verify(O.prove(a, b, log_n, threads=threads))
        ok = ok and rc == 0
    secs = time.perf_counter() - t0
    return {"value": n_proofs / secs, "unit": "proofs/s (prove + verify)", "cores": threads, "kind": "port",
            "verified": ok, "sample": f"{n_proofs} Fibonacci proofs, log_n={log_n}, a0=1, a1 seeded; "
                                      f"{secs:.2f} s on {threads} threads"}


def run_reference(args):
    """The CPU implementation of the path (the oracle port: the reference has no CPU
    path for it) on the host cores, one bounded sample of the workload per step:
    34 columns x 2^cpu_log_n rows, x4 LDE + row-packed root, and FRI of 2^(cpu_log_n+2).
    ms_per_step is the sample's own measured time."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if not (ROOT / "tests" / "oracle_lib.py").exists():
        print(json.dumps({"impl": "reference", "unavailable": "CPU oracle sources missing"}))
        return
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_sample(args, threads)
    vals, secs = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        vals.append(cpu_sample(args, threads))
        secs.append(time.perf_counter() - t0)
    v = statistics.mean(x["value"] for x in vals)
    n_cols, _, blow, _, _, committed = workload(args)
    s_log = args.cpu_log_n
    sample_elems = n_cols * (1 << (s_log + blow)) + 4 * ((1 << (s_log + blow)) - 8)
    cfg = dict(config_json(args), sample=f"{n_cols} cols x 2^{s_log} rows (LDE 2^{s_log + blow}) + FRI of "
                                         f"2^{s_log + blow} QM31 per step ({sample_elems} committed elements)",
               sample_log_n=s_log)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.mean(secs) * 1e3,
            "ms_per_step_full_config_derived": committed / v * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32 (M31)",
            "data": "synthetic (seeded SplitMix64 uniform M31)", "config": cfg,
            "cpu_baseline": dict(vals[-1], value=v),
            "cpu_proofs": cpu_proofs(threads),
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- OODS / DEEP quotient kernels
def oods_quotients(args, V, torch, lde, N, st, ev):
    """The reference's OODS quotient kernels over the step's LDE: numerators of all
    columns against one sample (cuda_accumulate_numerators), then the combine of two
    samples over the evaluation domain (cuda_compute_quotients_combine), as its Cairo
    prover runs them (cairo_air/prover.rs:2191-2266). Seeded coefficients and
    domain coordinates; CUDA-event time on the default stream."""
    L = V.lib()
    n_cols = lde.shape[0]
    log_eval = N.bit_length() - 1
    dev = lambda words: torch.empty(words, dtype=torch.int32, device="cuda")  # noqa: E731

    def seeded(words, seed):
        t = dev(words)
        V.check(L.vs_fill_uniform_m31(t.data_ptr(), words, seed, 0, None))
        return t

    col_ptrs = torch.tensor([lde[c].data_ptr() for c in range(n_cols)], dtype=torch.int64, device="cuda")
    idx = torch.arange(n_cols, dtype=torch.int32, device="cuda")
    b, c = seeded(4 * n_cols, SEED + 5), seeded(4 * n_cols, SEED + 6)
    numer = [dev(N) for _ in range(4)]
    out = [dev(N) for _ in range(4)]
    dxs, dys = seeded(N, SEED + 10), seeded(N, SEED + 11)  # stand-in domain coordinates (cost is value-independent)
    spx, spy, fla = seeded(8, SEED + 7), seeded(8, SEED + 8), seeded(8, SEED + 9)
    nptr = [torch.tensor([numer[k].data_ptr()] * 2, dtype=torch.int64, device="cuda") for k in range(4)]
    logs = torch.tensor([log_eval, log_eval], dtype=torch.int32, device="cuda")

    def acc():
        L.cuda_accumulate_numerators(col_ptrs.data_ptr(), idx.data_ptr(), b.data_ptr(), c.data_ptr(), n_cols, N,
                                     *[o.data_ptr() for o in numer])

    def comb():
        L.cuda_compute_quotients_combine(spx.data_ptr(), spy.data_ptr(), fla.data_ptr(), *[x.data_ptr() for x in nptr],
                                         logs.data_ptr(), 2, dxs.data_ptr(), dys.data_ptr(), log_eval, N,
                                         *[o.data_ptr() for o in out])

    res = {}
    hbm, hbm_src = hbm_peak()
    for name, fn, alg in (("accumulate_numerators", acc, 4 * n_cols * N + 16 * N),
                          ("quotients_combine", comb, 2 * 16 * N + 8 * N + 16 * N)):
        fn()
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        s0 = torch.cuda.default_stream()
        e0.record(s0)
        for _ in range(args.steps):
            fn()
        e1.record(s0)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        res[name] = {"ms": ms, "algorithmic_bytes": alg, "achieved_gbs": alg / (ms / 1e3) / 1e9,
                     "hbm_frac": alg / (ms / 1e3) / 1e9 / hbm}
    res["workload"] = f"{n_cols} LDE columns x 2^{log_eval} rows; combine of 2 samples"
    return res


def fold_dropins(args, V, torch, fri_src, ev):
    """The reference's plain FRI fold kernels (no commitment) on the step's QM31
    vector: cuda_fold_circle_into_line_soa of 2^k values into an accumulated line of
    2^(k-1) (fri.cu:44-78), then cuda_fold_line_soa of that line (fri.cu:10-39).
    Algorithmic bytes: circle 16N read + 2N twiddles + 8N accumulator read + 8N
    written; line fold of m values 16m + 2m + 8m. CUDA-event time, default stream."""
    L = V.lib()
    N = fri_src.shape[1]
    half = N // 2
    dev = lambda words: torch.empty(words, dtype=torch.int32, device="cuda")  # noqa: E731

    def seeded(words, seed):
        t = dev(words)
        V.check(L.vs_fill_uniform_m31(t.data_ptr(), words, seed, 0, None))
        return t

    tw_c, tw_l = seeded(half, SEED + 20), seeded(half // 2, SEED + 21)  # stand-in twiddles (value-independent cost)
    line = [seeded(half, SEED + 22 + k) for k in range(4)]
    out = [dev(half // 2) for _ in range(4)]
    alpha = (C.c_uint32 * 4)(1, 2, 3, 4)
    alpha_sq = (C.c_uint32 * 4)(5, 6, 7, 8)
    src = [fri_src[k].data_ptr() for k in range(4)]

    def circle():
        L.cuda_fold_circle_into_line_soa(*[x.data_ptr() for x in line], *src, tw_c.data_ptr(), alpha, alpha_sq, half)

    def fold_line():
        L.cuda_fold_line_soa(*[x.data_ptr() for x in line], tw_l.data_ptr(), *[o.data_ptr() for o in out], alpha,
                             half // 2)

    hbm, hbm_src = hbm_peak()
    res = {}
    for name, fn, alg in (("fold_circle_into_line", circle, 34 * N), ("fold_line", fold_line, 26 * half)):
        fn()
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        s0 = torch.cuda.default_stream()
        e0.record(s0)
        for _ in range(args.steps):
            fn()
        e1.record(s0)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        res[name] = {"ms": ms, "algorithmic_bytes": alg, "achieved_gbs": alg / (ms / 1e3) / 1e9,
                     "hbm_frac": alg / (ms / 1e3) / 1e9 / hbm}
    res["workload"] = f"circle fold 2^{N.bit_length() - 1} -> 2^{half.bit_length() - 1}, line fold of 2^{half.bit_length() - 1}"
    return res


# ---------------------------------------------------------------- Cairo trace chain
def cairo_chain(args, V, torch, ev):
    """The reference Cairo prover's commitment chain at production width, on the
    device: 34 trace columns (half-coset order) committed as groups 16 / 15 / 3
    with coefficients, blinding, half-coset copies and tile roots
    (cairo_air/prover.rs:899-1047), then the tail from the AIR-quotient commitment
    through OODS, the DEEP quotient and FRI (prover.rs:1937-2438) with 12
    interaction columns. Seeded inputs; the AIR quotient is a seeded polynomial of
    degree < 2n (the constraint evaluation itself is Cairo-specific and not on this
    path). CUDA-event time on the current stream."""
    from vortexstark_b200 import api
    log_n = args.cairo_log_n
    n, N = 1 << log_n, 4 << log_n
    dev = torch.device("cuda")
    mk = lambda *s: torch.empty(s, dtype=torch.int32, device=dev)  # noqa: E731
    cols = api.fill_uniform_m31(mk(34, n), SEED + 20)
    blind = [(SEED * 7919 + 104729 * c) % P for c in range(34)]
    coeffs, evals, evals_hc = mk(34, n), mk(34, N), mk(34, N)
    tiles = [mk(max(1, N // 1024) * 8) for _ in range(3)]
    groups = ((0, 16), (16, 31), (31, 34))
    inter = api.lde_stwo(api.fill_uniform_m31(mk(12, n), SEED + 21), log_n, 2)
    q_cn = api.lde_stwo(api.fill_uniform_m31(mk(4, 2 * n), SEED + 22), log_n + 1, 1)
    k = torch.arange(N, dtype=torch.int64, device=dev)
    cn = torch.where(k % 2 == 0, k // 2, N - 1 - k // 2)
    pos = torch.zeros_like(cn)
    for b in range(log_n + 2):
        pos |= ((cn >> b) & 1) << (log_n + 1 - b)
    q_hc = q_cn[:, pos].contiguous()
    del k, cn, pos
    L = V.lib()
    st = torch.cuda.current_stream()

    def commit():
        roots = []
        for g, (a, b) in enumerate(groups):
            root = mk(8)
            V.check(L.vs_commit_group_cairo(cols[a].data_ptr(), n, b - a, log_n, (C.c_uint32 * (b - a))(*blind[a:b]),
                                            coeffs[a].data_ptr(), evals[a].data_ptr(), evals_hc[a].data_ptr(),
                                            root.data_ptr(), tiles[g].data_ptr(), st.cuda_stream),
                    "vs_commit_group_cairo")
            roots.append(root)
        return roots

    def tail(roots):
        ch = api.Channel()
        for r in roots:
            ch.mix_digest(r.cpu().numpy().view("uint32"))
        return api.cairo_oods_fri(ch, log_n, list(coeffs), list(evals), list(inter), list(q_hc), zk_scalars=blind)

    tail(commit())
    torch.cuda.synchronize()
    t_commit, t_tail = [], []
    low_degree = True
    iters = max(1, args.steps // 2)
    c0 = api.launch_count()
    for _ in range(iters):
        e0, e1, e2 = ev(), ev(), ev()
        e0.record(st)
        roots = commit()
        e1.record(st)
        r = tail(roots)
        e2.record(st)
        torch.cuda.synchronize()
        t_commit.append(e0.elapsed_time(e1))
        t_tail.append(e1.elapsed_time(e2))
        nat = [r["last_layer_coeffs"][i] for i in (0, 4, 2, 6, 1, 5, 3, 7)]
        low_degree = low_degree and not any(any(c) for c in nat[4:])
    res = {"workload": f"34 trace columns (16/15/3) x 2^{log_n} rows, x4 LDE; 12 interaction columns; "
                       "AIR quotient of degree < 2n", "log_n": log_n,
           "commit_ms": statistics.median(t_commit), "tail_ms": statistics.median(t_tail),
           "trace_elements_committed": 34 * N, "last_layer_low_degree": low_degree,
           "gpu_launches_per_chain": (api.launch_count() - c0) // iters}
    del cols, coeffs, evals, evals_hc, inter, q_cn, q_hc
    torch.cuda.empty_cache()
    return res


# ---------------------------------------------------------------- proof workloads
def proof_workloads(args):
    """Proof throughput and latency. The plain path is the drop-in single-job
    entry points (vs_prove_fib, vs_commit_columns) called one job at a time; the
    engine runs the same jobs over slots of graph-captured provers. Timing is host
    wall clock around completed jobs (results back in host memory)."""
    from vortexstark_b200 import api
    from vortexstark_b200 import workloads as W

    def prep(eng, jobs):
        for j in W.shapes(jobs):
            eng.prepare(api.commit_job(j.log_n, 34, 0) if j.kind == api.COMMIT else j)

    # Start from an empty stream-ordered pool: the step, e2e and Cairo runs above
    # leave GBs of differently sized blocks cached in it (release threshold = all),
    # which slowed the plain path's per-call allocations twofold. A threshold of 0
    # releases them at the next synchronisation; then the pool keeps everything again.
    import torch
    api.init_memory_pool(0)
    torch.cuda.synchronize()
    api.init_memory_pool((1 << 64) - 1)

    out = {}
    plain = W.plain_jobs(64, 16)
    W.run_plain(plain[:4])
    t_plain, r_plain = W.run_plain(plain)
    lat = []
    for j in plain[:32]:
        t0 = time.perf_counter()
        api.prove_fib(j.a, j.b, j.log_n)
        lat.append((time.perf_counter() - t0) * 1e3)
    ok, _ = api.verify_fib(r_plain[0])
    out["plain"] = {"workload": "64 Fibonacci proofs, log_n=16, a0=1, a1 seeded; vs_prove_fib one at a time",
                    "proofs_per_s": len(plain) / t_plain, "p50_ms": W.percentile(lat, 0.5),
                    "p99_ms": W.percentile(lat, 0.99), "verified": ok}
    # Batches are throughput work: every job at the same stream priority (the
    # size-priority default is the serving policy, measured below). The engine
    # proves queued Fibonacci jobs of one size as one batch (one graph launch, one
    # kernel per stage for all of them); batch_limit 1 is one proof per launch.
    def batched(jobs, limit, warm):
        """Median of three timed runs of the job list, after an untimed warm-up run that
        creates the workspaces the runs use. The 120 GB budget bounds the cached
        workspaces of 16 slots (the engine frees idle ones of other shapes as needed)."""
        with api.Engine(args.batch_slots, 120 * 10**9, size_priority=False) as eng:
            eng.set_batch_limit(limit)
            W.run_list(eng, jobs[:warm], sequential=False)
            runs = [W.run_list(eng, jobs, sequential=False) for _ in range(3)]
        runs.sort(key=lambda x: x[0])
        return runs[1]

    t_e, r_e = batched(plain, 0, len(plain))
    t_1, r_1 = batched(plain, 1, len(plain))
    out["batched_fib16"] = {"workload": "the same 64 proofs submitted at once to the slot engine (median of 3 runs)",
                            "slots": args.batch_slots, "proofs_per_s": len(plain) / t_e,
                            "vs_plain": t_plain / t_e,
                            "one_proof_per_launch_proofs_per_s": len(plain) / t_1,
                            "identical_to_plain": all(x[0] == y for x, y in zip(r_e, r_plain)) and
                            all(x[0] == y for x, y in zip(r_1, r_plain))}

    jobs = W.batched_jobs(64)
    W.run_plain(W.shapes(jobs))
    # median of three runs, as for the engine arms (single runs of the plain path
    # varied between 130 and 218 jobs/s with the allocator pool's state)
    plain_runs = sorted((W.run_plain(jobs) for _ in range(3)), key=lambda x: x[0])
    t_p, r_p = plain_runs[1]
    with api.Engine(1, size_priority=False) as one:
        one.set_batch_limit(1)
        prep(one, jobs)
        t_one, r_one = W.run_list(one, jobs, sequential=True)
    t_b, r_b = batched(jobs, 0, len(jobs))
    t_b1, r_b1 = batched(jobs, 1, len(jobs))
    n_fib = sum(1 for j in jobs if j.kind == api.FIB)
    out["batched_mix"] = {
        "workload": "64 jobs, log_n U{16..22}: Fibonacci proofs (a1 seeded) or 1-34 seeded uniform columns (commit); "
                    "median of 3 runs",
        "slots": args.batch_slots, "jobs_per_s": len(jobs) / t_b, "proofs_per_s": n_fib / t_b,
        "plain_path_jobs_per_s": len(jobs) / t_p, "engine_one_slot_jobs_per_s": len(jobs) / t_one,
        "one_proof_per_launch_jobs_per_s": len(jobs) / t_b1,
        "vs_plain": t_p / t_b, "vs_one_slot": t_one / t_b,
        "identical_plain_one_slot_batched": all(a == b[0] == c[0] == d[0] for a, b, c, d in zip(r_p, r_one, r_b, r_b1)),
        "parity": mix_parity(jobs, r_p)}

    # Single-proof latency at the sizes the reference publishes (prove_lean(1, 1, log_n)
    # after a warm-up proof): the drop-in path and the graph-captured prover.
    lat = {}
    for L in args.prove_sizes:
        api.prove_fib(1, 1, L)
        t0 = time.perf_counter()
        proof = api.prove_fib(1, 1, L)
        t_plain = time.perf_counter() - t0
        with api.Engine(1) as eng:
            j = api.fib_job(L, 1, 1)
            eng.prepare(j)
            eng.wait(eng.submit(j))
            t0 = time.perf_counter()
            same = eng.wait(eng.submit(j))[0] == proof
            t_graph = time.perf_counter() - t0
        lat[str(L)] = {"vs_prove_fib_ms": t_plain * 1e3, "graph_prover_ms": t_graph * 1e3,
                       "proof_bytes": len(proof), "identical": same, "verified": api.verify_fib(proof)[0]}
    out["single_proof_latency"] = lat

    arrivals = W.served_arrivals(args.served_jobs)
    for key, by_size in (("served", True), ("served_fifo_priority", False)):
        with api.Engine(args.slots, 150 * 10**9, size_priority=by_size) as eng:
            prep(eng, [a[1] for a in arrivals])
            recs = W.run_served(eng, arrivals)
        out[key] = dict(W.summarize_served(recs), workload="Poisson 200 jobs/s: Fibonacci 16/20/24 (0.5/0.3/0.2) "
                        "and 34-col commits 18/20/22", slots=args.slots, hbm_budget_gb=150,
                        stream_priority="by job size, smallest first" if by_size else "equal for all jobs")
    return out


# ---------------------------------------------------------------- parity of the timed step
def step_parity(args, rank, world, root, roots, last):
    """The last timed step's row-packed root, FRI layer roots and last layer against
    the oracle's results for the same seeded inputs (tests/golden/bench_digests.json,
    written by tests/golden/gen_bench_digests.py). A mismatch stops the run: no
    number is reported for wrong results."""
    import numpy as np
    path = ROOT / "tests" / "golden" / "bench_digests.json"
    d = json.loads(path.read_text()).get("step") if path.exists() else None
    same_cfg = d is not None and (d["n_cols"], d["log_n"], d["fri_log_n"]) == (args.cols, args.log_n, args.fri_log)
    if not same_cfg or rank != 0:
        return {"status": "unchecked", "why": "no oracle digest for this configuration" if not same_cfg
                else "checked on rank 0 only"}
    hexw = lambda t: t.cpu().numpy().view(np.uint32).tobytes().hex()  # noqa: E731
    got_roots = [hexw(roots[8 * i:8 * i + 8]) for i in range(args.fri_log - 3)]
    ok = hexw(root) == d["root"] and got_roots == d["fri_roots"] and hexw(last) == d["last_layer"]
    if not ok:
        raise SystemExit(f"bench: the timed step's results differ from the oracle digests in {path.name}")
    return {"status": "digest-match", "checked": f"row-packed root, {args.fri_log - 3} FRI layer roots, last layer",
            "oracle": "tests/golden/bench_digests.json"}


def mix_parity(jobs, results):
    """Results of the 64-job mix against the oracle's (bench_digests.json)."""
    import hashlib
    path = ROOT / "tests" / "golden" / "bench_digests.json"
    exp = json.loads(path.read_text()).get("batched_mix", {}).get("results") if path.exists() else None
    if not exp or len(exp) != len(jobs):
        return "unchecked"
    for e, r in zip(exp, results):
        good = (len(r) == e["len"] and hashlib.sha256(r).hexdigest() == e["sha256"]) if e["kind"] == "fib" \
            else r.hex() == e["root"]
        if not good:
            return "MISMATCH"
    return "digest-match"


def profile_batch(log_n: int) -> None:
    """One batch of 64 Fibonacci proofs on one slot (batch limit 64) inside a profiler
    range, after preparing the workspace and one warm batch; checks the first proof
    against the plain path."""
    import torch

    from vortexstark_b200 import api
    from vortexstark_b200 import workloads as W
    jobs = W.plain_jobs(64, log_n)
    with api.Engine(1, size_priority=False) as eng:
        eng.set_batch_limit(64)
        eng.prepare(jobs[0])
        W.run_list(eng, jobs, sequential=False)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        t, r = W.run_list(eng, jobs, sequential=False)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
    if r[0][0] != api.prove_fib(jobs[0].a, jobs[0].b, log_n):
        raise SystemExit("profile batch: proof differs from the plain path")
    print(json.dumps({"profile_batch": {"log_n": log_n, "proofs": len(jobs), "ms": t * 1e3}}))


# ---------------------------------------------------------------- GPU arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="vstark", choices=["vstark", "reference"])
    ap.add_argument("--cols", type=int, default=34)
    ap.add_argument("--log-n", type=int, default=24)
    ap.add_argument("--fri-log", type=int, default=26)
    ap.add_argument("--cpu-log-n", type=int, default=None,
                    help="row log of the CPU sample (default 22 for the cpu_baseline, 20 per reference-arm step)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-proofs", action="store_true", help="skip the plain / batched / served proof runs")
    ap.add_argument("--no-oods", action="store_true", help="skip the OODS quotient kernels")
    ap.add_argument("--no-cairo", action="store_true", help="skip the Cairo trace commitment + tail chain")
    ap.add_argument("--cairo-log-n", type=int, default=22, help="trace rows (log) of the Cairo chain")
    ap.add_argument("--slots", type=int, default=8, help="concurrent slots of the served engines")
    ap.add_argument("--batch-slots", type=int, default=16,
                    help="concurrent slots of the batched (throughput) engines: more batches in flight let "
                         "one batch's host serialisation overlap another's kernels")
    ap.add_argument("--served-jobs", type=int, default=600)
    ap.add_argument("--no-autotune", action="store_true", help="keep the default NTT plans (no autotuning)")
    ap.add_argument("--merkle-split", type=int, default=None,
                    help="Merkle subtree split to use instead of tuning it (for profiler runs with --no-autotune)")
    ap.add_argument("--tune-sizes", type=int, nargs="*", default=list(range(16, 25)),
                    help="trace sizes (log) the NTT autotuner tunes before the timed runs")
    ap.add_argument("--prove-sizes", type=int, nargs="*", default=[20, 24, 28],
                    help="log_n of the single-proof latency runs")
    ap.add_argument("--profile-batch", type=int, default=None, metavar="LOG_N",
                    help="profiler run only: one warm batch of 64 Fibonacci proofs of 2^LOG_N rows, then one batch "
                         "inside cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    args = ap.parse_args()
    if args.profile_batch is not None:
        return profile_batch(args.profile_batch)
    args.warmup = max(args.warmup, 3)
    if args.cpu_log_n is None:
        args.cpu_log_n = 20 if args.impl == "reference" else 22
    if args.impl == "reference":
        return run_reference(args)

    import torch

    import vortexstark_b200 as V
    from vortexstark_b200 import api, replicas

    rank, world, local = replicas.env()
    torch.cuda.set_device(local)
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    replicas.init("nccl", timeout_s=120)
    V.lib()  # raises if the CUDA library is missing
    # The stream-ordered pool keeps what it has allocated, as the reference's own
    # benchmark sets it (init_memory_pool_greedy, src/bin/full_benchmark.rs:23).
    api.init_memory_pool((1 << 64) - 1)

    # NTT launch shapes per size chosen by the autotuner before anything is timed
    # (34-column stwo LDEs); every later transform of a tuned size uses its plan.
    tuning = None
    if args.merkle_split is not None:
        api.set_merkle_split(args.merkle_split)
    if not args.no_autotune:
        tuning = {}
        for tl in sorted(set(args.tune_sizes) | {args.log_n}):
            lo, items, radix = api.ntt_plan(tl)
            # the default's items (0) as the candidate it equals: one tile per CTA in
            # 13-layer lower passes, 8 tiles per CTA otherwise
            default = (lo, items or (1 if lo == 13 else 8), radix)
            r = api.autotune_lde(tl, n_cols=args.cols, blowup=2, reps=3)
            times = dict(r["candidates"])
            tuning[str(tl)] = {"plan": list(r["best"]), "ms": times[tuple(r["best"])],
                               "default_plan": list(default), "default_ms": times.get(tuple(default)),
                               "candidates": len(times)}
        # Merkle subtree split of the root-only trees, tuned on the step's row-packed root
        if args.merkle_split is None:
            m = api.autotune_merkle(args.log_n + 2, n_cols=args.cols, reps=3)
            tuning["merkle_split"] = {"split": m["best"], "ms_by_split": [round(x, 3) for x in m["ms"]],
                                      "log_leaves": args.log_n + 2}

    n_cols, log_n, blow, fri_log, N, committed = workload(args)
    n = 1 << log_n
    st = torch.cuda.current_stream()
    cols = torch.empty((n_cols, n), dtype=torch.int32, device="cuda")
    api.fill_uniform_m31(cols, SEED, offset=replicas.input_offset(rank, n_cols << log_n))
    fri_src = torch.empty((4, 1 << fri_log), dtype=torch.int32, device="cuda")
    api.fill_uniform_m31(fri_src, SEED + 1, offset=replicas.input_offset(rank, 4 << fri_log))
    alphas = splitmix_m31(SEED + 2, 0, 4 * (fri_log - 3))
    alphas = [alphas[4 * i:4 * i + 4] for i in range(fri_log - 3)]
    lde = torch.empty((n_cols, N), dtype=torch.int32, device="cuda")
    root = torch.zeros(8, dtype=torch.int32, device="cuda")
    work = torch.empty(4 << fri_log, dtype=torch.int32, device="cuda")
    roots = torch.zeros(8 * (fri_log - 3), dtype=torch.int32, device="cuda")
    last = torch.zeros(32, dtype=torch.int32, device="cuda")

    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def step(marks=None, c=None, f=None):
        c = cols if c is None else c
        f = fri_src if f is None else f
        if marks is not None:
            marks[0].record(st)
        api.lde_stwo(c, log_n, blow, out=lde)
        if marks is not None:
            marks[1].record(st)
        api.merkle_root_rowpacked(lde, root)
        if marks is not None:
            marks[2].record(st)
        api.fri_fold_commit(f, fri_log, alphas, work, roots, last)
        if marks is not None:
            marks[3].record(st)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    replicas.barrier()
    torch.cuda.synchronize()
    marks = [[ev() for _ in range(4)] for _ in range(args.steps)]
    l0 = api.launch_count()
    vis = [v for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
    with ClockSampler(vis[local] if local < len(vis) else local) as clk:
        t0, t1 = ev(), ev()
        t0.record(st)
        for k in range(args.steps):
            step(marks[k])
        t1.record(st)
        torch.cuda.synchronize()
    launches = (api.launch_count() - l0) // args.steps
    ms = t0.elapsed_time(t1) / args.steps
    parity = step_parity(args, rank, world, root, roots, last)
    phase = {"lde": 0.0, "merkle": 0.0, "fri": 0.0}
    for m in marks:
        phase["lde"] += m[0].elapsed_time(m[1]) / args.steps
        phase["merkle"] += m[1].elapsed_time(m[2]) / args.steps
        phase["fri"] += m[2].elapsed_time(m[3]) / args.steps
    ms = replicas.max_over_ranks(ms, "cuda")
    replicas.barrier()
    value = committed * world / (ms / 1e3)

    # The reference-faithful three-tree form of the same commitment (its Cairo
    # prover commits 34 columns as trees of 16 / 15 / 3 columns with the native
    # leaf of at most 16 words), over the same LDE, beside the row-packed root.
    groups = [(a, min(a + 16, n_cols)) for a in range(0, n_cols, 16)] if n_cols != 34 else [(0, 16), (16, 31), (31, 34)]
    roots3 = torch.zeros((len(groups), 8), dtype=torch.int32, device="cuda")

    def three_tree():
        for i, (a, b) in enumerate(groups):
            api.merkle_root_capped(lde[a:b], roots3[i])

    three_tree()
    torch.cuda.synchronize()
    m0, m1 = ev(), ev()
    m0.record(st)
    for _ in range(args.steps):
        three_tree()
    m1.record(st)
    torch.cuda.synchronize()
    three = {"groups": "/".join(str(b - a) for a, b in groups), "ms": m0.elapsed_time(m1) / args.steps,
             "row_packed_root_ms": phase["merkle"]}

    # Does the row-packed root pay for reading the LDE back from HBM? The same
    # launch (34 columns x 2^19 rows, 71 MB) hashed back to back from one buffer,
    # which stays in the 126 MB L2, against rotating over four such buffers (285 MB,
    # so each launch reads its columns from HBM). Equal times mean the re-read is
    # hidden behind the hashing, so fusing the LDE with the leaf hash could not
    # shorten the step.
    rows = 1 << 19
    bufs = [lde[:, k * rows:(k + 1) * rows].contiguous() for k in range(4)]
    root_p = torch.zeros(8, dtype=torch.int32, device="cuda")

    def timed(pick, reps=40):
        for k in range(4):
            api.merkle_root_rowpacked(bufs[pick(k)], root_p)
        torch.cuda.synchronize()
        m0.record(st)
        for k in range(reps):
            api.merkle_root_rowpacked(bufs[pick(k)], root_p)
        m1.record(st)
        torch.cuda.synchronize()
        return m0.elapsed_time(m1) / reps

    warm_ms, cold_ms = timed(lambda k: 0), timed(lambda k: k % 4)
    fusion = {"workload": f"row-packed root of {n_cols} columns x 2^19 rows: one L2-resident buffer vs four "
                          "buffers in rotation (read from HBM)",
              "l2_resident_ms": warm_ms, "hbm_ms": cold_ms, "hbm_over_l2": cold_ms / warm_ms}
    del bufs

    oods = oods_quotients(args, V, torch, lde, N, st, ev) if rank == 0 and not args.no_oods else None
    folds = fold_dropins(args, V, torch, fri_src, ev) if rank == 0 and not args.no_oods else None

    # End to end through the C ABI from pinned host buffers: every step copies its
    # inputs host -> device and reads its roots back. Inputs are double-buffered on
    # the device and copied on a second stream, so step k+1's upload overlaps step
    # k's compute (a step's upload waits until the step two back has released its
    # buffer). The timed region runs from before the first upload to after the
    # last read-back.
    e2e = None
    if not args.no_e2e:
        cols_h = torch.empty_like(cols, device="cpu").pin_memory()
        fri_h = torch.empty_like(fri_src, device="cpu").pin_memory()
        cols_h.copy_(cols)
        fri_h.copy_(fri_src)
        out_h = torch.empty(8 + 8 * (fri_log - 3) + 32, dtype=torch.int32).pin_memory()
        bufs = [(cols, fri_src), (torch.empty_like(cols), torch.empty_like(fri_src))]
        cs = torch.cuda.Stream()
        free = [torch.cuda.Event(), torch.cuda.Event()]
        for e in free:
            e.record(st)

        def e2e_run(k_steps):
            for k in range(k_steps):
                c, f = bufs[k & 1]
                ready = torch.cuda.Event()
                with torch.cuda.stream(cs):
                    cs.wait_event(free[k & 1])
                    c.copy_(cols_h, non_blocking=True)
                    f.copy_(fri_h, non_blocking=True)
                    ready.record(cs)
                st.wait_event(ready)
                step(c=c, f=f)
                out_h[:8].copy_(root, non_blocking=True)
                out_h[8:8 + roots.numel()].copy_(roots, non_blocking=True)
                out_h[8 + roots.numel():].copy_(last, non_blocking=True)
                free[k & 1].record(st)

        e2e_run(2)
        torch.cuda.synchronize()
        replicas.barrier()
        e0, e1 = ev(), ev()
        e0.record(st)
        cs.wait_event(e0)
        e2e_run(args.steps)
        e1.record(st)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1) / args.steps
        ems = replicas.max_over_ranks(ems, "cuda")
        e2e = {"value": committed * world / (ems / 1e3), "unit": UNIT, "ms_per_step": ems,
               "h2d_bytes_per_step": (cols.numel() + fri_src.numel()) * 4, "d2h_bytes_per_step": out_h.numel() * 4,
               "pipelining": "inputs double-buffered on the device; upload of step k+1 overlaps compute of step k"}
        del bufs

    # Roofline of the dominant kernel: merkle_subtree_kernel<LeafRowPacked> (the
    # largest single kernel of the step in the ncu launch list), timed by the events
    # around the row-packed root (which also cover the upper reduction of its 2^split
    # roots per tile). Algorithmic bytes: 4 * n_cols per leaf, each LDE word read
    # once. Traffic: the ncu capture of the same kernel (34 columns, 2^22 leaves,
    # split 8) read 570.6 MB = 1.0004 x algorithmic and wrote its subtree roots
    # (2^split hashes of 32 B per 1024-leaf tile, 33.6 MB); the same per-leaf
    # read ratio plus the roots at this run's split. Per-phase HBM fractions are listed beside it;
    # all phases are integer-ALU bound (Blake2s, M31 butterflies), not HBM bound.
    hbm, hbm_src = hbm_peak()
    clk_hz = (clk.summary()["sm_mhz"] or 1965.0) * 1e6
    alg = {"lde": n_cols * (4 * n + 4 * N), "merkle": n_cols * 4 * N,
           "fri": sum(24 * (1 << (l - 1)) for l in range(4, fri_log + 1))}
    ach = alg["merkle"] / (phase["merkle"] / 1e3) / 1e9
    roof = {"bound": "hbm", "kernel": "merkle_subtree_kernel<LeafRowPacked>", "achieved": ach, "peak": hbm,
            "peak_source": hbm_src, "unit": "GB/s", "frac": ach / hbm,
            "traffic": alg["merkle"] * 1.0004 + (N >> 10 << api.merkle_split()) * 32,
            "algorithmic_bytes": alg["merkle"],
            # The binding resource is integer issue: instructions per launch (1179
            # per Blake2s compression on average, the ncu count of this kernel at
            # split 8: 579.4 M warp instructions for 2^22 leaves x 3.75 compressions;
            # one compression per 64 B of leaf plus one per node) over 148 SMs x 4
            # schedulers x 32 lanes x the sampled SM clock.
            "int_issue_frac": (-(-n_cols * 4 // 64) + 1) * 1179 * N / (phase["merkle"] / 1e3)
                              / (148 * 4 * 32 * clk_hz),
            "int_issue_basis": "derived: 1179 instructions per compression from one ncu count "
                               "(profiles/merkle_rowpacked_fold_log22.md), not measured in this run",
            "launch_ms": phase["merkle"], "phase_ms": phase,
            "phase_hbm_frac": {k: alg[k] / (phase[k] / 1e3) / 1e9 / hbm for k in phase}}

    proofs = cairo = None
    if rank == 0 and world == 1 and not (args.no_proofs and args.no_cairo):
        del lde, cols, fri_src, work
        torch.cuda.empty_cache()
        if not args.no_cairo:
            cairo = cairo_chain(args, V, torch, ev)
        if not args.no_proofs:
            proofs = proof_workloads(args)
    if rank == 0:
        cpu = None
        if not args.no_cpu:
            cpu = cpu_sample(args, os.cpu_count() or 1)
            cpu["proofs"] = cpu_proofs(os.cpu_count() or 1)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "u32 (M31)", "data": "synthetic (seeded SplitMix64 uniform M31)",
                "config": config_json(args), "parity": parity, "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": launches, "clocks": clk.summary(), "three_tree_commit": three, "lde_leaf_fusion_probe": fusion, "oods": oods, "fri_fold_dropins": folds, "ntt_autotune": tuning,
                "cairo": cairo, "proofs": proofs}
        print(json.dumps(line), flush=True)
    replicas.finalize()


if __name__ == "__main__":
    main()
