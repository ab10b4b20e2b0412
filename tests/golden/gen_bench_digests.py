"""Writes bench_digests.json: the oracle's results for the benchmark workloads at
their own sizes, so GPU tests and bench.py can check the timed work bit for bit
without minutes of CPU work at run time.

* "step": the commitment-layer step of bench.py (34 columns x 2^24 rows of seeded
  uniform M31, x4 stwo LDE, row-packed Blake2s root; FRI fold+commit of a seeded
  2^26 QM31 vector with seeded challenges): the root, the 23 FRI layer roots and
  the 8-value last layer.
* "batched_mix": every job of the 64-job mix (log_n 16..22, Fibonacci proofs and
  1..34-column commitments; vortexstark_b200.workloads.batched_jobs): the
  commitment root, or the SHA-256 and length of the KRAK proof.
* "served": the first job of each size class of the served arrival stream
  (workloads.served_arrivals): Fibonacci 16/20/24 and 34-column commits 18/20/22.

    python tests/golden/gen_bench_digests.py [step] [mix] [served]

Runs the oracle on every host core: about 10 minutes and 12 GB of host memory on 8
cores. The oracle is pinned to the reference's own kernels at small sizes
(ref_golden.npz)."""
import hashlib
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE.parent.parent))
import oracle_lib as O  # noqa: E402
import bench  # noqa: E402
from vortexstark_b200 import workloads as W  # noqa: E402

OUT = HERE / "bench_digests.json"
THREADS = os.cpu_count() or 1


def hexw(words) -> str:
    return np.asarray(words, np.uint32).tobytes().hex()


def commit_root(log_n: int, n_cols: int, seed: int, blowup: int = 2) -> str:
    """Root of n_cols seeded columns (one SplitMix64 stream, column-major), x4 stwo LDE, row-packed leaves."""
    cols = O.seeded_m31(seed, n_cols << log_n).reshape(n_cols, -1)
    root = np.zeros(8, np.uint32)
    O.lib().oracle_bench_commit(O.ptr(cols), n_cols, log_n, blowup, THREADS, O.ptr(root))
    return hexw(root)


def job_result(job) -> dict:
    if job.kind == W.FIB:
        proof = O.prove(job.a, job.b, job.log_n, threads=THREADS)
        return {"kind": "fib", "log_n": job.log_n, "a": job.a, "b": job.b, "len": len(proof),
                "sha256": hashlib.sha256(proof).hexdigest()}
    return {"kind": "commit", "log_n": job.log_n, "n_cols": job.n_cols, "seed": job.seed,
            "root": commit_root(job.log_n, job.n_cols, job.seed)}


def step_digest() -> dict:
    n_cols, log_n, blow, fri_log = 34, 24, 2, 26
    t0 = time.time()
    root = commit_root(log_n, n_cols, bench.SEED, blow)
    src = O.seeded_m31(bench.SEED + 1, 4 << fri_log).reshape(4, -1)
    alphas = np.array(bench.splitmix_m31(bench.SEED + 2, 0, 4 * (fri_log - 3)), np.uint32)
    roots = np.zeros((fri_log - 3, 8), np.uint32)
    last = np.zeros((8, 4), np.uint32)
    O.lib().oracle_bench_fri(O.ptr_array(list(src)), fri_log, O.ptr(alphas), THREADS, O.ptr(roots), O.ptr(last))
    print(f"step {time.time() - t0:.1f}s", flush=True)
    return {"n_cols": n_cols, "log_n": log_n, "blowup": 1 << blow, "fri_log_n": fri_log, "seed": hex(bench.SEED),
            "root": root, "fri_roots": [hexw(r) for r in roots], "last_layer": hexw(last)}


def main(parts):
    data = json.loads(OUT.read_text()) if OUT.exists() else {}

    def save():
        OUT.write_text(json.dumps(data, indent=1, sort_keys=True) + "\n")

    if "step" in parts:
        data["step"] = step_digest()
        save()
    if "mix" in parts:
        res = []
        for i, j in enumerate(W.batched_jobs(64)):
            t0 = time.time()
            res.append(job_result(j))
            print("mix", i, res[-1]["kind"], j.log_n, f"{time.time() - t0:.1f}s", flush=True)
        data["batched_mix"] = {"jobs": "workloads.batched_jobs(64)", "results": res}
        save()
    if "served" in parts:
        first = {}
        for i, (_, job, cls) in enumerate(W.served_arrivals(600)):
            first.setdefault(cls, (i, job))
        out = {}
        for cls, (i, job) in sorted(first.items()):
            t0 = time.time()
            out[cls] = dict(job_result(job), index=i)
            print("served", cls, f"{time.time() - t0:.1f}s", flush=True)
        data["served"] = {"jobs": "workloads.served_arrivals(600): first job of each class", "results": out}
        save()


if __name__ == "__main__":
    main(sys.argv[1:] or ["step", "mix", "served"])
