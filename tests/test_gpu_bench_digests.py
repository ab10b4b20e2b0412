"""GPU: the benchmark workloads at their own sizes, bit for bit against the
oracle's results (tests/golden/bench_digests.json, written by
tests/golden/gen_bench_digests.py, which runs the oracle for minutes).

* the commitment-layer step of bench.py: 34 columns x 2^24 rows, x4 stwo LDE,
  row-packed root (at split 0 and the largest split), and the FRI fold+commit of
  the seeded 2^26 QM31 vector: 23 layer roots and the last layer;
* the 64-job batched mix (log_n 16..22 Fibonacci proofs and 1..34-column
  commitments) through the batching engine and through the plain path;
* the first job of each served size class (Fibonacci 16/20/24, commits 34 x
  2^18/2^20/2^22) through the engine."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import bench  # noqa: E402
from vortexstark_b200 import api  # noqa: E402
from vortexstark_b200 import workloads as W  # noqa: E402

D = json.loads((Path(__file__).resolve().parent / "golden" / "bench_digests.json").read_text())


def hexw(t) -> str:
    return t.cpu().numpy().view(np.uint32).tobytes().hex()


def matches(expected: dict, got: bytes) -> bool:
    if expected["kind"] == "fib":
        return len(got) == expected["len"] and hashlib.sha256(got).hexdigest() == expected["sha256"]
    return got.hex() == expected["root"]


@pytest.fixture(scope="module")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def test_commitment_step_at_bench_size(cuda):
    d = D["step"]
    n_cols, log_n, fri_log = d["n_cols"], d["log_n"], d["fri_log_n"]
    dev = torch.device("cuda")
    cols = api.fill_uniform_m31(torch.empty((n_cols, 1 << log_n), dtype=torch.int32, device=dev), bench.SEED)
    lde = api.lde_stwo(cols, log_n, 2)
    root = torch.zeros(8, dtype=torch.int32, device=dev)
    prev = api.merkle_split()
    try:
        for split in (0, 8):
            api.set_merkle_split(split)
            root.zero_()
            api.merkle_root_rowpacked(lde, root)
            assert hexw(root) == d["root"], f"row-packed root differs at split {split}"
    finally:
        api.set_merkle_split(prev)
    root.zero_()
    api.commit_columns(cols, log_n, 2, lde, root)
    assert hexw(root) == d["root"]
    del lde, cols
    torch.cuda.empty_cache()
    src = api.fill_uniform_m31(torch.empty((4, 1 << fri_log), dtype=torch.int32, device=dev), bench.SEED + 1)
    a = bench.splitmix_m31(bench.SEED + 2, 0, 4 * (fri_log - 3))
    alphas = [a[4 * i:4 * i + 4] for i in range(fri_log - 3)]
    work = torch.empty(4 << fri_log, dtype=torch.int32, device=dev)
    roots = torch.zeros(8 * (fri_log - 3), dtype=torch.int32, device=dev)
    last = torch.zeros(32, dtype=torch.int32, device=dev)
    api.fri_fold_commit(src, fri_log, alphas, work, roots, last)
    got = [hexw(roots[8 * i:8 * i + 8]) for i in range(fri_log - 3)]
    assert got == d["fri_roots"]
    assert hexw(last) == d["last_layer"]


def test_batched_mix_at_bench_size(cuda):
    jobs = W.batched_jobs(64)
    exp = D["batched_mix"]["results"]
    assert len(exp) == len(jobs)
    with api.Engine(8, size_priority=False) as eng:
        res = [eng.wait(t)[0] for t in [eng.submit(j) for j in jobs]]
    bad = [i for i, (e, r) in enumerate(zip(exp, res)) if not matches(e, r)]
    assert not bad, f"engine results differ from the oracle for jobs {bad}"
    _, plain = W.run_plain(jobs)
    bad = [i for i, (e, r) in enumerate(zip(exp, plain)) if not matches(e, r)]
    assert not bad, f"plain-path results differ from the oracle for jobs {bad}"


def test_served_classes_at_bench_size(cuda):
    arrivals = W.served_arrivals(600)
    with api.Engine(4, 150 * 10**9) as eng:
        for cls, e in sorted(D["served"]["results"].items()):
            job = arrivals[e["index"]][1]
            assert arrivals[e["index"]][2] == cls
            got = eng.wait(eng.submit(job))[0]
            assert matches(e, got), cls
