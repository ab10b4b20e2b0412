"""CPU, world size 2 over gloo: the replica path of bench.py --gpus N (job-level
sharding, rank input windows, max over ranks of the timed region).

Each rank commits its share of a mixed job list with the oracle; rank 0 checks
that the gathered results equal the one-process results job by job, that the
ranks' seeded input windows concatenate to the single-process stream, and that
the reported time is the slowest rank's."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle_lib as O
from vortexstark_b200 import replicas
from vortexstark_b200.workloads import batched_jobs


def small_jobs():
    # the batched mix, shrunk to oracle-friendly sizes (log_n 4..7, up to 6 columns)
    jobs = batched_jobs(16)
    return [(j.kind, 4 + j.log_n % 4, j.a, j.b, 1 + j.n_cols % 6, j.seed) for j in jobs]


def run_job(job):
    kind, log_n, a, b, n_cols, seed = job
    if kind == 0:
        return O.prove(a, b, log_n, threads=1)
    cols = O.seeded_m31(seed, n_cols << log_n).reshape(n_cols, -1)
    return O.merkle_root_rowpacked(O.stwo_lde_columns(cols, log_n, 2)).tobytes()


def worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    try:
        r, w, _ = replicas.init("gloo", timeout_s=60)
        jobs = small_jobs()
        mine = replicas.shard(list(enumerate(jobs)), r, w)
        out = [(i, run_job(j)) for i, j in mine]
        words = 3 << 10
        window = O.seeded_m31(0x56530001, words, replicas.input_offset(r, words))
        slowest = replicas.max_over_ranks(1.5 + r)
        gathered = [None] * w
        dist.all_gather_object(gathered, (out, window.tobytes(), slowest))
        replicas.barrier()
        if r == 0:
            q.put(gathered)
        replicas.finalize()
    except Exception as e:  # surfaced to the parent
        q.put(repr(e))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_replicas_over_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        gathered = q.get(timeout=240)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert not isinstance(gathered, str), gathered
    jobs = small_jobs()
    results = {}
    for out, _, _ in gathered:
        for i, res in out:
            assert i not in results  # every job on exactly one rank
            results[i] = res
    assert sorted(results) == list(range(len(jobs)))
    for i, j in enumerate(jobs):
        assert results[i] == run_job(j)
    words = 3 << 10
    whole = O.seeded_m31(0x56530001, world * words)
    assert b"".join(g[1] for g in gathered) == whole.tobytes()
    assert all(g[2] == 1.5 + world - 1 for g in gathered)


def test_shard_rejects_bad_rank():
    with pytest.raises(ValueError):
        replicas.shard([1, 2, 3], 2, 2)
    assert replicas.shard(range(5), 1, 2) == [1, 3]
    assert np.array_equal(np.array(replicas.shard(range(6), 0, 3)), [0, 3])

