"""GPU: the graph-captured prover and the batched / served engine.

Every result must be byte-identical to the oracle, and identical whether a job
runs alone (one slot) or in a mix of concurrently admitted jobs."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import vortexstark_b200 as V  # noqa: E402


class Job(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("log_n", C.c_uint32), ("a", C.c_uint32), ("b", C.c_uint32),
                ("n_cols", C.c_uint32), ("pad", C.c_uint32), ("seed", C.c_uint64)]


class JobResult(C.Structure):
    _fields_ = [("status", C.c_int), ("pad", C.c_uint32), ("out_len", C.c_uint64), ("t_submit", C.c_double),
                ("t_start", C.c_double), ("t_end", C.c_double)]


@pytest.fixture(scope="module")
def L():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return V.lib()


def graph_prove(L, log_n, pairs):
    h = C.c_void_p()
    V.check(L.vs_prover_create(log_n, C.byref(h)), "vs_prover_create")
    cap = 16 << 20
    buf = (C.c_uint8 * cap)()
    n = C.c_uint64()
    out = []
    for a, b in pairs:
        V.check(L.vs_prover_prove(h, a, b, buf, cap, C.byref(n)), "vs_prover_prove")
        out.append(bytes(buf[: n.value]))
    L.vs_prover_destroy(h)
    return out


@pytest.mark.parametrize("log_n", [4, 6, 9, 12, 16])
def test_graph_prover_matches_oracle(L, log_n):
    pairs = [(1, 1), (7, 123456789)]
    proofs = graph_prove(L, log_n, pairs)
    for (a, b), p in zip(pairs, proofs):
        assert p == O.prove(a, b, log_n)
    assert O.verify(proofs[0]) == (0, "")


def commit_root_oracle(log_n, n_cols, seed):
    cols = O.seeded_m31(seed, n_cols << log_n).reshape(n_cols, -1)
    return O.merkle_root_rowpacked(O.stwo_lde_columns(cols, log_n, 2, threads=8), threads=8).tobytes()


def run_engine(L, jobs, slots, budget=0, flags=None):
    eng = C.c_void_p()
    if flags is None:
        V.check(L.vs_engine_create(slots, budget, C.byref(eng)), "vs_engine_create")
    else:
        V.check(L.vs_engine_create_ex(slots, budget, flags, C.byref(eng)), "vs_engine_create_ex")
    try:
        tickets = []
        for j in jobs:
            t = C.c_uint64()
            V.check(L.vs_engine_submit(eng, C.byref(j), C.byref(t)), "submit")
            tickets.append(t.value)
        out = []
        buf = (C.c_uint8 * (16 << 20))()
        for t in tickets:
            r = JobResult()
            V.check(L.vs_engine_wait(eng, t, C.byref(r), buf, len(buf)), "wait")
            out.append((bytes(buf[: r.out_len]), r.t_submit, r.t_start, r.t_end))
        return out
    finally:
        L.vs_engine_destroy(eng)


def mixed_jobs():
    rng = np.random.default_rng(5)
    jobs = []
    for i in range(12):
        if i % 3 == 2:
            jobs.append(Job(1, int(rng.integers(5, 11)), 0, 0, int(rng.integers(1, 35)), 0, 0x9000 + i))
        else:
            jobs.append(Job(0, int(rng.integers(4, 12)), 1, int(rng.integers(1, 2**31 - 1)), 0, 0, 0))
    return jobs


def test_engine_mix_equals_alone_and_oracle(L):
    jobs = mixed_jobs()
    alone = run_engine(L, jobs, slots=1)
    mixed = run_engine(L, jobs, slots=6)
    for j, (a, *_), (m, *_) in zip(jobs, alone, mixed):
        assert a == m
        if j.kind == 0:
            assert a == O.prove(j.a, j.b, j.log_n)
        else:
            assert a == commit_root_oracle(j.log_n, j.n_cols, j.seed)


def test_engine_budget_admission(L):
    """A budget below two jobs' working sets serialises them; results are unchanged."""
    jobs = [Job(0, 10, 1, 2, 0, 0, 0), Job(0, 10, 3, 4, 0, 0, 0), Job(1, 9, 0, 0, 20, 0, 77)]
    res = run_engine(L, jobs, slots=3, budget=1 << 20)
    assert res[0][0] == O.prove(1, 2, 10) and res[1][0] == O.prove(3, 4, 10)
    assert res[2][0] == commit_root_oracle(9, 20, 77)
    spans = sorted((r[2], r[3]) for r in res)
    for (s0, e0), (s1, e1) in zip(spans, spans[1:]):
        assert s1 >= e0 - 1e-6  # no two ran at the same time


def test_engine_rejects_bad_jobs(L):
    eng = C.c_void_p()
    V.check(L.vs_engine_create(2, 0, C.byref(eng)))
    try:
        t = C.c_uint64()
        assert L.vs_engine_submit(eng, C.byref(Job(9, 10, 1, 1, 0, 0, 0)), C.byref(t)) == 1
        V.check(L.vs_engine_submit(eng, C.byref(Job(0, 2, 1, 1, 0, 0, 0)), C.byref(t)))
        r = JobResult()
        assert L.vs_engine_wait(eng, t.value, C.byref(r), None, 0) == 1 and r.status == 1
    finally:
        L.vs_engine_destroy(eng)


def test_engine_priority_policy_does_not_change_results(L):
    """Size-based stream priorities (default) and equal priorities give the same bytes."""
    jobs = mixed_jobs()
    by_size = run_engine(L, jobs, slots=6, flags=0)
    fifo = run_engine(L, jobs, slots=6, flags=1)
    assert [r[0] for r in by_size] == [r[0] for r in fifo]
    eng = C.c_void_p()
    assert L.vs_engine_create_ex(2, 0, 0x80, C.byref(eng)) == 1  # unknown flag rejected
