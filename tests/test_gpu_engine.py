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
    """A budget that holds one workspace at a time (here any two workspaces exceed
    it) serialises jobs of different shapes: the idle workspace of one shape is
    freed for the next. Results are unchanged."""
    from vortexstark_b200 import api
    # commitment workspaces of equal size (rows x columns held constant): any two
    # exceed the budget (batched proofs get workspaces sized to their batch, which
    # for single jobs are small enough to share a budget like this)
    jobs = [api.commit_job(20, 34, 77), api.commit_job(19, 68, 78), api.commit_job(18, 136, 79)]
    with api.Engine(1) as probe:
        sizes = sorted(probe.workspace_bytes(j) for j in jobs)
        tw_now = probe.stats()["twiddle_bytes"]
    margin = 128 << 20  # the twiddle tables these shapes build (stwo tables of 2^18-2^22: about 62 MB)
    budget = sizes[-1] + tw_now + margin
    assert sizes[0] + sizes[1] > sizes[-1] + margin
    with api.Engine(3, budget) as eng:
        tickets = [eng.submit(j) for j in jobs]
        res = [eng.wait(t) for t in tickets]
        st = eng.stats()
    for j, r in zip(jobs, res):
        assert r[0] == api.commit_seeded(j.log_n, j.n_cols, j.seed)
    spans = sorted((r[2], r[3]) for r in res)
    for (s0, e0), (s1, e1) in zip(spans, spans[1:]):
        assert s1 >= e0 - 1e-6  # no two ran at the same time
    assert st["peak_held_bytes"] <= budget and st["evictions"] >= 2


# ---------------------------------------------------------------- batched proofs, budget, failure paths
def _occupy_then_submit(eng, jobs, log_n_block=18):
    """Submits a blocking commitment first, so the following jobs queue up and a
    slot takes them as one batch."""
    from vortexstark_b200 import api
    first = eng.submit(api.commit_job(log_n_block, 34, 0x77))
    return first, [eng.submit(j) for j in jobs]


def test_batch_workspace_sized_to_batch(L):
    """A batch that finds no idle workspace of its size gets one sized to it (the
    next power of two of its proofs), far below the full-capacity workspace; a
    prepared full-capacity workspace serves a batch of any size, so nothing new is
    created for it. Results are the oracle's either way."""
    from vortexstark_b200 import api
    jobs = [api.fib_job(12, 1, k) for k in range(3)]
    expected = [O.prove(1, k, 12) for k in range(3)]
    block = api.commit_job(18, 34, 0x77)
    with api.Engine(1) as eng:
        full = eng.workspace_bytes(jobs[0])
        commit_bytes = eng.workspace_bytes(block)
        first, ts = _occupy_then_submit(eng, jobs)
        eng.wait(first)
        assert [eng.wait(t)[0] for t in ts] == expected
        st = eng.stats()
    assert st["workspaces_created"] == 2  # the blocking commitment's and the batch's
    assert st["resident_bytes"] - commit_bytes < full // 4  # a workspace for 4 proofs, not 64
    with api.Engine(1) as eng:
        eng.prepare(jobs[0])
        created = eng.stats()["workspaces_created"]
        first, ts = _occupy_then_submit(eng, jobs)
        eng.wait(first)
        assert [eng.wait(t)[0] for t in ts] == expected
        assert eng.stats()["workspaces_created"] == created + 1  # only the commitment's


@pytest.mark.parametrize("log_n", [4, 7, 10, 13])
def test_batched_proofs_match_oracle_and_plain(L, log_n):
    """Jobs of one size queued together run as one batch (one graph launch); every
    proof equals the oracle's, vs_prove_fib's and the unbatched engine's bytes."""
    from vortexstark_b200 import api
    pairs = [(1, 1), (1, 5), (3, 4), (7, 123456789), (2**31 - 2, 0), (0, 0)]
    jobs = [api.fib_job(log_n, a, b) for a, b in pairs]
    with api.Engine(1) as eng:
        first, ts = _occupy_then_submit(eng, jobs)
        eng.wait(first)
        batched = [eng.wait(t) for t in ts]
    # all but possibly the first job started together: one batch
    assert len({round(r[2], 9) for r in batched[1:]}) == 1
    with api.Engine(2) as eng:
        eng.set_batch_limit(1)
        single = [eng.wait(eng.submit(j))[0] for j in jobs]
    for (a, b), r, s1 in zip(pairs, batched, single):
        assert r[0] == s1 == O.prove(a, b, log_n) == api.prove_fib(a, b, log_n)
    assert api.verify_fib(batched[0][0]) == (True, "")


def test_batch_capacity_limit_and_mixed_sizes(L):
    """Batches never mix sizes or exceed the limit; results do not depend on batching."""
    from vortexstark_b200 import api
    rng = np.random.default_rng(11)
    jobs = [api.fib_job(int(rng.integers(5, 9)), 1, int(rng.integers(0, 2**31 - 1))) for _ in range(20)]
    with api.Engine(2) as eng:
        eng.set_batch_limit(3)
        first, ts = _occupy_then_submit(eng, jobs)
        eng.wait(first)
        res = [eng.wait(t) for t in ts]
    starts = {}
    for j, r in zip(jobs, res):
        starts.setdefault(round(r[2], 9), set()).add(j.log_n)
    assert all(len(v) == 1 for v in starts.values())  # one size per batch
    counts = {}
    for r in res:
        counts[round(r[2], 9)] = counts.get(round(r[2], 9), 0) + 1
    assert max(counts.values()) <= 3
    for j, r in zip(jobs, res):
        assert r[0] == O.prove(j.a, j.b, j.log_n)


def test_engine_holds_at_most_the_budget(L):
    """With a budget below the sum of the shapes' workspaces the engine frees idle
    workspaces to admit new shapes: its accounted peak and the device memory it
    actually takes (cudaMemGetInfo) stay within the budget, and results match an
    unlimited engine."""
    import threading
    import time

    from vortexstark_b200 import api
    shapes = [api.fib_job(15, 1, 0), api.fib_job(16, 1, 0), api.commit_job(17, 20, 0), api.commit_job(16, 34, 0),
              api.fib_job(17, 1, 0)]
    rng = np.random.default_rng(3)
    jobs = []
    for i in range(24):
        s = shapes[int(rng.integers(0, len(shapes)))]
        if s.kind == api.FIB:
            jobs.append(api.fib_job(s.log_n, 1, int(rng.integers(0, 2**31 - 1))))
        else:
            jobs.append(api.commit_job(s.log_n, s.n_cols, int(rng.integers(1, 1 << 40))))
    with api.Engine(1) as probe:
        probe.set_batch_limit(4)
        sizes = [probe.workspace_bytes(s) for s in shapes]
    with api.Engine(1) as e:
        tw_now = e.stats()["twiddle_bytes"]
    extra = 32 << 20  # the twiddle tables these shapes build
    budget = max(sizes) * 2 + tw_now + extra
    assert max(sizes) * 2 + extra < sum(sizes) * 2  # not every shape (two slots' worth) fits at once
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    low = [free0]
    stop = False

    def poll():
        while not stop:
            low[0] = min(low[0], torch.cuda.mem_get_info()[0])
            time.sleep(0.002)

    th = threading.Thread(target=poll)
    th.start()
    try:
        with api.Engine(2, budget, size_priority=False) as eng:
            eng.set_batch_limit(4)
            ts = [eng.submit(j) for j in jobs]
            got = [eng.wait(t)[0] for t in ts]
            st = eng.stats()
    finally:
        stop = True
        th.join()
    assert st["peak_held_bytes"] <= budget
    assert st["evictions"] > 0
    assert free0 - low[0] <= budget + (64 << 20)  # context-side graph/stream memory as slack
    with api.Engine(2) as eng:
        eng.set_batch_limit(4)
        ref = [eng.wait(eng.submit(j))[0] for j in jobs]
    assert got == ref


def test_engine_small_budget_gets_smaller_batches(L):
    """A budget below a full batch workspace (64 proofs at log_n 16) still runs the
    jobs, in smaller batches, with the same proofs."""
    from vortexstark_b200 import api
    torch.cuda.synchronize()
    V.check(L.vs_release_caches(), "vs_release_caches")  # earlier tests' twiddle tables would count
    job = api.fib_job(16, 1, 7)
    with api.Engine(1) as probe:
        full = probe.workspace_bytes(job)
    budget = full // 4 + (64 << 20)  # + the twiddle tables of log_n 16 and 18
    with api.Engine(2, budget) as eng:
        small = eng.workspace_bytes(job)
        assert small < full
        jobs = [api.fib_job(16, 1, k) for k in range(6)]
        res = [eng.wait(t)[0] for t in eng.submit_many(jobs)]
        assert eng.stats()["peak_held_bytes"] <= budget
    assert res == [api.prove_fib(1, k, 16) for k in range(6)]


def test_engine_rejects_job_above_budget(L):
    from vortexstark_b200 import api
    with api.Engine(2, 1 << 20) as eng:
        rc, out = eng.wait_status(eng.submit(api.fib_job(10, 1, 1)))
        assert rc == api.VS_ERR_BUDGET and out == b""
        assert eng.stats()["resident_bytes"] == 0


def test_engine_cancel_and_timeout(L):
    """A queued job can be cancelled; a bounded wait on a running job times out
    (the ticket stays valid) and the job still completes."""
    import time

    from vortexstark_b200 import api
    with api.Engine(1) as eng:
        eng.prepare(api.fib_job(22, 1, 1))
        long_t = eng.submit(api.fib_job(22, 1, 1))
        t0 = time.time()
        while eng.stats()["running"] == 0 and time.time() - t0 < 10:
            time.sleep(0.0001)
        queued = [eng.submit(api.fib_job(8, 1, k)) for k in range(3)]
        assert eng.cancel(queued[1]) == 0
        r = JobResult()
        rc = L.vs_engine_wait_for(eng.h, long_t, 0.0, C.byref(r), None, 0)  # length query: nothing retired
        assert rc in (0, api.VS_ERR_TIMEOUT)
        assert eng.cancel(long_t) == api.VS_ERR_BUSY  # running or finished: not cancellable
        assert eng.wait(long_t)[0] == api.prove_fib(1, 1, 22)
        assert eng.wait_status(queued[1])[0] == api.VS_ERR_CANCELLED
        assert eng.wait(queued[0])[0] == O.prove(1, 0, 8)
        assert eng.wait(queued[2])[0] == O.prove(1, 2, 8)
        assert L.vs_engine_cancel(eng.h, 10**9) == 1  # unknown ticket


def test_engine_injected_allocation_failure(L):
    """A workspace allocation that fails (injected on the host) fails its job with
    VS_ERR_OOM and leaves the engine usable, with nothing counted as resident."""
    from vortexstark_b200 import api
    with api.Engine(1) as eng:
        eng.inject_alloc_failures(1)
        rc, _ = eng.wait_status(eng.submit(api.fib_job(9, 1, 3)))
        assert rc == api.VS_ERR_OOM
        assert eng.stats()["resident_bytes"] == 0
        assert eng.wait(eng.submit(api.fib_job(9, 1, 3)))[0] == O.prove(1, 3, 9)
        st = eng.stats()
        assert st["resident_bytes"] > 0 and st["idle_workspaces"] == 1
