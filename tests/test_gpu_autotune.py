"""GPU checks of the NTT launch-shape autotuner: every candidate plan gives the
oracle's LDE and NTT bit for bit (plans regroup layers into launches, nothing
else), and the tuner keeps one of the candidates and leaves results unchanged."""
import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from gpu_util import dev, empty, host, ptr, rand_m31  # noqa: E402
import vortexstark_b200 as V  # noqa: E402
from vortexstark_b200 import api  # noqa: E402


@pytest.fixture(scope="module")
def L():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return V.lib()


@pytest.fixture(autouse=True)
def default_plans():
    yield
    if torch.cuda.is_available():
        for log_n in range(5, 31):
            api.set_ntt_plan(log_n)


def _lde(L, cols, log_n, native=False):
    n_cols = cols.shape[0]
    N = 1 << (log_n + 2)
    dst = empty(n_cols * N)
    fn = L.vs_lde_native if native else L.vs_lde_stwo
    V.check(fn(ptr(dev(cols.reshape(-1))), 1 << log_n, ptr(dst), N, n_cols, log_n, 2, None), "lde")
    return host(dst).reshape(n_cols, N)


@pytest.mark.parametrize("log_n", [14, 16, 18])
def test_every_candidate_plan_matches_oracle(L, log_n):
    rng = np.random.default_rng(700 + log_n)
    cols = rand_m31(rng, 3, 1 << log_n)
    exp = O.stwo_lde_columns(cols, log_n, 2, threads=4)
    cands = api.ntt_plan_candidates(log_n)
    assert len(cands) >= 6
    for plan in cands:
        api.set_ntt_plan(log_n, *plan)
        assert api.ntt_plan(log_n) == tuple(plan)
        assert np.array_equal(_lde(L, cols, log_n), exp), plan


@pytest.mark.parametrize("log_n", [15, 17])
def test_plans_native_lde_and_transforms(L, log_n):
    rng = np.random.default_rng(800 + log_n)
    x = rand_m31(rng, 1, 1 << log_n)
    padded = np.zeros(1 << (log_n + 2), np.uint32)
    padded[: 1 << log_n] = O.native_interpolate(x[0], log_n)
    ref = O.native_evaluate(padded, log_n + 2)[None, :]
    fwd_tw, inv_tw = O.stwo_twiddles(log_n)
    exp_eval = O.stwo_evaluate(x[0], log_n)
    for plan in api.ntt_plan_candidates(log_n)[::5]:
        api.set_ntt_plan(log_n, *plan)
        assert np.array_equal(_lde(L, x, log_n, native=True), ref), plan
        d = dev(x[0])
        L.cuda_stwo_ntt_evaluate(ptr(d), ptr(dev(fwd_tw)), 1 << log_n)
        assert np.array_equal(host(d), exp_eval), plan
        L.cuda_stwo_ntt_interpolate(ptr(d), ptr(dev(inv_tw)), 1 << log_n)
        assert np.array_equal(host(d), x[0]), plan
    api.set_ntt_plan(log_n)
    assert np.array_equal(_lde(L, x, log_n, native=True), ref)


def test_autotune_keeps_a_candidate_and_results(L):
    log_n = 18
    res = api.autotune_lde(log_n, n_cols=4, reps=2)
    cands = api.ntt_plan_candidates(log_n)
    assert tuple(res["best"]) in [tuple(c) for c in cands]
    assert api.ntt_plan(log_n) == tuple(res["best"])
    times = [ms for _, ms in res["candidates"]]
    assert len(times) == len(cands) and all(t > 0 for t in times)
    assert dict((tuple(c), t) for c, t in res["candidates"])[tuple(res["best"])] == min(times)
    rng = np.random.default_rng(9)
    cols = rand_m31(rng, 2, 1 << log_n)
    assert np.array_equal(_lde(L, cols, log_n), O.stwo_lde_columns(cols, log_n, 2, threads=4))


# ------------------------------------------------------------------ Merkle split
@pytest.fixture
def default_split():
    yield
    if torch.cuda.is_available():
        api.set_merkle_split(0)


@pytest.mark.parametrize("log_n,n_cols", [(11, 34), (15, 34), (17, 5)])
def test_every_split_gives_the_oracle_roots(L, default_split, log_n, n_cols):
    from gpu_util import u32_host
    rng = np.random.default_rng(900 + log_n)
    cols = rand_m31(rng, n_cols, 1 << log_n)
    exp_rp = O.merkle_root_rowpacked(cols, threads=4)
    n_cap = min(16, n_cols)
    exp_cap = O.merkle_root_capped(cols[:n_cap], threads=4)
    fri_log = log_n
    src = rand_m31(rng, 4, 1 << fri_log)
    alphas = rand_m31(rng, fri_log - 3, 4)
    er = np.zeros((fri_log - 3, 8), np.uint32)
    el = np.zeros((8, 4), np.uint32)
    O.lib().oracle_bench_fri(O.ptr_array(list(src)), fri_log, O.ptr(alphas.reshape(-1).copy()), 4, O.ptr(er), O.ptr(el))
    d_cols = dev(cols.reshape(-1))
    for split in range(9):
        api.set_merkle_split(split)
        root = empty(8)
        V.check(L.vs_merkle_root_rowpacked(ptr(d_cols), 1 << log_n, n_cols, log_n, ptr(root), None), "rowpacked")
        assert np.array_equal(host(root), exp_rp), split
        V.check(L.vs_merkle_root_capped(ptr(d_cols), 1 << log_n, n_cap, log_n, ptr(root), None), "capped")
        assert np.array_equal(host(root), exp_cap), split
        work, roots, last = empty(4 << fri_log), empty(8 * (fri_log - 3)), empty(32)
        V.check(L.vs_fri_fold_commit(ptr(dev(src.reshape(-1))), fri_log, u32_host(alphas.reshape(-1)), ptr(work),
                                     ptr(roots), ptr(last), None), "vs_fri_fold_commit")
        assert np.array_equal(host(roots).reshape(-1, 8), er), split
        assert np.array_equal(host(last).reshape(8, 4), el), split


def test_autotune_merkle_keeps_a_split(L, default_split):
    res = api.autotune_merkle(16, n_cols=34, reps=2)
    assert 0 <= res["best"] <= 8 and api.merkle_split() == res["best"]
    assert all(t > 0 for t in res["ms"]) and res["ms"][res["best"]] == min(res["ms"])


@pytest.mark.parametrize("split", [1, 5, 8])
def test_prover_trees_with_split_match_oracle(L, default_split, split):
    """Proof trees of 2^20 leaves (log_n 18) go through 2^min(split, 5) subtree
    roots per tile in both provers; the bytes stay the oracle's."""
    import ctypes as C
    exp = O.prove(3, 77, 18)
    api.set_merkle_split(split)
    assert api.prove_fib(3, 77, 18) == exp
    h = C.c_void_p()
    V.check(L.vs_prover_create(18, C.byref(h)), "vs_prover_create")
    try:
        cap = 16 << 20
        buf = (C.c_uint8 * cap)()
        n = C.c_uint64()
        V.check(L.vs_prover_prove(h, 3, 77, buf, cap, C.byref(n)), "vs_prover_prove")
        assert bytes(buf[: n.value]) == exp
    finally:
        L.vs_prover_destroy(h)
