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
