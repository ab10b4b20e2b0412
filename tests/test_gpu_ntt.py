"""GPU parity: circle NTT entry points (both conventions) against the CPU oracle, bit-exact."""
import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from gpu_util import dev, empty, host, ptr, ptr_array, u32_host, rand_m31  # noqa: E402
import vortexstark_b200 as V  # noqa: E402


@pytest.fixture(scope="module")
def L():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return V.lib()


NATIVE_SIZES = [2, 3, 4, 5, 6, 8, 10, 12, 13, 14, 15, 17, 20, 24]


@pytest.mark.parametrize("log_n", NATIVE_SIZES)
def test_native_evaluate_interpolate(L, log_n):
    rng = np.random.default_rng(log_n)
    x = rand_m31(rng, 1 << log_n)
    tw = O.native_twiddles(log_n)
    d = dev(x)
    L.cuda_circle_ntt_evaluate(ptr(d), ptr(dev(tw["line"])), ptr(dev(tw["circle"])), u32_host(tw["offsets"]),
                               u32_host(tw["sizes"]), log_n - 1, 1 << log_n)
    ev = host(d)
    assert np.array_equal(ev, O.native_evaluate(x, log_n)), L.vs_last_error()
    L.cuda_circle_ntt_interpolate(ptr(d), ptr(dev(tw["iline"])), ptr(dev(tw["icircle"])), u32_host(tw["offsets"]),
                                  u32_host(tw["sizes"]), log_n - 1, 1 << log_n)
    assert np.array_equal(host(d), O.native_interpolate(ev, log_n))
    assert np.array_equal(host(d), x)


@pytest.mark.parametrize("log_n", [6, 14])
@pytest.mark.parametrize("forward", [True, False])
def test_native_batch(L, log_n, forward):
    rng = np.random.default_rng(100 + log_n)
    cols = [rand_m31(rng, 1 << log_n) for _ in range(3)]
    tw = O.native_twiddles(log_n)
    ds = [dev(c) for c in cols]
    arr = ptr_array(ds)
    fn = L.cuda_circle_ntt_evaluate_batch if forward else L.cuda_circle_ntt_interpolate_batch
    fn(ptr(arr), ptr(dev(tw["line" if forward else "iline"])), ptr(dev(tw["circle" if forward else "icircle"])),
       u32_host(tw["offsets"]), u32_host(tw["sizes"]), log_n - 1, 1 << log_n, 3)
    for c, d in zip(cols, ds):
        ref = O.native_evaluate(c, log_n) if forward else O.native_interpolate(c, log_n)
        assert np.array_equal(host(d), ref)


@pytest.mark.parametrize("layer", [0, 1, 5, 9])
@pytest.mark.parametrize("forward", [True, False])
def test_single_layer(L, layer, forward):
    log_n = 10
    rng = np.random.default_rng(layer)
    x = rand_m31(rng, 1 << log_n)
    tw = rand_m31(rng, (1 << log_n) >> (layer + 1))
    d = dev(x)
    L.cuda_circle_ntt_layer(ptr(d), ptr(dev(tw)), layer, 1 << log_n, int(forward))
    assert np.array_equal(host(d), O.ntt_layer(x, tw, layer, forward))


STWO_SIZES = [2, 3, 4, 5, 7, 9, 11, 13, 14, 16, 19, 22]


@pytest.mark.parametrize("log_n", STWO_SIZES)
def test_stwo_evaluate_interpolate(L, log_n):
    rng = np.random.default_rng(200 + log_n)
    x = rand_m31(rng, 1 << log_n)
    fwd, inv = O.stwo_twiddles(log_n)
    d = dev(x)
    L.cuda_stwo_ntt_evaluate(ptr(d), ptr(dev(fwd)), 1 << log_n)
    ev = host(d)
    assert np.array_equal(ev, O.stwo_evaluate(x, log_n)), L.vs_last_error()
    L.cuda_stwo_ntt_interpolate(ptr(d), ptr(dev(inv)), 1 << log_n)
    assert np.array_equal(host(d), x)


@pytest.mark.parametrize("log_n,ncols", [(5, 1), (8, 3), (13, 2), (14, 2), (16, 5), (18, 2), (22, 2), (23, 1),
                                         (24, 1)])
def test_lde_stwo(L, log_n, ncols):
    rng = np.random.default_rng(300 + log_n)
    cols = rand_m31(rng, ncols, 1 << log_n)
    src = dev(cols.reshape(-1))
    N = 1 << (log_n + 2)
    dst = empty(ncols * N)
    V.check(L.vs_lde_stwo(ptr(src), 1 << log_n, ptr(dst), N, ncols, log_n, 2, None), "vs_lde_stwo")
    out = host(dst).reshape(ncols, N)
    if log_n <= 23:
        assert np.array_equal(out, O.stwo_lde_columns(cols, log_n, 2, threads=8))
    else:  # size-independent property: interpolating the LDE gives the trace coefficients zero-padded
        fwd, inv = O.stwo_twiddles(log_n + 2)
        d = dev(out[0])
        L.cuda_stwo_ntt_interpolate(ptr(d), ptr(dev(inv)), N)
        c_big = host(d)
        fwd_s, inv_s = O.stwo_twiddles(log_n)
        d2 = dev(cols[0])
        L.cuda_stwo_ntt_interpolate(ptr(d2), ptr(dev(inv_s)), 1 << log_n)
        assert np.array_equal(c_big[: 1 << log_n], host(d2))
        assert not c_big[1 << log_n:].any()
    assert np.array_equal(host(src).reshape(ncols, -1), cols)  # input untouched


@pytest.mark.parametrize("log_n,blowup", [(22, 1), (22, 3), (23, 1), (24, 1)])
def test_lde_stwo_blowups(L, log_n, blowup):
    """The LDE top pass at the trace sizes whose tile rows are 16-64 bytes (2^24, 2^23
    and 2^22: rows of 16, 32 and 64 bytes; the 16-byte rows run as CTA pairs that
    store whole sectors) for blowups other than 4, two columns at a padded column
    stride, against the oracle."""
    rng = np.random.default_rng(700 + 10 * log_n + blowup)
    ncols, n = 2, 1 << log_n
    N = n << blowup
    cols = rand_m31(rng, ncols, n)
    stride = N + 64  # 64 words of padding between the evaluation columns
    dst = empty(ncols * stride)
    V.check(L.vs_lde_stwo(ptr(dev(cols.reshape(-1))), n, ptr(dst), stride, ncols, log_n, blowup, None), "vs_lde_stwo")
    out = host(dst).reshape(ncols, stride)[:, :N]
    assert np.array_equal(out, O.stwo_lde_columns(cols, log_n, blowup, threads=8))


@pytest.mark.parametrize("log_n", [5, 13, 14, 20, 24])
@pytest.mark.parametrize("native", [False, True])
def test_lde_blowup_one_is_identity(L, log_n, native):
    """An LDE onto the trace's own domain (blowup bits 0) interpolates and evaluates
    on the same domain: it returns its input, bit for bit (the oracle does the same),
    at every pass structure up to the 2^24 top pass run as CTA pairs."""
    rng = np.random.default_rng(900 + log_n)
    ncols, n = 2, 1 << log_n
    cols = rand_m31(rng, ncols, n)
    dst = empty(ncols * n)
    fn = L.vs_lde_native if native else L.vs_lde_stwo
    V.check(fn(ptr(dev(cols.reshape(-1))), n, ptr(dst), n, ncols, log_n, 0, None), "lde")
    assert np.array_equal(host(dst).reshape(ncols, n), cols)


@pytest.mark.parametrize("log_n", [5, 9, 13, 16, 22])
def test_lde_native(L, log_n):
    rng = np.random.default_rng(400 + log_n)
    x = rand_m31(rng, 1 << log_n)
    N = 1 << (log_n + 2)
    dst = empty(N)
    V.check(L.vs_lde_native(ptr(dev(x)), 0, ptr(dst), 0, 1, log_n, 2, None), "vs_lde_native")
    coeffs = O.native_interpolate(x, log_n)
    padded = np.zeros(N, np.uint32)
    padded[: 1 << log_n] = coeffs
    assert np.array_equal(host(dst), O.native_evaluate(padded, log_n + 2))


@pytest.mark.parametrize("log_n", [1, 4, 10, 17])
def test_bit_reverse(L, log_n):
    rng = np.random.default_rng(log_n)
    x = rand_m31(rng, 1 << log_n)
    d = dev(x)
    L.cuda_bit_reverse_m31(ptr(d), log_n)
    assert np.array_equal(host(d), O.bit_reverse(x, log_n))
    q = rand_m31(rng, (1 << log_n) * 4)
    out = empty(q.size)
    L.cuda_bit_reverse_qm31(ptr(dev(q)), ptr(out), 1 << log_n, log_n)
    idx = np.array([int(format(i, f"0{log_n}b")[::-1], 2) if log_n else 0 for i in range(1 << log_n)])
    exp = np.empty_like(q.reshape(-1, 4))
    exp[idx] = q.reshape(-1, 4)
    assert np.array_equal(host(out).reshape(-1, 4), exp)


def test_eval_at_point(L):
    from gpu_util import qm_add, qm_mul
    log_n = 6
    rng = np.random.default_rng(5)
    c = rand_m31(rng, 1 << log_n)
    f = rand_m31(rng, log_n, 4)
    s1, s2 = empty(4 << log_n), empty(4 << log_n)
    res = (__import__("ctypes").c_uint32 * 4)()
    L.cuda_eval_at_point(ptr(dev(c)), ptr(dev(f.reshape(-1))), res, 1 << log_n, ptr(s1), ptr(s2))
    cur = [[int(v), 0, 0, 0] for v in c]
    for lvl in range(log_n):
        h = len(cur) // 2
        cur = [qm_add(cur[i], qm_mul(cur[i + h], f[lvl])) for i in range(h)]
    assert list(res) == cur[0]
