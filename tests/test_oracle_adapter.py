"""CPU checks of the oracle's restatement of the stwo Backend adapter kernels
(cuda/gather.cu, cuda/barycentric_eval.cu, cuda/accumulate_lift.cu,
cuda/pack_leaves.cu) against a second, numpy statement of the same formulas."""
import numpy as np
import pytest

import oracle_lib as O

P = O.P


def _m31(rng, n):
    return rng.integers(0, P, size=n, dtype=np.uint64).astype(np.uint32)


def test_gather_u32_and_u256():
    rng = np.random.default_rng(1)
    src = _m31(rng, 1000)
    idx = rng.integers(0, 1000, size=333).astype(np.uint32)
    assert np.array_equal(O.gather_u32(src, idx), src[idx])
    hashes = _m31(rng, 8 * 77).reshape(77, 8)
    idx = rng.integers(0, 77, size=50).astype(np.uint32)
    assert np.array_equal(O.gather_u256(hashes.ravel(), idx), hashes[idx].ravel())
    assert O.gather_u32(src, np.zeros(0, np.uint32)).size == 0


@pytest.mark.parametrize("n,n_blocks", [(1, 1), (255, 1), (256, 3), (1000, 4), (5000, 7), (70000, 256), (300, 256)])
def test_barycentric_partials(n, n_blocks):
    rng = np.random.default_rng(n)
    e = _m31(rng, n).astype(object)
    w = _m31(rng, 4 * n).reshape(n, 4).astype(object)
    exp = np.zeros((n_blocks, 4), dtype=object)
    for i in range(n):
        exp[(i // 256) % n_blocks] += w[i] * e[i]
    exp = (exp % P).astype(np.uint32)
    got = O.barycentric_partials(e.astype(np.uint32), w.astype(np.uint32).ravel(), n_blocks)
    assert np.array_equal(got, exp)


@pytest.mark.parametrize("log_col,log_curr", [(1, 1), (4, 1), (6, 3), (10, 10), (12, 5)])
def test_accumulate_lift(log_col, log_curr):
    rng = np.random.default_rng(log_col * 31 + log_curr)
    col = _m31(rng, 4 << log_col).reshape(-1, 4)
    curr = _m31(rng, 4 << log_curr).reshape(-1, 4)
    r = log_col - log_curr
    i = np.arange(1 << log_col)
    s = ((i >> (r + 1)) << 1) | (i & 1)
    exp = ((col.astype(np.uint64) + curr[s].astype(np.uint64)) % P).astype(np.uint32)
    assert np.array_equal(O.accumulate_lift(col.ravel(), curr.ravel(), r).reshape(-1, 4), exp)


@pytest.mark.parametrize("n", [16, 64, 4096, 40, 7])
def test_pack_leaves(n):
    rng = np.random.default_rng(n)
    cols = _m31(rng, 4 * n).reshape(4, n)
    got = O.pack_leaves(cols)
    g = (n + 15) // 16
    exp = np.zeros((64, g), np.uint32)
    for c in range(4):
        for k in range(n):
            exp[16 * c + k % 16, k // 16] = cols[c, k]
    assert np.array_equal(got, exp)
    if n % 16 == 0:
        # the stwo PackLeaves layout: output column 16c + p holds input c's words p, p+16, ...
        assert np.array_equal(got.reshape(4, 16, n // 16), cols.reshape(4, n // 16, 16).transpose(0, 2, 1))


# ---- domain helpers behind the adapter (fri_ops.rs:50-56,100-106; quotient_ops.rs:135-140)
G = (2, 1268011823)


def _pmul(a, b):
    return ((a[0] * b[0] - a[1] * b[1]) % P, (a[0] * b[1] + a[1] * b[0]) % P)


def _dbl(p, k):
    for _ in range(k):
        p = _pmul(p, p)
    return p


def _ppow(p, e):
    r = (1, 0)
    while e:
        if e & 1:
            r = _pmul(r, p)
        p = _pmul(p, p)
        e >>= 1
    return r


def _brev(i, bits):
    return int(format(i, f"0{bits}b")[::-1], 2) if bits else 0


def _half_odds(l):
    return _dbl(G, 29 - l if l < 29 else 0), _dbl(G, 31 - l)


def _circle_domain_at(half, i, log_size):
    """stwo CircleDomain::at: half_coset.at(i) for i < 2^(log_size-1), else its conjugate."""
    init, step = half
    h = 1 << (log_size - 1)
    p = _pmul(init, _ppow(step, i % h))
    return p if i < h else (p[0], (-p[1]) % P)


@pytest.mark.parametrize("log_size", [1, 2, 3, 5, 8])
def test_canonic_domain_points_restatement(log_size):
    xs, ys = O.canonic_domain_points(log_size)
    half = _half_odds(log_size - 1)
    for r in range(1 << log_size):
        assert (int(xs[r]), int(ys[r])) == _circle_domain_at(half, _brev(r, log_size), log_size)
        assert (int(xs[r]) ** 2 + int(ys[r]) ** 2) % P == 1
    assert len(set(zip(xs.tolist(), ys.tolist()))) == 1 << log_size


@pytest.mark.parametrize("log_size", [2, 4, 7])
def test_fold_twiddles_of_stwo_domains(log_size):
    """1/y of CircleDomain.at(brev(2i)) and 1/x of LineDomain.at(brev(2i)): the
    generic coset formula (initial * step^brev(2i)) covers both, because every
    bit-reversed even index lies in the domain's first half."""
    half = _half_odds(log_size - 1)  # CanonicCoset(log_size).circle_domain()
    got = O.fold_twiddles_generic(*half[0], *half[1], log_size, True)
    for i in range(1 << (log_size - 1)):
        y = _circle_domain_at(half, _brev(2 * i, log_size), log_size)[1]
        assert int(got[i]) == pow(y, P - 2, P)
    line = _half_odds(log_size)  # a line domain of 2^log_size points
    got = O.fold_twiddles_generic(*line[0], *line[1], log_size, False)
    for i in range(1 << (log_size - 1)):
        x = _pmul(line[0], _ppow(line[1], _brev(2 * i, log_size)))[0]
        assert int(got[i]) == pow(x, P - 2, P)
