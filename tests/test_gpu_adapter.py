"""GPU parity of the stwo Backend adapter drop-ins (cuda_gather_u32,
cuda_gather_u256, cuda_barycentric_eval, cuda_accumulate_lift, cuda_pack_leaves)
against the CPU oracle, bit for bit, called through the C ABI. Each case runs with
16-byte-aligned buffers and with buffers one word off (the word-access variants)."""
import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from gpu_util import P, empty, host, ptr, ptr_array, rand_m31, zeros  # noqa: E402
import vortexstark_b200 as V  # noqa: E402


@pytest.fixture(scope="module")
def L():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return V.lib()


def placed(a, off):
    """Device copy of `a` starting `off` words into a fresh allocation: (pointer, view)."""
    a = np.ascontiguousarray(a, np.uint32).ravel()
    t = torch.zeros(a.size + off + 4, dtype=torch.int32, device="cuda")
    t[off:off + a.size] = torch.from_numpy(a.view(np.int32).copy()).cuda()
    return ptr(t) + 4 * off, t[off:off + a.size]


@pytest.mark.parametrize("n", [0, 1, 1000, 1 << 20])
def test_gather_u32(L, n):
    rng = np.random.default_rng(n + 1)
    src = rand_m31(rng, 4096)
    idx = rng.integers(0, 4096, size=n).astype(np.uint32)
    ps, _ = placed(src, 0)
    pi, _ = placed(idx, 0)
    pd, out = placed(np.zeros(n, np.uint32), 0)
    L.cuda_gather_u32(ps, pi, pd, n)
    assert np.array_equal(host(out), O.gather_u32(src, idx))


@pytest.mark.parametrize("n,off", [(1, 0), (1000, 0), (1 << 18, 0), (1000, 1), (777, 3)])
def test_gather_u256(L, n, off):
    rng = np.random.default_rng(n + off)
    src = rand_m31(rng, 8 * 5000)
    idx = rng.integers(0, 5000, size=n).astype(np.uint32)
    ps, _ = placed(src, off)
    pi, _ = placed(idx, 0)
    pd, out = placed(np.zeros(8 * n, np.uint32), off)
    L.cuda_gather_u256(ps, pi, pd, n)
    assert np.array_equal(host(out), O.gather_u256(src, idx))


@pytest.mark.parametrize("n,n_blocks,off", [(1, 1, 0), (255, 1, 0), (1000, 4, 0), (70000, 256, 0), (300, 256, 0),
                                            (1 << 22, 256, 0), (1 << 22, 148, 1), (99999, 7, 2), (5000, 3, 1)])
def test_barycentric_eval(L, n, n_blocks, off):
    rng = np.random.default_rng(n * 3 + n_blocks)
    e = rand_m31(rng, n)
    w = rand_m31(rng, 4 * n)
    pe, _ = placed(e, 0)
    pw, _ = placed(w, off)
    out = zeros(4 * n_blocks) - 1  # every partial must be written
    L.cuda_barycentric_eval(pe, pw, n, ptr(out), n_blocks)
    got = host(out).reshape(n_blocks, 4)
    exp = O.barycentric_partials(e, w, n_blocks)
    assert np.array_equal(got, exp)
    # the value the adapter returns: the partial sums added mod p
    total = [int(v) for v in (exp.astype(np.uint64).sum(axis=0) % P)]
    assert total == [int(v) for v in (got.astype(np.uint64).sum(axis=0) % P)]


@pytest.mark.parametrize("log_col,log_curr,off", [(1, 1, 0), (4, 1, 0), (10, 10, 0), (20, 13, 0), (16, 2, 1),
                                                  (12, 11, 3)])
def test_accumulate_lift(L, log_col, log_curr, off):
    rng = np.random.default_rng(log_col * 64 + log_curr)
    col = rand_m31(rng, 4 << log_col)
    curr = rand_m31(rng, 4 << log_curr)
    pc, view = placed(col, off)
    pu, _ = placed(curr, 0)
    L.cuda_accumulate_lift(pc, pu, 1 << log_col, log_col - log_curr)
    assert np.array_equal(host(view), O.accumulate_lift(col, curr, log_col - log_curr))


def test_accumulate_lift_chain(L):
    """The adapter's lift_and_accumulate loop (accumulation_ops.rs:50-85): columns of
    ascending size, each lifted onto the next, starting from a zero column of 2."""
    rng = np.random.default_rng(5)
    sizes = [1, 3, 3, 6, 9]
    cols = [rand_m31(rng, 4 << s) for s in sizes]
    dev_cols = [placed(c, 0) for c in cols]
    curr_p, _ = placed(np.zeros(8, np.uint32), 0)
    exp_curr, curr_log = np.zeros(8, np.uint32), 1
    for (pc, view), c, s in zip(dev_cols, cols, sizes):
        L.cuda_accumulate_lift(pc, curr_p, 1 << s, s - curr_log)
        exp_curr = O.accumulate_lift(c, exp_curr, s - curr_log)
        curr_p, curr_log = pc, s
        assert np.array_equal(host(view), exp_curr)


@pytest.mark.parametrize("n,off", [(16, 0), (4096, 0), (1 << 20, 0), (40, 0), (7, 0), (4096, 1), (1000, 2)])
def test_pack_leaves(L, n, off):
    rng = np.random.default_rng(n + 7 * off)
    cols = rand_m31(rng, 4, n)
    ins = [placed(cols[c], off)[1] for c in range(4)]
    g = (n + 15) // 16
    outs = [zeros(g) for _ in range(64)]
    L.cuda_pack_leaves(ptr(ptr_array(ins)), ptr(ptr_array(outs)), n)
    got = np.stack([host(o) for o in outs])
    assert np.array_equal(got, O.pack_leaves(cols))


# ---- domain helpers behind the adapter (fri_ops.rs:50-56,100-106; quotient_ops.rs:135-140)
@pytest.mark.parametrize("log_size", [1, 2, 4, 9, 13, 16, 20])
def test_canonic_domain_points(L, log_size):
    n = 1 << log_size
    xs, ys = zeros(n), zeros(n)
    V.check(L.vs_canonic_domain_points(log_size, ptr(xs), ptr(ys), None), "vs_canonic_domain_points")
    ex, ey = O.canonic_domain_points(log_size)
    assert np.array_equal(host(xs), ex) and np.array_equal(host(ys), ey)


def _coset(kind, log_size):
    c = O.coset(kind, log_size)
    return c[0], c[1], c[2], c[3]


@pytest.mark.parametrize("log_size", [1, 4, 7, 12, 16, 20])
@pytest.mark.parametrize("is_line", [0, 1])
def test_fold_twiddles_stwo(L, log_size, is_line):
    """Circle: the half coset of CanonicCoset(log_size)'s domain (half_odds(log_size-1));
    line: the coset half_odds(log_size) of a 2^log_size-point line domain; and, for
    both, the coset half_coset(log_size) (whose small sizes hold points with a zero
    coordinate, which map to 0 on both sides)."""
    half = 1 << (log_size - 1)
    cosets = [_coset(O.HALF_ODDS, log_size - 1) if not is_line else _coset(O.HALF_ODDS, log_size)]
    hc = _coset(O.HALF_COSET, log_size)
    cosets.append((hc[0], hc[1], hc[2], hc[3]))
    for ix, iy, sx, sy in cosets:
        out = zeros(half)
        V.check(L.vs_fold_twiddles_stwo(is_line, ix, iy, sx, sy, log_size, ptr(out), None), "vs_fold_twiddles_stwo")
        exp = O.fold_twiddles_generic(ix, iy, sx, sy, log_size, not is_line)
        assert np.array_equal(host(out), exp)


def test_domain_helpers_reject_bad_arguments(L):
    out = zeros(8)
    assert L.vs_fold_twiddles_stwo(0, P, 0, 1, 0, 4, ptr(out), None) == 1
    assert L.vs_fold_twiddles_stwo(0, 1, 0, 1, 0, 0, ptr(out), None) == 1
    assert L.vs_canonic_domain_points(31, ptr(out), ptr(out), None) == 1
