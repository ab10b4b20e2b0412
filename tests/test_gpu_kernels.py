"""GPU parity: twiddle, Merkle, FRI and quotient entry points against the CPU oracle, bit-exact."""
import ctypes as C
import hashlib

import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from gpu_util import P, dev, empty, host, ptr, ptr_array, u32_host, zeros, rand_m31  # noqa: E402
import vortexstark_b200 as V  # noqa: E402


@pytest.fixture(scope="module")
def L():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return V.lib()


# ------------------------------------------------------------------ twiddles
@pytest.mark.parametrize("kind,log_n", [(O.HALF_COSET, 3), (O.HALF_COSET, 12), (O.HALF_ODDS, 9), (O.SUBGROUP, 16)])
def test_coset_points(L, kind, log_n):
    ix, iy, sx, sy = O.coset(kind, log_n)
    n = 1 << log_n
    ox, oy = empty(n), empty(n)
    L.cuda_compute_coset_points(ix, iy, sx, sy, ptr(ox), ptr(oy), n)
    ex, ey = O.coset_points(ix, iy, sx, sy, n)
    assert np.array_equal(host(ox), ex) and np.array_equal(host(oy), ey)


def test_extract_and_squash(L):
    rng = np.random.default_rng(1)
    x = rand_m31(rng, 1024)
    tw, sq, sq2 = empty(512), empty(512), empty(512)
    d = dev(x)
    L.cuda_extract_and_squash(ptr(d), ptr(tw), ptr(sq), 512)
    L.cuda_squash_x(ptr(d), ptr(sq2), 512)
    ev = x[::2].astype(np.uint64)
    exp = (2 * ev * ev % P + P - 1) % P
    assert np.array_equal(host(tw), x[::2])
    assert np.array_equal(host(sq), exp.astype(np.uint32)) and np.array_equal(host(sq2), exp.astype(np.uint32))


@pytest.mark.parametrize("kind,log_n,y", [(O.HALF_COSET, 10, True), (O.HALF_ODDS, 13, False), (O.HALF_COSET, 4, True)])
def test_fold_twiddles(L, kind, log_n, y):
    ix, iy, sx, sy = O.coset(kind, log_n)
    half = 1 << (log_n - 1)
    src, out = empty(half), empty(half)
    L.cuda_compute_fold_twiddle_sources(ix, iy, sx, sy, ptr(src), 1 << log_n, log_n, int(y))
    L.cuda_batch_inverse_m31(ptr(src), ptr(out), half)
    assert np.array_equal(host(out), O.fold_twiddles(kind, log_n, y))


@pytest.mark.parametrize("n", [1, 63, 64, 65, 200, 8192, 100003])
def test_batch_inverse(L, n):
    rng = np.random.default_rng(n)
    x = rand_m31(rng, n)
    x[rng.integers(0, n, max(1, n // 50))] = 0
    if n > 64:
        x[64] = 0  # chunk starting with zero
    out = empty(n)
    L.cuda_batch_inverse_m31(ptr(dev(x)), ptr(out), n)
    assert np.array_equal(host(out), O.batch_inverse(x))


# ------------------------------------------------------------------ Merkle
def tile_roots(leaf_hashes: np.ndarray, tile: int = 1024) -> np.ndarray:
    return np.stack([O.merkle_root_hashes(leaf_hashes[i:i + tile]) for i in range(0, len(leaf_hashes), tile)])


@pytest.mark.parametrize("n_cols", [0, 1, 2, 4, 15, 16, 17, 34])
def test_hash_leaves_capped(L, n_cols):
    rng = np.random.default_rng(n_cols)
    n = 300
    cols = rand_m31(rng, max(n_cols, 1), n)[:n_cols]
    ds = [dev(c) for c in cols] or [dev(np.zeros(n, np.uint32))]
    out = empty(8 * n)
    L.cuda_merkle_hash_leaves(ptr(ptr_array(ds)), ptr(out), n_cols, n)
    exp = O.leaf_hashes_capped(cols if n_cols else np.zeros((0, n), np.uint32))
    assert np.array_equal(host(out).reshape(n, 8), exp)


def test_hash_nodes_and_reduce(L):
    rng = np.random.default_rng(2)
    h = rng.integers(0, 2**32, (1024, 8), dtype=np.uint64).astype(np.uint32)
    out = empty(512 * 8)
    L.cuda_merkle_hash_nodes(ptr(dev(h.reshape(-1))), ptr(out), 512)
    assert np.array_equal(host(out).reshape(512, 8), O.hash_nodes(h))
    for n in [1, 2, 64, 1024]:
        root = empty(8)
        L.cuda_merkle_reduce_to_root(ptr(dev(h[:n].reshape(-1))), ptr(root), n)
        assert np.array_equal(host(root), O.merkle_root_hashes(h[:n]) if n > 1 else h[0])


@pytest.mark.parametrize("log_n", [1, 5, 11, 12])
def test_soa4_small_and_merge(L, log_n):
    rng = np.random.default_rng(log_n)
    n = 1 << log_n
    c = rand_m31(rng, 4, n)
    ds = [dev(x) for x in c]
    root = empty(8)
    L.cuda_merkle_commit_small_soa4(*map(ptr, ds), ptr(root), n)
    assert np.array_equal(host(root), O.merkle_root_soa4(c))
    par = empty(8 * (n // 2))
    L.cuda_merkle_hash_leaves_merge_soa4(*map(ptr, ds), ptr(par), n)
    leaves = np.stack([O.blake2s_words(c[:, i]) for i in range(n)])
    assert np.array_equal(host(par).reshape(-1, 8), O.hash_nodes(leaves))


@pytest.mark.parametrize("log_n", [10, 13])
def test_tiled_soa4_and_generic(L, log_n):
    rng = np.random.default_rng(log_n)
    n = 1 << log_n
    c = rand_m31(rng, 4, n)
    ds = [dev(x) for x in c]
    out = empty(8 * (n // 1024))
    L.cuda_merkle_tiled_soa4(*map(ptr, ds), ptr(out), n)
    leaves = np.stack([O.blake2s_words(c[:, i]) for i in range(n)])
    assert np.array_equal(host(out).reshape(-1, 8), tile_roots(leaves))
    cols = rand_m31(rng, 5, n)
    dcs = [dev(x) for x in cols]
    out2 = empty(8 * (n // 1024))
    L.cuda_merkle_tiled_generic(ptr(ptr_array(dcs)), ptr(out2), 5, n)
    assert np.array_equal(host(out2).reshape(-1, 8), tile_roots(O.leaf_hashes_capped(cols)))


def test_lifted_leaves(L):
    rng = np.random.default_rng(9)
    S = 8
    logs = [8, 8, 6, 7, 8, 5] + [8] * 14  # 20 columns of mixed sizes, > 16 words per leaf
    cols = [rand_m31(rng, 1 << lg) for lg in logs]
    # chunks of <= 16 columns with one log size each, in hashing order
    order = sorted(range(len(cols)), key=lambda i: -logs[i])
    chunks, cur = [], []
    for i in order:
        if cur and (len(cur) == 16 or logs[cur[0]] != logs[i]):
            chunks.append(cur)
            cur = []
        cur.append(i)
    chunks.append(cur)
    sched = np.zeros((len(chunks), 18), np.uint32)
    for k, ch in enumerate(chunks):
        sched[k, : len(ch)] = ch
        sched[k, 16] = len(ch)
        sched[k, 17] = logs[ch[0]]
    ds = [dev(c) for c in cols]
    out = empty(8 << S)
    L.cuda_build_leaves_lifted(ptr(ptr_array(ds)), ptr(dev(sched.reshape(-1))), len(chunks), S, ptr(out), 1 << S)
    flat = [i for ch in chunks for i in ch]
    exp = O.lifted_leaves([cols[i] for i in flat], [logs[i] for i in flat], S)
    assert np.array_equal(host(out).reshape(-1, 8), exp)


@pytest.mark.parametrize("log_n,n_cols", [(0, 3), (4, 34), (10, 34), (11, 7), (14, 34), (21, 2)])
def test_vs_merkle_roots(L, log_n, n_cols):
    rng = np.random.default_rng(log_n * 100 + n_cols)
    n = 1 << log_n
    cols = rand_m31(rng, n_cols, n)
    d = dev(cols.reshape(-1))
    root = empty(8)
    V.check(L.vs_merkle_root_rowpacked(ptr(d), n, n_cols, log_n, ptr(root), None))
    assert np.array_equal(host(root), O.merkle_root_rowpacked(cols, threads=8))
    V.check(L.vs_merkle_root_capped(ptr(d), n, n_cols, log_n, ptr(root), None))
    assert np.array_equal(host(root), O.merkle_root_capped(cols, threads=8))
    if n_cols >= 4:
        V.check(L.vs_merkle_root_soa4(ptr(d), ptr(d) + 4 * n, ptr(d) + 8 * n, ptr(d) + 12 * n, log_n, ptr(root), None))
        assert np.array_equal(host(root), O.merkle_root_soa4(cols[:4], threads=8))


def test_merkle_root_matches_hashlib(L):
    rng = np.random.default_rng(77)
    cols = rand_m31(rng, 34, 16)
    lv = [hashlib.blake2s(cols[:, i].tobytes(), digest_size=32).digest() for i in range(16)]
    while len(lv) > 1:
        lv = [hashlib.blake2s(lv[2 * i] + lv[2 * i + 1], digest_size=32).digest() for i in range(len(lv) // 2)]
    root = empty(8)
    V.check(L.vs_merkle_root_rowpacked(ptr(dev(cols.reshape(-1))), 16, 34, 4, ptr(root), None))
    assert host(root).tobytes() == lv[0]


# ------------------------------------------------------------------ FRI
@pytest.mark.parametrize("log_n", [5, 12, 16])
def test_fold_line(L, log_n):
    rng = np.random.default_rng(log_n)
    n = 1 << log_n
    src = rand_m31(rng, 4, n)
    tw = O.fold_twiddles(O.HALF_ODDS, log_n, False)
    alpha = rand_m31(rng, 4)
    outs = [empty(n // 2) for _ in range(4)]
    L.cuda_fold_line_soa(*[ptr(dev(x)) for x in src], ptr(dev(tw)), *map(ptr, outs), u32_host(alpha), n // 2)
    assert np.array_equal(np.stack([host(o) for o in outs]), O.fold_line(src, tw, alpha))


@pytest.mark.parametrize("log_n", [5, 14])
def test_fold_circle_into_line(L, log_n):
    rng = np.random.default_rng(log_n + 50)
    n = 1 << log_n
    src = rand_m31(rng, 4, n)
    dst0 = rand_m31(rng, 4, n // 2)
    tw = O.fold_twiddles(O.HALF_COSET, log_n, True)
    alpha = rand_m31(rng, 4)
    a2 = rand_m31(rng, 4)
    dds = [dev(x) for x in dst0]
    L.cuda_fold_circle_into_line_soa(*map(ptr, dds), *[ptr(dev(x)) for x in src], ptr(dev(tw)), u32_host(alpha),
                                     u32_host(a2), n // 2)
    assert np.array_equal(np.stack([host(o) for o in dds]), O.fold_circle_into_line(dst0, src, tw, alpha, a2))


@pytest.mark.parametrize("log_n", [4, 11, 16])
def test_vs_fri_fold_commit(L, log_n):
    rng = np.random.default_rng(log_n + 7)
    n = 1 << log_n
    src = rand_m31(rng, 4, n)
    alphas = rand_m31(rng, log_n - 3, 4)
    work = empty(4 * n)
    roots = empty(8 * (log_n - 3))
    last = empty(32)
    V.check(L.vs_fri_fold_commit(ptr(dev(src.reshape(-1))), log_n, u32_host(alphas.reshape(-1)), ptr(work), ptr(roots),
                                 ptr(last), None), "vs_fri_fold_commit")
    er = np.zeros((log_n - 3, 8), np.uint32)
    el = np.zeros((8, 4), np.uint32)
    O.lib().oracle_bench_fri(O.ptr_array(list(src)), log_n, O.ptr(alphas.reshape(-1).copy()), 4, O.ptr(er), O.ptr(el))
    assert np.array_equal(host(roots).reshape(-1, 8), er)
    assert np.array_equal(host(last).reshape(8, 4), el)


# ------------------------------------------------------------------ constraint / quotient
@pytest.mark.parametrize("n", [4, 1000, 1 << 16])
def test_fib_quotient(L, n):
    rng = np.random.default_rng(n)
    t = rand_m31(rng, n)
    alpha = rand_m31(rng, 4)
    outs = [empty(n) for _ in range(4)]
    d = dev(t)
    L.cuda_fibonacci_quotient(ptr(d), *map(ptr, outs), u32_host(alpha), n)
    exp = O.fib_quotient(t, alpha)
    assert np.array_equal(np.stack([host(o) for o in outs]), exp)
    off, cn = n // 3, n - n // 3 - 1
    outs2 = [empty(cn) for _ in range(4)]
    L.cuda_fibonacci_quotient_chunk(ptr(d), *map(ptr, outs2), u32_host(alpha), off, cn, n)
    assert np.array_equal(np.stack([host(o) for o in outs2]), exp[:, off:off + cn])


def test_zero_pad_interleave_fields(L):
    rng = np.random.default_rng(3)
    x = rand_m31(rng, 1000)
    y = rand_m31(rng, 1000)
    out = empty(4096)
    L.cuda_zero_pad(ptr(dev(x)), ptr(out), 1000, 4096)
    exp = np.zeros(4096, np.uint32)
    exp[:1000] = x
    assert np.array_equal(host(out), exp)
    il = empty(2000)
    L.cuda_interleave_u32(ptr(dev(x)), ptr(dev(y)), ptr(il), 1000)
    assert np.array_equal(host(il)[0::2], x) and np.array_equal(host(il)[1::2], y)
    o = empty(1000)
    L.cuda_m31_add(ptr(dev(x)), ptr(dev(y)), ptr(o), 1000)
    assert np.array_equal(host(o), ((x.astype(np.uint64) + y) % P).astype(np.uint32))
    L.cuda_m31_mul(ptr(dev(x)), ptr(dev(y)), ptr(o), 1000)
    assert np.array_equal(host(o), ((x.astype(np.uint64) * y) % P).astype(np.uint32))


def test_accumulate_numerators_and_combine(L):
    rng = np.random.default_rng(11)
    log_n = 10
    n = 1 << log_n
    cols = [rand_m31(rng, n) for _ in range(6)]
    idx = np.array([4, 0, 5, 2], np.uint32)
    b = rand_m31(rng, 4, 4)
    c = rand_m31(rng, 4, 4)
    outs = [empty(n) for _ in range(4)]
    L.cuda_accumulate_numerators(ptr(ptr_array([dev(x) for x in cols])), ptr(dev(idx)), ptr(dev(b.reshape(-1))),
                                 ptr(dev(c.reshape(-1))), 4, n, *map(ptr, outs))
    numer = np.stack([host(o) for o in outs])
    assert np.array_equal(numer, O.accumulate_numerators(cols, idx, b, c, n))
    # combine: two accumulations, one at a smaller (lifted) size
    numer_small = rand_m31(rng, 4, n // 4)
    spx, spy, fla = rand_m31(rng, 2, 4), rand_m31(rng, 2, 4), rand_m31(rng, 2, 4)
    dxs, dys = rand_m31(rng, n), rand_m31(rng, n)
    nums = [numer, numer_small]
    dn = [[dev(x[k]) for k in range(4)] for x in nums]
    outs2 = [empty(n) for _ in range(4)]
    L.cuda_compute_quotients_combine(ptr(dev(spx.reshape(-1))), ptr(dev(spy.reshape(-1))), ptr(dev(fla.reshape(-1))),
                                     *[ptr(ptr_array([dn[j][k] for j in range(2)])) for k in range(4)],
                                     ptr(dev(np.array([log_n, log_n - 2], np.uint32))), 2, ptr(dev(dxs)), ptr(dev(dys)),
                                     log_n, n, *map(ptr, outs2))
    exp = O.quotients_combine(spx, spy, fla, nums, [log_n, log_n - 2], dxs, dys, log_n)
    assert np.array_equal(np.stack([host(o) for o in outs2]), exp)


# ------------------------------------------------------------------ commitment layer
def test_fill_uniform_matches_oracle(L):
    out = empty(100000)
    V.check(L.vs_fill_uniform_m31(ptr(out), 100000, 0x56530001, 12345, None))
    assert np.array_equal(host(out), O.seeded_m31(0x56530001, 100000, offset=12345))


@pytest.mark.parametrize("log_n,n_cols", [(5, 34), (10, 34), (14, 3)])
def test_commit_columns(L, log_n, n_cols):
    n = 1 << log_n
    cols = O.seeded_m31(0x77 + log_n, n_cols * n).reshape(n_cols, n)
    lde = empty(n_cols * 4 * n)
    root = empty(8)
    V.check(L.vs_commit_columns(ptr(dev(cols.reshape(-1))), n_cols, log_n, 2, ptr(lde), ptr(root), None))
    exp_lde = O.stwo_lde_columns(cols, log_n, 2, threads=8)
    assert np.array_equal(host(lde).reshape(n_cols, -1), exp_lde)
    assert np.array_equal(host(root), O.merkle_root_rowpacked(exp_lde, threads=8))


def test_three_tree_commit_16_15_3(L):
    """The reference's three-tree commitment of 34 LDE columns (16 / 15 / 3 columns,
    native leaf) through api.merkle_root_capped on row slices of one LDE tensor."""
    from vortexstark_b200 import api
    log_n = 11
    cols = O.seeded_m31(0x5653, 34 << log_n).reshape(34, -1)
    lde = dev(O.stwo_lde_columns(cols, log_n, 2, threads=8).reshape(34, -1))
    for a, b in ((0, 16), (16, 31), (31, 34)):
        root = zeros(8)
        api.merkle_root_capped(lde[a:b], root)
        torch.cuda.synchronize()
        assert np.array_equal(host(root), O.merkle_root_capped(host(lde[a:b]).reshape(b - a, -1), threads=8))


@pytest.mark.parametrize("log_n", [3, 10, 17])
def test_quotients_combine_zero_denominators(L, log_n):
    """Rows whose denominator vanishes (domain point equal to the sample point's real
    parts) get inverse 0, as the reference's per-row Fermat inverse gives; the
    batched inversion must not let them spoil the other rows of the batch."""
    rng = np.random.default_rng(20 + log_n)
    n = 1 << log_n
    spx, spy, fla = rand_m31(rng, 2, 4), rand_m31(rng, 2, 4), rand_m31(rng, 2, 4)
    spx[0, 1] = 0
    spy[0, 1] = 0
    dxs, dys = rand_m31(rng, n), rand_m31(rng, n)
    hit = rng.choice(n, size=max(1, n // 7), replace=False)
    dxs[hit], dys[hit] = spx[0, 0], spy[0, 0]
    nums = [rand_m31(rng, 4, n), rand_m31(rng, 4, max(2, n // 2))]
    logs = [log_n, max(1, log_n - 1)]
    dn = [[dev(x[k]) for k in range(4)] for x in nums]
    outs = [empty(n) for _ in range(4)]
    L.cuda_compute_quotients_combine(ptr(dev(spx.reshape(-1))), ptr(dev(spy.reshape(-1))), ptr(dev(fla.reshape(-1))),
                                     *[ptr(ptr_array([dn[j][k] for j in range(2)])) for k in range(4)],
                                     ptr(dev(np.array(logs, np.uint32))), 2, ptr(dev(dxs)), ptr(dev(dys)),
                                     log_n, n, *map(ptr, outs))
    exp = O.quotients_combine(spx, spy, fla, nums, logs, dxs, dys, log_n)
    assert np.array_equal(np.stack([host(o) for o in outs]), exp)


@pytest.mark.parametrize("n_batch,n,shift", [(1, 3000, 0), (34, 3000, 0), (300, 3000, 0), (34, 3001, 0),
                                              (7, 1027, 1), (34, 4096, 3)])
def test_accumulate_numerators_many_columns(L, n_batch, n, shift):
    """Column counts past the 3-term fold period, ragged row counts and columns /
    outputs that start off a 16-byte boundary (the 128-bit paths fall back)."""
    rng = np.random.default_rng(n_batch + n)
    cols = [rand_m31(rng, n) for _ in range(8)]
    idx = rng.integers(0, 8, n_batch).astype(np.uint32)
    b, c = rand_m31(rng, n_batch, 4), rand_m31(rng, n_batch, 4)
    c[0] = P - 1
    dcols = [dev(np.concatenate([np.zeros(shift, np.uint32), x])) for x in cols]
    col_ptrs = ptr_array([d[shift:] for d in dcols])
    outs = [empty(n + shift) for _ in range(4)]
    L.cuda_accumulate_numerators(ptr(col_ptrs), ptr(dev(idx)), ptr(dev(b.reshape(-1))), ptr(dev(c.reshape(-1))),
                                 n_batch, n, *[ptr(o[shift:]) for o in outs])
    got = np.stack([host(o)[shift:] for o in outs])
    assert np.array_equal(got, O.accumulate_numerators(cols, idx, b, c, n))
