"""Pins the CPU oracle to the reference's own CUDA kernels.

oracle/_ref/libvortex_ref.so is built from the reference's kernel sources by
oracle/build_ref.sh. Here those kernels run on the GPU and their outputs must
equal the oracle's, bit for bit. The reference's host orchestration (Rust) is
restated in Python where needed (circle.rs:277-340 twiddle assembly).

Launch shapes were checked against the reference sources: every kernel here is
given sizes at which all threads of a warp that issue __shfl_sync are live
(stwo NTT: n >= 128), and shared-memory tree kernels are called within their
documented limits (<= 1024 nodes, <= 2048 SoA4 leaves).
"""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from gpu_util import P, dev, empty, host, ptr, ptr_array, u32_host, zeros, rand_m31  # noqa: E402


@pytest.fixture(scope="module")
def R():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not O.REF_SO.exists():
        pytest.skip("reference kernels not built (oracle/build_ref.sh)")
    return C.CDLL(str(O.REF_SO))


def sync():
    torch.cuda.synchronize()


def ref_native_twiddles(R, log_n):
    """circle.rs:277-340 (compute_twiddles) + compute_itwiddles, with the reference kernels."""
    ix, iy, sx, sy = O.coset(O.HALF_COSET, log_n)
    n = 1 << log_n
    dx, dy = empty(n), empty(n)
    R.cuda_compute_coset_points(C.c_uint32(ix), C.c_uint32(iy), C.c_uint32(sx), C.c_uint32(sy), C.c_void_p(ptr(dx)),
                                C.c_void_p(ptr(dy)), C.c_uint32(n))
    line = zeros(n - 1)
    cur, cur_n, off = dx, n, 0
    for _ in range(log_n - 1):
        ls = cur_n // 2
        sq = empty(ls)
        R.cuda_extract_and_squash(C.c_void_p(ptr(cur)), C.c_void_p(ptr(line) + 4 * off), C.c_void_p(ptr(sq)), C.c_uint32(ls))
        off += ls
        cur, cur_n = sq, ls
    iline, icirc = empty(n - 1), empty(n // 2)
    R.cuda_batch_inverse_m31(C.c_void_p(ptr(line)), C.c_void_p(ptr(iline)), C.c_uint32(n - 1))
    circ = dy[: n // 2].clone()
    R.cuda_batch_inverse_m31(C.c_void_p(ptr(circ)), C.c_void_p(ptr(icirc)), C.c_uint32(n // 2))
    sync()
    return host(line), host(circ), host(iline), host(icirc)


@pytest.mark.parametrize("log_n", [4, 7, 12, 16])
def test_native_twiddles_and_ntt(R, log_n):
    line, circ, iline, icirc = ref_native_twiddles(R, log_n)
    tw = O.native_twiddles(log_n)
    assert np.array_equal(line, tw["line"]) and np.array_equal(circ, tw["circle"])
    assert np.array_equal(iline, tw["iline"]) and np.array_equal(icirc, tw["icircle"])
    rng = np.random.default_rng(log_n)
    x = rand_m31(rng, 1 << log_n)
    d = dev(x)
    offs = u32_host(tw["offsets"])
    R.cuda_circle_ntt_evaluate(C.c_void_p(ptr(d)), C.c_void_p(ptr(dev(line))), C.c_void_p(ptr(dev(circ))), offs, offs,
                               C.c_uint32(log_n - 1), C.c_uint32(1 << log_n))
    ev = host(d)
    assert np.array_equal(ev, O.native_evaluate(x, log_n))
    R.cuda_circle_ntt_interpolate(C.c_void_p(ptr(d)), C.c_void_p(ptr(dev(iline))), C.c_void_p(ptr(dev(icirc))), offs,
                                  offs, C.c_uint32(log_n - 1), C.c_uint32(1 << log_n))
    assert np.array_equal(host(d), x)


@pytest.mark.parametrize("log_n", [7, 10, 12, 15])
def test_stwo_ntt(R, log_n):
    fwd, inv = O.stwo_twiddles(log_n)
    rng = np.random.default_rng(log_n + 1)
    x = rand_m31(rng, 1 << log_n)
    d = dev(x)
    R.cuda_stwo_ntt_evaluate(C.c_void_p(ptr(d)), C.c_void_p(ptr(dev(fwd))), C.c_uint32(1 << log_n))
    ev = host(d)
    assert np.array_equal(ev, O.stwo_evaluate(x, log_n))
    R.cuda_stwo_ntt_interpolate(C.c_void_p(ptr(d)), C.c_void_p(ptr(dev(inv))), C.c_uint32(1 << log_n))
    assert np.array_equal(host(d), O.stwo_interpolate(ev, log_n))


@pytest.mark.parametrize("kind,log_n,y", [(O.HALF_COSET, 9, 1), (O.HALF_ODDS, 11, 0)])
def test_fold_twiddles(R, kind, log_n, y):
    ix, iy, sx, sy = O.coset(kind, log_n)
    half = 1 << (log_n - 1)
    src, out = empty(half), empty(half)
    R.cuda_compute_fold_twiddle_sources(*(C.c_uint32(v) for v in (ix, iy, sx, sy)), C.c_void_p(ptr(src)),
                                        C.c_uint32(1 << log_n), C.c_uint32(log_n), C.c_int(y))
    R.cuda_batch_inverse_m31(C.c_void_p(ptr(src)), C.c_void_p(ptr(out)), C.c_uint32(half))
    assert np.array_equal(host(out), O.fold_twiddles(kind, log_n, bool(y)))


def test_batch_inverse_quirks(R):
    rng = np.random.default_rng(3)
    x = rand_m31(rng, 1000)
    x[[3, 64, 130, 999]] = 0
    out = empty(1000)
    R.cuda_batch_inverse_m31(C.c_void_p(ptr(dev(x))), C.c_void_p(ptr(out)), C.c_uint32(1000))
    assert np.array_equal(host(out), O.batch_inverse(x))


@pytest.mark.parametrize("n_cols", [1, 4, 16, 20])
def test_merkle_leaves_nodes(R, n_cols):
    rng = np.random.default_rng(n_cols)
    n = 512
    cols = rand_m31(rng, n_cols, n)
    ds = [dev(c) for c in cols]
    out = empty(8 * n)
    R.cuda_merkle_hash_leaves(C.c_void_p(ptr(ptr_array(ds))), C.c_void_p(ptr(out)), C.c_uint32(n_cols), C.c_uint32(n))
    leaves = host(out).reshape(n, 8)
    assert np.array_equal(leaves, O.leaf_hashes_capped(cols))
    par = empty(8 * n // 2)
    R.cuda_merkle_hash_nodes(C.c_void_p(ptr(dev(leaves.reshape(-1)))), C.c_void_p(ptr(par)), C.c_uint32(n // 2))
    assert np.array_equal(host(par).reshape(-1, 8), O.hash_nodes(leaves))
    root = empty(8)
    R.cuda_merkle_reduce_to_root(C.c_void_p(ptr(dev(leaves.reshape(-1)))), C.c_void_p(ptr(root)), C.c_uint32(n))
    assert np.array_equal(host(root), O.merkle_root_capped(cols))


@pytest.mark.parametrize("log_n", [11, 12])
def test_merkle_soa4(R, log_n):
    rng = np.random.default_rng(log_n)
    n = 1 << log_n
    c = rand_m31(rng, 4, n)
    ds = [C.c_void_p(ptr(dev(x))) for x in c]
    tiles = empty(8 * (n // 1024))
    R.cuda_merkle_tiled_soa4(*ds, C.c_void_p(ptr(tiles)), C.c_uint32(n))
    leaves = np.stack([O.blake2s_words(c[:, i]) for i in range(n)])
    exp_tiles = np.stack([O.merkle_root_hashes(leaves[i:i + 1024]) for i in range(0, n, 1024)])
    assert np.array_equal(host(tiles).reshape(-1, 8), exp_tiles)
    if n <= 2048:
        root = empty(8)
        R.cuda_merkle_commit_small_soa4(*ds, C.c_void_p(ptr(root)), C.c_uint32(n))
        assert np.array_equal(host(root), O.merkle_root_soa4(c))


def test_lifted_leaves(R):
    rng = np.random.default_rng(5)
    S = 7
    logs = [7] * 17 + [6, 6, 5]
    cols = [rand_m31(rng, 1 << lg) for lg in logs]
    chunks = [list(range(0, 16)), [16], [17, 18], [19]]
    sched = np.zeros((4, 18), np.uint32)
    for k, ch in enumerate(chunks):
        sched[k, : len(ch)] = ch
        sched[k, 16] = len(ch)
        sched[k, 17] = logs[ch[0]]
    out = empty(8 << S)
    R.cuda_build_leaves_lifted(C.c_void_p(ptr(ptr_array([dev(c) for c in cols]))), C.c_void_p(ptr(dev(sched.reshape(-1)))),
                               C.c_uint32(4), C.c_uint32(S), C.c_void_p(ptr(out)), C.c_uint32(1 << S))
    assert np.array_equal(host(out).reshape(-1, 8), O.lifted_leaves(cols, logs, S))


def test_folds(R):
    rng = np.random.default_rng(8)
    log_n = 10
    n = 1 << log_n
    src = rand_m31(rng, 4, n)
    alpha = rand_m31(rng, 4)
    tw = O.fold_twiddles(O.HALF_ODDS, log_n, False)
    outs = [empty(n // 2) for _ in range(4)]
    R.cuda_fold_line_soa(*[C.c_void_p(ptr(dev(x))) for x in src], C.c_void_p(ptr(dev(tw))),
                         *[C.c_void_p(ptr(o)) for o in outs], u32_host(alpha), C.c_uint32(n // 2))
    assert np.array_equal(np.stack([host(o) for o in outs]), O.fold_line(src, tw, alpha))
    dst0 = rand_m31(rng, 4, n // 2)
    a2 = rand_m31(rng, 4)
    twc = O.fold_twiddles(O.HALF_COSET, log_n, True)
    dds = [dev(x) for x in dst0]
    R.cuda_fold_circle_into_line_soa(*[C.c_void_p(ptr(d)) for d in dds], *[C.c_void_p(ptr(dev(x))) for x in src],
                                     C.c_void_p(ptr(dev(twc))), u32_host(alpha), u32_host(a2), C.c_uint32(n // 2))
    assert np.array_equal(np.stack([host(d) for d in dds]), O.fold_circle_into_line(dst0, src, twc, alpha, a2))


def test_quotients(R):
    rng = np.random.default_rng(12)
    n = 1 << 12
    t = rand_m31(rng, n)
    alpha = rand_m31(rng, 4)
    outs = [empty(n) for _ in range(4)]
    R.cuda_fibonacci_quotient(C.c_void_p(ptr(dev(t))), *[C.c_void_p(ptr(o)) for o in outs], u32_host(alpha), C.c_uint32(n))
    assert np.array_equal(np.stack([host(o) for o in outs]), O.fib_quotient(t, alpha))
    cols = [rand_m31(rng, n) for _ in range(3)]
    idx = np.array([2, 0], np.uint32)
    b, c = rand_m31(rng, 2, 4), rand_m31(rng, 2, 4)
    outs = [empty(n) for _ in range(4)]
    R.cuda_accumulate_numerators(C.c_void_p(ptr(ptr_array([dev(x) for x in cols]))), C.c_void_p(ptr(dev(idx))),
                                 C.c_void_p(ptr(dev(b.reshape(-1)))), C.c_void_p(ptr(dev(c.reshape(-1)))), C.c_uint32(2),
                                 C.c_uint32(n), *[C.c_void_p(ptr(o)) for o in outs])
    numer = np.stack([host(o) for o in outs])
    assert np.array_equal(numer, O.accumulate_numerators(cols, idx, b, c, n))
    spx, spy, fla = rand_m31(rng, 1, 4), rand_m31(rng, 1, 4), rand_m31(rng, 1, 4)
    dxs, dys = rand_m31(rng, n), rand_m31(rng, n)
    outs2 = [empty(n) for _ in range(4)]
    dn = [dev(numer[k]) for k in range(4)]
    R.cuda_compute_quotients_combine(C.c_void_p(ptr(dev(spx.reshape(-1)))), C.c_void_p(ptr(dev(spy.reshape(-1)))),
                                     C.c_void_p(ptr(dev(fla.reshape(-1)))),
                                     *[C.c_void_p(ptr(ptr_array([dn[k]]))) for k in range(4)],
                                     C.c_void_p(ptr(dev(np.array([12], np.uint32)))), C.c_uint32(1),
                                     C.c_void_p(ptr(dev(dxs))), C.c_void_p(ptr(dev(dys))), C.c_uint32(12), C.c_uint32(n),
                                     *[C.c_void_p(ptr(o)) for o in outs2])
    exp = O.quotients_combine(spx, spy, fla, [numer], [12], dxs, dys, 12)
    assert np.array_equal(np.stack([host(o) for o in outs2]), exp)


def test_bit_reverse(R):
    rng = np.random.default_rng(1)
    x = rand_m31(rng, 1 << 12)
    d = dev(x)
    R.cuda_bit_reverse_m31(C.c_void_p(ptr(d)), C.c_uint32(12))
    assert np.array_equal(host(d), O.bit_reverse(x, 12))


def test_adapter_kernels(R):
    """cuda/gather.cu, barycentric_eval.cu, accumulate_lift.cu, pack_leaves.cu against the oracle."""
    rng = np.random.default_rng(3)
    src = rand_m31(rng, 8 * 600)
    idx = rng.integers(0, 600, size=500).astype(np.uint32)
    out = zeros(500)
    R.cuda_gather_u32(C.c_void_p(ptr(dev(src))), C.c_void_p(ptr(dev(idx))), C.c_void_p(ptr(out)), C.c_uint32(500))
    assert np.array_equal(host(out), O.gather_u32(src, idx))
    out8 = zeros(8 * 500)
    R.cuda_gather_u256(C.c_void_p(ptr(dev(src))), C.c_void_p(ptr(dev(idx))), C.c_void_p(ptr(out8)), C.c_uint32(500))
    assert np.array_equal(host(out8), O.gather_u256(src, idx))

    for n, n_blocks in [(1000, 4), (70000, 256), (300, 3)]:
        e = rand_m31(rng, n)
        w = rand_m31(rng, 4 * n)
        part = zeros(4 * n_blocks)
        R.cuda_barycentric_eval(C.c_void_p(ptr(dev(e))), C.c_void_p(ptr(dev(w))), C.c_uint32(n), C.c_void_p(ptr(part)),
                                C.c_uint32(n_blocks))
        assert np.array_equal(host(part).reshape(n_blocks, 4), O.barycentric_partials(e, w, n_blocks))

    for log_col, log_curr in [(1, 1), (8, 3), (12, 11)]:
        col = rand_m31(rng, 4 << log_col)
        curr = rand_m31(rng, 4 << log_curr)
        d = dev(col)
        R.cuda_accumulate_lift(C.c_void_p(ptr(d)), C.c_void_p(ptr(dev(curr))), C.c_uint32(1 << log_col),
                               C.c_uint32(log_col - log_curr))
        assert np.array_equal(host(d), O.accumulate_lift(col, curr, log_col - log_curr))

    for n in (4096, 40):
        cols = rand_m31(rng, 4, n)
        outs = [zeros((n + 15) // 16) for _ in range(64)]
        R.cuda_pack_leaves(C.c_void_p(ptr(ptr_array([dev(c) for c in cols]))), C.c_void_p(ptr(ptr_array(outs))),
                           C.c_uint32(n))
        sync()
        assert np.array_equal(np.stack([host(o) for o in outs]), O.pack_leaves(cols))
