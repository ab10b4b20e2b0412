"""GPU parity of the device-resident Cairo column-group commitment
(vs_commit_group_cairo; cairo_air/prover.rs:899-1047 with merkle.rs:360-417)
against the CPU oracle, bit-exact: coefficients, blinded BRT-canonic LDE, the
half-coset copy, root and 1024-leaf tile roots."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from gpu_util import P, dev, empty, host, ptr, u32_host  # noqa: E402
import vortexstark_b200 as V  # noqa: E402


@pytest.fixture(scope="module")
def L():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return V.lib()


def run_group(L, cols, log_n, blind=None, stride=None, want=("coeffs", "hc", "tiles")):
    nc, n = cols.shape
    N = n << 2
    stride = stride or n
    buf = np.zeros((nc, stride), np.uint32)
    buf[:, :n] = cols
    d_cols = dev(buf.reshape(-1))
    coeffs = empty(nc * n) if "coeffs" in want else None
    ev_cn = empty(nc * N)
    ev_hc = empty(nc * N) if "hc" in want else None
    root = empty(8)
    tiles = empty(max(1, N // 1024) * 8) if "tiles" in want else None
    rc = L.vs_commit_group_cairo(ptr(d_cols), stride, nc, log_n, u32_host(blind) if blind is not None else None,
                                 ptr(coeffs) if coeffs is not None else None, ptr(ev_cn),
                                 ptr(ev_hc) if ev_hc is not None else None, ptr(root),
                                 ptr(tiles) if tiles is not None else None, None)
    assert rc == 0, L.vs_last_error()
    out = {"eval_cn": host(ev_cn).reshape(nc, N), "root": host(root)}
    if coeffs is not None:
        out["coeffs"] = host(coeffs).reshape(nc, n)
    if ev_hc is not None:
        out["eval_hc"] = host(ev_hc).reshape(nc, N)
    if tiles is not None:
        out["tile_roots"] = host(tiles).reshape(-1, 8)
    return out


def check(got, ref):
    for k, v in got.items():
        assert np.array_equal(v, ref[k]), k


@pytest.mark.parametrize("log_n,nc", [(2, 1), (4, 3), (7, 16), (8, 2), (10, 16), (12, 15), (13, 3)])
def test_group_commit_matches_oracle(L, log_n, nc):
    n = 1 << log_n
    cols = np.stack([O.seeded_m31(0x7200 + 31 * log_n + c, n) for c in range(nc)])
    blind = [(0x5EED * (c + 1) * (log_n + 7)) % P if c % 3 != 1 else 0 for c in range(nc)]
    check(run_group(L, cols, log_n, blind), O.commit_group_cairo(cols, log_n, blind))


@pytest.mark.parametrize("log_n,pad", [(6, 12), (11, 12), (12, 3)])
def test_group_commit_unblinded_and_optional_outputs(L, log_n, pad):
    """No blinding scalars, no coefficient / half-coset / tile-root outputs, padded
    column stride (an odd stride takes the word-by-word permutation)."""
    n, nc = 1 << log_n, 5
    cols = np.stack([O.seeded_m31(0x7300 + c, n) for c in range(nc)])
    got = run_group(L, cols, log_n, None, stride=n + pad, want=())
    check(got, O.commit_group_cairo(cols, log_n))


@pytest.mark.parametrize("log_n", [9, 12])
def test_group_commit_half_coset_copy_with_odd_stride_blinded(L, log_n):
    """Blinded group with an odd input stride: word permutation in, tiled blind + copy out."""
    n, nc = 1 << log_n, 3
    cols = np.stack([O.seeded_m31(0x7350 + c, n) for c in range(nc)])
    blind = [5, 0, P - 2]
    check(run_group(L, cols, log_n, blind, stride=n + 1), O.commit_group_cairo(cols, log_n, blind))


def test_group_commit_three_groups_of_34_columns(L):
    """The reference's 34-column trace split 16 / 15 / 3, every column blinded."""
    log_n = 10
    n = 1 << log_n
    cols = np.stack([O.seeded_m31(0x7400 + c, n) for c in range(34)])
    blind = [(0x1234567 + 7919 * c) % P for c in range(34)]
    for lo, hi in ((0, 16), (16, 31), (31, 34)):
        check(run_group(L, cols[lo:hi], log_n, blind[lo:hi]), O.commit_group_cairo(cols[lo:hi], log_n, blind[lo:hi]))


def test_group_commit_rejects_bad_arguments(L):
    d = empty(64)
    out = empty(256)
    root = empty(8)
    assert L.vs_commit_group_cairo(ptr(d), 16, 17, 4, None, None, ptr(out), None, ptr(root), None, None) != 0
    assert L.vs_commit_group_cairo(ptr(d), 8, 1, 4, None, None, ptr(out), None, ptr(root), None, None) != 0
    assert L.vs_commit_group_cairo(ptr(d), 16, 1, 4, u32_host([P]), None, ptr(out), None, ptr(root), None, None) != 0


# ------------------------------------------------------------------ evaluation at OODS points
@pytest.mark.parametrize("log_len,n_cols,n_points,offset", [(2, 1, 1, 0), (5, 3, 2, 0), (11, 2, 2, 0), (12, 5, 1, 0),
                                                           (16, 3, 2, 0), (14, 2, 2, 1), (13, 1, 1, 2)])
def test_eval_at_oods_points_matches_oracle(L, log_len, n_cols, n_points, offset):
    """Aligned columns of 2^12 words and more take the cp.async ring kernel; an
    offset of 1 or 2 words takes the register kernel."""
    n = 1 << log_len
    cols = [O.seeded_m31(0x7500 + 7 * log_len + c, n) for c in range(n_cols)]
    ch = O.Channel()
    ch.mix_u64(log_len)
    pts = [ch.oods_point() for _ in range(n_points)]
    d = [dev(np.concatenate([np.zeros(offset, np.uint32), c]))[offset:] for c in cols]
    hc = (C.c_uint64 * n_cols)(*[ptr(t) for t in d])
    hp = u32_host(np.concatenate(pts))
    out = (C.c_uint32 * (4 * n_cols * n_points))()
    assert L.vs_eval_at_oods_points(hc, n_cols, log_len, hp, n_points, out, None) == 0, L.vs_last_error()
    got = np.array(out, np.uint32).reshape(n_cols, n_points, 4)
    for c in range(n_cols):
        for p in range(n_points):
            assert np.array_equal(got[c, p], O.eval_at_oods(cols[c], pts[p])), (c, p)


# ------------------------------------------------------------------ OODS + FRI tail
def tail_inputs(log_n, nt, ni, seed):
    from test_oracle_cairo import cairo_tail_inputs
    return cairo_tail_inputs(log_n, nt, ni, seed)


def run_gpu_tail(inp, log_n, offset=0):
    """offset > 0 places every input column that many words past an allocation
    start (word-aligned only), which takes the word-access fallbacks."""
    from vortexstark_b200 import api
    ch = api.Channel()
    ch.mix_digest(inp["root"])
    nt = inp["coeffs"].shape[0]

    def put(a):
        t = dev(np.concatenate([np.zeros(offset, np.uint32), a]))
        return t[offset:] if offset else t
    tc = [put(inp["coeffs"][c]) for c in range(nt)]
    te = [put(inp["evals"][c]) for c in range(nt)]
    ie = [put(inp["inter"][c]) for c in range(inp["inter"].shape[0])]
    qh = [put(inp["q_hc"][k]) for k in range(4)]
    N = 4 << log_n
    oq = [empty(N) for _ in range(4)]
    qcn = [empty(N) for _ in range(4)]
    tiles_q, tiles_o = empty(max(1, N // 1024) * 8), empty(max(1, N // 1024) * 8)
    KEEP = tc + te + ie + qh + oq + qcn  # noqa: F841 (alive until the call returns)
    r = api.cairo_oods_fri(ch, log_n, tc, te, ie, qh, zk_scalars=inp["zk"], quotient_cn=qcn, oods_quotient=oq,
                           quotient_tile_roots=tiles_q, oods_tile_roots=tiles_o)
    r["oods_quotient"] = np.stack([host(t) for t in oq])
    r["quotient_cn"] = np.stack([host(t) for t in qcn])
    r["quotient_tiles"] = host(tiles_q).reshape(-1, 8)
    r["oods_tiles"] = host(tiles_o).reshape(-1, 8)
    return r, ch


@pytest.mark.parametrize("log_n,nt,ni,offset", [(2, 1, 0, 0), (4, 3, 4, 0), (6, 34, 12, 0), (8, 16, 5, 0),
                                                (9, 2, 12, 0), (10, 5, 4, 1), (6, 3, 2, 3)])
def test_cairo_tail_matches_oracle(L, log_n, nt, ni, offset):
    inp = tail_inputs(log_n, nt, ni, 0x7600 + log_n)
    ref_ch = O.Channel()
    ref_ch.mix_digest(inp["root"])
    ref = O.cairo_oods_fri(ref_ch, log_n, inp["coeffs"], inp["zk"], inp["evals"], inp["inter"], inp["q_hc"])
    got, ch = run_gpu_tail(inp, log_n, offset)
    for k in ("quotient_root", "oods_point", "trace_at_z", "trace_at_z_next", "quotient_at_z", "oods_alpha",
              "oods_root", "last_layer", "last_layer_coeffs", "oods_quotient", "quotient_tiles", "oods_tiles"):
        assert np.array_equal(np.array(got[k], np.uint32).reshape(ref[k].shape), ref[k]), k
    if ni:
        assert np.array_equal(np.array(got["interaction_at_z"], np.uint32), ref["interaction_at_z"])
        assert np.array_equal(np.array(got["interaction_at_z_next"], np.uint32), ref["interaction_at_z_next"])
    assert np.array_equal(np.array(got["fri_roots"], np.uint32).reshape(-1, 8), ref["fri_roots"])
    assert np.array_equal(np.array(got["fri_alphas"], np.uint32), ref["fri_alphas"])
    assert np.array_equal(got["quotient_cn"], inp["q_cn"])
    assert ch.state()[0] == ref_ch.state_bytes()


def _hc_index_map_dev(log_n: int, device) -> torch.Tensor:
    n = 1 << log_n
    k = torch.arange(n, dtype=torch.int64, device=device)
    cn = torch.where(k % 2 == 0, k // 2, n - 1 - k // 2)
    rev = torch.zeros_like(cn)
    for b in range(log_n):
        rev |= ((cn >> b) & 1) << (log_n - 1 - b)
    return rev


@pytest.mark.parametrize("log_n", [16, 20])
def test_cairo_tail_full_width_is_low_degree(L, log_n):
    """34 trace columns committed 16 / 15 / 3 with blinding, 12 interaction columns,
    an AIR quotient of degree < 2n: at sizes the oracle cannot follow, the DEEP
    quotient's last FRI layer must still have line degree < 4, and the quotient's
    BRT-canonic copy must be the inverse permutation of its input."""
    from vortexstark_b200 import api
    n, N = 1 << log_n, 4 << log_n
    devc = torch.device("cuda")
    cols = api.fill_uniform_m31(torch.empty((34, n), dtype=torch.int32, device=devc), seed=0x7700 + log_n)
    blind = [(0x2468ACE + 7919 * c) % P for c in range(34)]
    coeffs = torch.empty((34, n), dtype=torch.int32, device=devc)
    evals_hc = torch.empty((34, N), dtype=torch.int32, device=devc)
    evals, ch = [], api.Channel()
    for lo, hi in ((0, 16), (16, 31), (31, 34)):
        ev, root = api.commit_group_cairo(cols[lo:hi].contiguous(), log_n, blind[lo:hi], coeffs=coeffs[lo:hi],
                                          eval_hc=evals_hc[lo:hi])
        evals.append(ev)
        ch.mix_digest(host(root))
    evals = torch.cat(evals)
    pos = _hc_index_map_dev(log_n + 2, devc)
    assert torch.equal(evals_hc, evals[:, pos])  # the half-coset copy is the inverse permutation
    # decommit the first group at 80 queries and their next rows, convert the paths
    # to stwo's hash witness and rebuild the group's root from it
    rng = np.random.default_rng(log_n)
    qs = [int(x) for x in rng.integers(0, N, 80)]
    idx = sorted(set(qs + [_canonic_next(q, log_n + 2) for q in qs]))
    tiles0 = empty(max(1, N // 1024) * 8)
    ev0, root0 = api.commit_group_cairo(cols[0:16].contiguous(), log_n, blind[0:16], tile_roots=tiles0)
    vals, paths = _gpu_paths(L, 0, list(ev0), log_n + 2, tiles0, idx)
    flat = paths.reshape(-1)
    wit = (C.c_uint32 * flat.size)()
    m = C.c_uint32()
    assert L.vs_stwo_hash_witness((C.c_uint64 * len(idx))(*idx), len(idx), (C.c_uint32 * flat.size)(*flat.tolist()),
                                  log_n + 2, wit, len(idx) * (log_n + 2), C.byref(m)) == 0
    rebuilt = (C.c_uint32 * 8)()
    assert L.vs_stwo_root_from_witness(log_n + 2, (C.c_uint64 * len(idx))(*idx), len(idx),
                                       (C.c_uint32 * vals.size)(*vals.reshape(-1).tolist()), 16, wit, m.value,
                                       rebuilt) == 0, L.vs_last_error()
    assert np.array_equal(np.array(rebuilt, np.uint32), host(root0))
    assert m.value < len(idx) * (log_n + 2)
    inter_src = api.fill_uniform_m31(torch.empty((12, n), dtype=torch.int32, device=devc), seed=0x7800 + log_n)
    inter = api.lde_stwo(inter_src, log_n, 2)
    q_src = api.fill_uniform_m31(torch.empty((4, 2 * n), dtype=torch.int32, device=devc), seed=0x7900 + log_n)
    q_cn = api.lde_stwo(q_src, log_n + 1, 1)
    q_hc = q_cn[:, _hc_index_map_dev(log_n + 2, devc)].contiguous()
    out_cn = [empty(N) for _ in range(4)]
    torch.cuda.synchronize()
    r = api.cairo_oods_fri(ch, log_n, list(coeffs), list(evals), list(inter), list(q_hc), zk_scalars=blind,
                           quotient_cn=out_cn)
    nat = np.array(r["last_layer_coeffs"], np.uint32)[[0, 4, 2, 6, 1, 5, 3, 7]]
    assert not nat[4:].any() and nat[:4].any()
    for k in range(4):
        assert torch.equal(out_cn[k], q_cn[k])
    assert len(r["fri_roots"]) == log_n - 2


# ------------------------------------------------------------------ decommitment of tile-rooted trees
def _gpu_paths(L, kind, cols_dev, log_n, tiles_dev, idx):
    nc = len(cols_dev)
    hc = (C.c_uint64 * nc)(*[ptr(t) for t in cols_dev])
    ix = (C.c_uint64 * len(idx))(*[int(i) for i in idx])
    vals = (C.c_uint32 * (len(idx) * nc))()
    paths = (C.c_uint32 * max(1, len(idx) * log_n * 8))()
    rc = L.vs_tile_tree_paths(kind, hc, nc, log_n, ptr(tiles_dev), ix, len(idx), vals, paths, None)
    assert rc == 0, L.vs_last_error()
    return (np.array(vals, np.uint32).reshape(len(idx), nc),
            np.array(paths, np.uint32)[: len(idx) * log_n * 8].reshape(len(idx), log_n, 8))


def _canonic_next(qi, log_eval):
    """prover.rs:170-179: the BRT-canonic index one trace step (4 rows) on."""
    n = 1 << log_eval
    cn = int(format(qi, f"0{log_eval}b")[::-1], 2)
    k = 2 * cn if cn < n // 2 else 2 * (n - 1 - cn) + 1
    kn = (k + 4) % n
    cnn = kn // 2 if kn % 2 == 0 else n - 1 - kn // 2
    return int(format(cnn, f"0{log_eval}b")[::-1], 2)


@pytest.mark.parametrize("log_n,nc", [(4, 3), (8, 16), (9, 15), (11, 3)])
def test_trace_group_decommitment_matches_oracle(L, log_n, nc):
    """Trace-group queries at q and at the next trace row (prover.rs:2510-2560)."""
    n, N = 1 << log_n, 4 << log_n
    cols = np.stack([O.seeded_m31(0x7B00 + c, n) for c in range(nc)])
    blind = [(77 + 13 * c) % P for c in range(nc)]
    d_cols = dev(cols.reshape(-1))
    ev = empty(nc * N)
    root = empty(8)
    tiles = empty(max(1, N // 1024) * 8)
    assert L.vs_commit_group_cairo(ptr(d_cols), n, nc, log_n, u32_host(blind), None, ptr(ev), None, ptr(root),
                                   ptr(tiles), None) == 0, L.vs_last_error()
    ref = O.commit_group_cairo(cols, log_n, blind)
    rng = np.random.default_rng(log_n)
    q = [0, N - 1] + [int(x) for x in rng.integers(0, N, 14)] + [3, 3]
    idx = q + [_canonic_next(i, log_n + 2) for i in q]
    cols_dev = [ev[c * N:(c + 1) * N] for c in range(nc)]
    vals, paths = _gpu_paths(L, 0, cols_dev, log_n + 2, tiles, idx)
    assert np.array_equal(vals, ref["eval_cn"][:, idx].T)
    assert np.array_equal(paths, O.tree_paths(0, ref["eval_cn"], idx))


@pytest.mark.parametrize("log_n", [4, 9])
def test_quotient_decommitment_matches_oracle(L, log_n):
    """SoA4 trees of the tail (AIR quotient and DEEP quotient): queries and their fold siblings."""
    inp = tail_inputs(log_n, 3, 4, 0x7C00 + log_n)
    got, _ = run_gpu_tail(inp, log_n)
    N = 4 << log_n
    rng = np.random.default_rng(7)
    q = [int(x) for x in rng.integers(0, N, 20)]
    idx = q + [i ^ 1 for i in q]
    for key, tkey in (("quotient_cn", "quotient_tiles"), ("oods_quotient", "oods_tiles")):
        cols = got[key]
        vals, paths = _gpu_paths(L, 1, [dev(cols[k]) for k in range(4)], log_n + 2, dev(got[tkey].reshape(-1)), idx)
        assert np.array_equal(vals, cols[:, idx].T), key
        assert np.array_equal(paths, O.tree_paths(1, cols, idx)), key


def test_tile_tree_paths_rejects_bad_arguments(L):
    t = empty(64)
    hc = (C.c_uint64 * 4)(*[ptr(t)] * 4)
    ix = (C.c_uint64 * 1)(64)
    out = (C.c_uint32 * 64)()
    assert L.vs_tile_tree_paths(1, hc, 3, 6, ptr(t), ix, 1, out, out, None) != 0   # SoA4 needs 4 columns
    assert L.vs_tile_tree_paths(0, hc, 4, 6, ptr(t), ix, 1, out, out, None) != 0   # index out of range
    assert L.vs_tile_tree_paths(7, hc, 4, 6, ptr(t), ix, 0, out, out, None) != 0   # unknown leaf


@pytest.mark.parametrize("split", [0, 5])
def test_group_commit_tile_roots_with_split(L, split):
    """2^20 evaluation rows: the tile roots go through 2^split subtree roots per tile
    when a split is set; roots and tile roots stay the oracle's."""
    from vortexstark_b200 import api
    log_n, nc = 18, 2
    n = 1 << log_n
    cols = np.stack([O.seeded_m31(0x7300 + c, n) for c in range(nc)])
    blind = [12345, 0]
    api.set_merkle_split(split)
    try:
        got = run_group(L, cols, log_n, blind)
    finally:
        api.set_merkle_split(0)
    check(got, O.commit_group_cairo(cols, log_n, blind))
