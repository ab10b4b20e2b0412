"""The oracle's Cairo column-group commitment (cairo_air/prover.rs:899-1047):
half-coset natural order -> BRT-canonic, stwo LDE x4, ZK blinding with Z_H,
half-coset copy, capped-leaf root and 1024-leaf tile roots (merkle.rs:360-417).
Checked against properties that hold independently of the implementation."""
import numpy as np
import pytest

import oracle_lib as O

P = 0x7FFFFFFF


def hc_to_cn_brt(k: int, log_n: int) -> int:
    n = 1 << log_n
    cn = k // 2 if k % 2 == 0 else n - 1 - k // 2
    return int(format(cn, f"0{log_n}b")[::-1], 2)


@pytest.mark.parametrize("log_n", [3, 6])
def test_zh_vanishes_on_trace_domain(log_n):
    """circle.rs:241-254: Z_H is zero at every point of half_coset(log_n)."""
    n = 1 << log_n
    ix, iy, sx, sy = O.coset(O.HALF_COSET, log_n)
    xs, ys = O.coset_points(ix, iy, sx, sy, n)
    assert all(O.coset_vanishing_half_coset(log_n, int(x), int(y)) == 0 for x, y in zip(xs, ys))
    # ... and not on the next coset over (the points of half_odds(log_n))
    ix, iy, sx, sy = O.coset(O.HALF_ODDS, log_n)
    xs, ys = O.coset_points(ix, iy, sx, sy, n)
    assert all(O.coset_vanishing_half_coset(log_n, int(x), int(y)) != 0 for x, y in zip(xs, ys))


@pytest.mark.parametrize("log_n", [4, 7])
def test_zh_eval_domain_is_low_degree_and_nonzero(log_n):
    """Z_H on the 4x domain never vanishes (the domains are disjoint) and interpolates
    to a circle polynomial with no coefficient at index >= 2n."""
    zh = O.zh_eval_domain(log_n)
    assert zh.min() > 0 and zh.max() < P
    c = O.stwo_interpolate(zh, log_n + 2)
    assert not c[2 << log_n:].any()
    assert c[: 2 << log_n].any()


def test_zh_eval_domain_matches_pointwise():
    """prover.rs:924-935: entry i is Z_H at half_odds(log_eval - 1).at(brev(i)), conjugated in the upper half."""
    log_n = 3
    log_eval = log_n + 2
    N = 1 << log_eval
    ix, iy, sx, sy = O.coset(O.HALF_ODDS, log_eval - 1)
    hx, hy = O.coset_points(ix, iy, sx, sy, N // 2)
    zh = O.zh_eval_domain(log_n)
    for i in range(N):
        b = int(format(i, f"0{log_eval}b")[::-1], 2)
        x, y = (int(hx[b]), int(hy[b])) if b < N // 2 else (int(hx[b - N // 2]), (P - int(hy[b - N // 2])) % P)
        assert int(zh[i]) == O.coset_vanishing_half_coset(log_n, x, y)


@pytest.mark.parametrize("log_n,nc", [(3, 1), (6, 3), (8, 16), (9, 5)])
def test_group_commit_unblinded(log_n, nc):
    n, N = 1 << log_n, 4 << log_n
    cols = np.stack([O.seeded_m31(0x7000 + c, n) for c in range(nc)])
    g = O.commit_group_cairo(cols, log_n)
    canon = np.empty_like(cols)
    for k in range(n):
        canon[:, hc_to_cn_brt(k, log_n)] = cols[:, k]
    for c in range(nc):
        assert np.array_equal(g["coeffs"][c], O.stwo_interpolate(canon[c], log_n))
    assert np.array_equal(g["eval_cn"], O.stwo_lde_columns(canon, log_n, 2))
    for k in range(0, N, max(1, N // 64)):
        assert np.array_equal(g["eval_hc"][:, k], g["eval_cn"][:, hc_to_cn_brt(k, log_n + 2)])
    assert np.array_equal(g["root"], O.merkle_root_capped(g["eval_cn"]))
    if N < 1024:
        assert np.array_equal(g["tile_roots"][0], g["root"])
    else:
        assert g["tile_roots"].shape[0] == N // 1024
        for t in range(N // 1024):
            assert np.array_equal(g["tile_roots"][t], O.merkle_root_capped(g["eval_cn"][:, 1024 * t: 1024 * (t + 1)]))
        assert np.array_equal(O.merkle_root_hashes(g["tile_roots"]), g["root"])


def test_group_commit_blinding_adds_r_times_zh():
    log_n, nc = 6, 4
    n = 1 << log_n
    cols = np.stack([O.seeded_m31(0x7100 + c, n) for c in range(nc)])
    r = np.array([0, 12345, P - 1, 1 << 30], np.uint32)
    g0 = O.commit_group_cairo(cols, log_n)
    g1 = O.commit_group_cairo(cols, log_n, r)
    zh = O.zh_eval_domain(log_n).astype(np.uint64)
    for c in range(nc):
        want = (g0["eval_cn"][c].astype(np.uint64) + int(r[c]) * zh) % P
        assert np.array_equal(g1["eval_cn"][c], want.astype(np.uint32))
    assert np.array_equal(g1["coeffs"], g0["coeffs"])  # coefficients are those of the unblinded trace
    assert not np.array_equal(g1["root"], g0["root"])
    # the blinded columns still agree with the trace on the trace domain: the
    # blinded polynomial's LDE interpolates to the trace's coefficients + r * Z_H's
    c_bl = O.stwo_interpolate(g1["eval_cn"][1], log_n + 2)
    c_zh = O.stwo_interpolate(O.zh_eval_domain(log_n), log_n + 2).astype(np.uint64)
    want = (np.concatenate([g0["coeffs"][1], np.zeros(3 * n, np.uint32)]).astype(np.uint64) + 12345 * c_zh) % P
    assert np.array_equal(c_bl, want.astype(np.uint32))


# ---------------------------------------------------------------- OODS + FRI tail (prover.rs:1937-2438)
def hc_index_map(log_n: int) -> np.ndarray:
    """pos[k] = BRT-canonic position of half-coset natural index k."""
    n = 1 << log_n
    k = np.arange(n, dtype=np.uint64)
    cn = np.where(k % 2 == 0, k // 2, n - 1 - k // 2)
    rev = np.zeros(n, np.uint64)
    for b in range(log_n):
        rev |= ((cn >> np.uint64(b)) & np.uint64(1)) << np.uint64(log_n - 1 - b)
    return rev.astype(np.int64)


def cairo_tail_inputs(log_n: int, nt: int, ni: int, seed: int):
    """Consistent low-degree inputs: blinded trace group (coefficients + LDE),
    interaction LDEs of degree < n, AIR quotient limbs of degree < 2n given in
    half-coset natural order."""
    n = 1 << log_n
    rng = np.random.default_rng(seed)
    cols = rng.integers(0, P, size=(nt, n), dtype=np.uint64).astype(np.uint32)
    zk = rng.integers(1, P, size=nt, dtype=np.uint64).astype(np.uint32)
    zk[::3] = 0
    g = O.commit_group_cairo(cols, log_n, zk)
    inter = O.stwo_lde_columns(rng.integers(0, P, size=(ni, n), dtype=np.uint64).astype(np.uint32), log_n, 2)
    q_cn = O.stwo_lde_columns(rng.integers(0, P, size=(4, 2 * n), dtype=np.uint64).astype(np.uint32), log_n + 1, 1)
    q_hc = q_cn[:, hc_index_map(log_n + 2)]
    return {"coeffs": g["coeffs"], "zk": zk, "evals": g["eval_cn"], "root": g["root"], "inter": inter,
            "q_hc": q_hc, "q_cn": q_cn}


def brt_to_natural(c: np.ndarray) -> np.ndarray:
    return c[[int(format(i, "03b")[::-1], 2) for i in range(8)]]


def run_tail(inp, log_n):
    ch = O.Channel()
    ch.mix_digest(inp["root"])
    r = O.cairo_oods_fri(ch, log_n, inp["coeffs"], inp["zk"], inp["evals"], inp["inter"], inp["q_hc"])
    return r, ch


@pytest.mark.parametrize("log_n,nt,ni", [(4, 3, 4), (6, 5, 12), (8, 16, 0)])
def test_cairo_tail_deep_quotient_is_low_degree(log_n, nt, ni):
    """With consistent inputs the DEEP quotient is a polynomial of degree < 2n, and
    after the folds the 8-value last layer has line degree < 4 (the reference's own
    OODS-degree and last-layer round-trip checks, prover.rs:2287-2307, 2391-2423)."""
    inp = cairo_tail_inputs(log_n, nt, ni, 0x6A00 + log_n)
    r, _ = run_tail(inp, log_n)
    N = 4 << log_n
    for k in range(4):
        c = O.stwo_interpolate(r["oods_quotient"][k], log_n + 2)
        assert not c[N // 2:].any()
    nat = brt_to_natural(r["last_layer_coeffs"])
    assert not nat[4:].any() and nat[:4].any()
    assert np.array_equal(r["quotient_root"], O.merkle_root_hashes(r["quotient_tiles"])) or N < 1024


def test_cairo_tail_sampled_values_match_the_committed_polynomials():
    """The trace values at z (coefficients + r * Z_H(z)) equal the blinded LDE's own
    interpolant at z; the quotient limbs at z equal their interpolant at z."""
    log_n = 5
    inp = cairo_tail_inputs(log_n, 4, 4, 0x6B00)
    r, _ = run_tail(inp, log_n)
    z = r["oods_point"]
    for c in range(4):
        full = O.stwo_interpolate(inp["evals"][c], log_n + 2)
        assert np.array_equal(O.eval_at_oods(full, z), r["trace_at_z"][c])
    for k in range(4):
        full = O.stwo_interpolate(inp["q_cn"][k], log_n + 2)
        assert np.array_equal(O.eval_at_oods(full, z), r["quotient_at_z"][k])
    assert r["fri_roots"].shape == (log_n - 2, 8) and r["fri_alphas"].shape == (log_n - 1, 4)


def test_cairo_tail_detects_an_inconsistent_column():
    """A planted error (one trace evaluation changed after its coefficients were
    taken) gives the DEEP quotient a pole: the last layer is no longer low degree."""
    log_n = 5
    inp = cairo_tail_inputs(log_n, 3, 4, 0x6C00)
    inp["evals"] = inp["evals"].copy()
    inp["evals"][1, 17] = (int(inp["evals"][1, 17]) + 1) % P
    r, _ = run_tail(inp, log_n)
    assert brt_to_natural(r["last_layer_coeffs"])[4:].any()


def test_cairo_tail_advances_channel_deterministically():
    log_n = 4
    inp = cairo_tail_inputs(log_n, 2, 4, 0x6D00)
    r1, c1 = run_tail(inp, log_n)
    r2, c2 = run_tail(inp, log_n)
    assert c1.state_bytes() == c2.state_bytes()
    assert np.array_equal(r1["oods_root"], r2["oods_root"])
    assert c1.state_bytes() != O.Channel().state_bytes()


# ---------------------------------------------------------------- decommitment paths (merkle.rs:846-861)
def _climb(leaf_hash, idx, path):
    h = leaf_hash
    for k, sib in enumerate(path):
        pair = np.concatenate([h, sib]) if ((idx >> k) & 1) == 0 else np.concatenate([sib, h])
        h = O.blake2s_words(pair)
    return h


@pytest.mark.parametrize("kind,nc,log_n", [(0, 5, 6), (0, 16, 9), (1, 4, 7)])
def test_oracle_tree_paths_reach_the_root(kind, nc, log_n):
    n = 1 << log_n
    cols = np.stack([O.seeded_m31(0x7A00 + c, n) for c in range(nc)])
    idx = [0, n - 1, 5, 5, n // 2 + 1]
    paths = O.tree_paths(kind, cols, idx)
    root = O.merkle_root_capped(cols) if kind == 0 else O.merkle_root_soa4(cols)
    for q, i in enumerate(idx):
        leaf = O.blake2s_words(cols[:min(nc, 16), i] if kind == 0 else cols[:4, i])
        assert np.array_equal(_climb(leaf, i, paths[q]), root)
