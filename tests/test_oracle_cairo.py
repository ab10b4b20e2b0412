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
