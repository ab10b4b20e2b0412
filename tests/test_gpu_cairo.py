"""GPU parity of the device-resident Cairo column-group commitment
(vs_commit_group_cairo; cairo_air/prover.rs:899-1047 with merkle.rs:360-417)
against the CPU oracle, bit-exact: coefficients, blinded BRT-canonic LDE, the
half-coset copy, root and 1024-leaf tile roots."""
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


@pytest.mark.parametrize("log_n", [6, 11])
def test_group_commit_unblinded_and_optional_outputs(L, log_n):
    """No blinding scalars, no coefficient / half-coset / tile-root outputs, padded column stride."""
    n, nc = 1 << log_n, 5
    cols = np.stack([O.seeded_m31(0x7300 + c, n) for c in range(nc)])
    got = run_group(L, cols, log_n, None, stride=n + 12, want=())
    check(got, O.commit_group_cairo(cols, log_n))


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
