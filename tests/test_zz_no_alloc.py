"""vs_merkle_root_rowpacked_noalloc: the Merkle root for callers that cannot
allocate device memory at call time (its scratch is a fixed array inside the
library). Called through the C ABI twice in a row with different inputs, it must
match vs_merkle_root_rowpacked and the CPU oracle's row-packed root bit for bit
(the integer tests' tolerance is exact). Kept in its own, last-collected file so a
failure here does not hide the other tests; it also passes alone in a fresh
process."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import vortexstark_b200 as V  # noqa: E402


@pytest.fixture(scope="module")
def L():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return V.lib()


def _cols(n_cols, log_n, seed):
    t = torch.empty((n_cols, 1 << log_n), dtype=torch.int32, device="cuda")
    V.check(V.lib().vs_fill_uniform_m31(t.data_ptr(), t.numel(), seed, 0, None), "fill")
    return t


def _roots(L, cols, log_n):
    n_cols = cols.shape[0]
    a = torch.zeros(8, dtype=torch.int32, device="cuda")
    b = torch.full((8,), -1, dtype=torch.int32, device="cuda")
    V.check(L.vs_merkle_root_rowpacked(cols.data_ptr(), 1 << log_n, n_cols, log_n, a.data_ptr(), None), "alloc path")
    V.check(L.vs_merkle_root_rowpacked_noalloc(cols.data_ptr(), 1 << log_n, n_cols, log_n, b.data_ptr(), None),
            "noalloc path")
    torch.cuda.synchronize()
    return a.cpu().numpy(), b.cpu().numpy()


def _oracle_root(n_cols, log_n, seed):
    cols = O.seeded_m31(seed, n_cols << log_n).reshape(n_cols, -1)
    return O.merkle_root_rowpacked(cols, threads=os.cpu_count() or 1).view(np.int32)


def test_noalloc_matches_allocating_root_twice(L):
    first = _cols(34, 16, 0x1001)   # uses the scratch array (64 subtree roots)
    second = _cols(5, 21, 0x1002)   # reuses it with different contents (2048 + 2 roots)
    for cols, log_n, seed in ((first, 16, 0x1001), (second, 21, 0x1002)):
        a, b = _roots(L, cols, log_n)
        assert np.array_equal(a, b)
        assert np.array_equal(b, _oracle_root(cols.shape[0], log_n, seed))
    small = _cols(3, 8, 0x1003)     # at most 1024 leaves: no scratch at all
    a, b = _roots(L, small, 8)
    assert np.array_equal(a, b)


def test_noalloc_largest_accepted_and_rejects_beyond(L):
    cols = _cols(2, 26, 0x1004)
    a, b = _roots(L, cols, 26)
    assert np.array_equal(a, b)
    assert np.array_equal(b, _oracle_root(2, 26, 0x1004))
    root = torch.zeros(8, dtype=torch.int32, device="cuda")
    rc = L.vs_merkle_root_rowpacked_noalloc(cols.data_ptr(), 1 << 26, 1, 27, root.data_ptr(), None)
    assert rc == 1 and b"exceeds" in L.vs_last_error()
