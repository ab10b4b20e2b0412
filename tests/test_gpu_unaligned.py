"""GPU: entry points given device pointers that are only 4-byte aligned.

The reference's kernels read caller buffers word by word, so a caller may pass
any word-aligned pointer (a column at an odd offset inside a larger buffer, a
stride that is not a multiple of four words). The kernels here use 64/128-bit
accesses and 16-byte async copies where the address allows and words elsewhere;
results must equal the oracle's either way."""
import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from gpu_util import dev, empty, host, ptr, rand_m31  # noqa: E402
import vortexstark_b200 as V  # noqa: E402


@pytest.fixture(scope="module")
def L():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return V.lib()


def shifted(x: np.ndarray, shift: int) -> torch.Tensor:
    """Device copy of x starting `shift` words into its allocation."""
    return dev(np.concatenate([np.zeros(shift, np.uint32), np.asarray(x, np.uint32).reshape(-1)]))[shift:]


@pytest.mark.parametrize("log_n", [5, 10, 16, 20])
@pytest.mark.parametrize("shift,tw_shift", [(1, 0), (3, 1), (2, 2)])
def test_stwo_ntt_unaligned(L, log_n, shift, tw_shift):
    rng = np.random.default_rng(log_n * 10 + shift)
    x = rand_m31(rng, 1 << log_n)
    fwd, inv = O.stwo_twiddles(log_n)
    d = shifted(x, shift)
    L.cuda_stwo_ntt_evaluate(ptr(d), ptr(shifted(fwd, tw_shift)), 1 << log_n)
    ev = host(d)
    assert np.array_equal(ev, O.stwo_evaluate(x, log_n))
    L.cuda_stwo_ntt_interpolate(ptr(d), ptr(shifted(inv, tw_shift)), 1 << log_n)
    assert np.array_equal(host(d), x)


@pytest.mark.parametrize("log_n", [12, 14, 16, 20])
def test_lde_stwo_unaligned_strides(L, log_n):
    """Columns at word offsets 1 and 3 with strides that are not multiples of 4."""
    rng = np.random.default_rng(200 + log_n)
    n, N, nc = 1 << log_n, 1 << (log_n + 2), 3
    cols = rand_m31(rng, nc, n)
    ss, ds = n + 1, N + 3
    src_buf = np.zeros(1 + nc * ss, np.uint32)
    for c in range(nc):
        src_buf[1 + c * ss: 1 + c * ss + n] = cols[c]
    src = dev(src_buf)[1:]
    dst = empty(3 + nc * ds)[3:]
    V.check(L.vs_lde_stwo(ptr(src), ss, ptr(dst), ds, nc, log_n, 2, None), "vs_lde_stwo")
    got = host(dst)
    exp = O.stwo_lde_columns(cols, log_n, 2, threads=8).reshape(nc, N)
    for c in range(nc):
        assert np.array_equal(got[c * ds: c * ds + N], exp[c])


def test_hash_nodes_and_interleave_unaligned(L):
    rng = np.random.default_rng(7)
    h = rand_m31(rng, 1024, 8)
    out = empty(1 + 512 * 8)[1:]
    L.cuda_merkle_hash_nodes(ptr(shifted(h, 1)), ptr(out), 512)
    assert np.array_equal(host(out).reshape(512, 8), O.hash_nodes(h))
    x, y = rand_m31(rng, 1000), rand_m31(rng, 1000)
    il = empty(1 + 2000)[1:]
    L.cuda_interleave_u32(ptr(dev(x)), ptr(dev(y)), ptr(il), 1000)
    assert np.array_equal(host(il), np.stack([x, y], 1).reshape(-1))


@pytest.mark.parametrize("log_n", [10, 16])
def test_fri_fold_commit_unaligned(L, log_n):
    """The same seeded QM31 vector from an aligned and a word-offset buffer commits identically."""
    N = 1 << log_n
    rng = np.random.default_rng(log_n)
    src = rand_m31(rng, 4 * N)
    alphas = rand_m31(rng, 4 * (log_n - 3))
    import ctypes as C
    arr = (C.c_uint32 * alphas.size)(*[int(a) for a in alphas])
    outs = []
    for shift in (0, 1):
        work = empty(shift + 4 * N)[shift:]
        roots = empty(8 * (log_n - 3))
        last = empty(32)
        V.check(L.vs_fri_fold_commit(ptr(shifted(src, shift)), log_n, arr, ptr(work), ptr(roots), ptr(last), None),
                "vs_fri_fold_commit")
        outs.append((host(roots).tobytes(), host(last).tobytes()))
    assert outs[0] == outs[1]
