"""GPU: proof-of-work grinding (cuda_grind_pow, cuda_grind_pow_m31_output and the
channel's grind) against the oracle's brute-force minimum nonce."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from gpu_util import dev, ptr  # noqa: E402
import vortexstark_b200 as V  # noqa: E402

U64_MAX = 2**64 - 1


@pytest.fixture(scope="module")
def L():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return V.lib()


def prefix_for(seed, bits):
    ch = O.Channel()
    ch.mix_digest(np.arange(seed, seed + 8, dtype=np.uint32))
    return ch, ch.pow_prefix(bits)


@pytest.mark.parametrize("m31", [False, True])
@pytest.mark.parametrize("bits,offset,n", [(8, 0, 1 << 12), (12, 0, 1 << 16), (12, 70000, 50000), (14, 3, 1 << 18),
                                           (20, 0, 1000)])
def test_grind_dropin_minimum(L, m31, bits, offset, n):
    _, prefix = prefix_for(bits + offset % 97, bits)
    res = torch.full((1,), -1, dtype=torch.int64, device="cuda")  # UINT64_MAX
    fn = L.cuda_grind_pow_m31_output if m31 else L.cuda_grind_pow
    fn(ptr(dev(prefix)), ptr(res), bits, offset, n)
    torch.cuda.synchronize()
    got = int(res.cpu().numpy().view(np.uint64)[0])
    assert got == O.pow_grind_min(prefix, bits, offset, n, m31)


def test_grind_batches_keep_first_found(L):
    """A later batch never replaces a nonce found by an earlier one (offsets grow)."""
    _, prefix = prefix_for(1, 10)
    res = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    d = dev(prefix)
    for off in range(0, 1 << 16, 1 << 12):
        L.cuda_grind_pow(ptr(d), ptr(res), 10, off, 1 << 12)
    torch.cuda.synchronize()
    assert int(res.cpu().numpy().view(np.uint64)[0]) == O.pow_grind_min(prefix, 10, 0, 1 << 16)


@pytest.mark.parametrize("bits", [4, 16, 20])
def test_channel_grind_then_mix(L, bits):
    ch = C.c_void_p()
    V.check(L.vs_channel_create(C.byref(ch)))
    try:
        ref, _ = prefix_for(7, bits)
        d = np.arange(7, 15, dtype=np.uint32)
        V.check(L.vs_channel_mix_digest(ch, d.ctypes.data))
        nonce = C.c_uint64()
        V.check(L.vs_channel_grind_pow(ch, bits, 1 << 28, C.byref(nonce), None), "vs_channel_grind_pow")
        n = nonce.value
        assert n == O.pow_grind_min(ref.pow_prefix(bits), bits, 0, n + 1)
        assert L.vs_channel_verify_pow_nonce(ch, bits, n) == 1 and ref.verify_pow(bits, n)
        V.check(L.vs_channel_mix_u64(ch, n))
        ref.mix_u64(n)
        b = (C.c_uint8 * 32)()
        V.check(L.vs_channel_state(ch, b, None))
        assert bytes(b) == ref.state_bytes()
    finally:
        L.vs_channel_destroy(ch)
