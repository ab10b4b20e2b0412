"""The channel C ABI (host code in libvstark, no GPU needed) against the oracle's
channel, call for call: mix_digest, mix_felts, draw_felt, draw_number,
draw_query_indices, mix_u64, the PoW prefix and nonce check."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
import vortexstark_b200 as V


@pytest.fixture(scope="module")
def L():
    return V.lib()


class Ch:
    def __init__(self, L):
        self.L, self.h = L, C.c_void_p()
        V.check(L.vs_channel_create(C.byref(self.h)))

    def state(self):
        b = (C.c_uint8 * 32)()
        n = C.c_uint32()
        V.check(self.L.vs_channel_state(self.h, b, C.byref(n)))
        return bytes(b), n.value

    def close(self):
        self.L.vs_channel_destroy(self.h)


def u32(a):
    a = np.ascontiguousarray(a, np.uint32)
    return a, a.ctypes.data


def test_channel_matches_oracle_call_for_call(L):
    rng = np.random.default_rng(5)
    ch, ref = Ch(L), O.Channel()
    try:
        for step in range(40):
            op = step % 7
            if op == 0:
                d = rng.integers(0, 2**32, 8, dtype=np.uint64).astype(np.uint32)
                a, p = u32(d)
                V.check(L.vs_channel_mix_digest(ch.h, p))
                ref.mix_digest(d)
            elif op == 1:
                f = rng.integers(0, 2**31 - 1, (1 + step % 5, 4)).astype(np.uint32)
                a, p = u32(f)
                V.check(L.vs_channel_mix_felts(ch.h, p, f.shape[0]))
                ref.mix_felts(f)
            elif op == 2:
                o = np.empty(4, np.uint32)
                V.check(L.vs_channel_draw_felt(ch.h, o.ctypes.data))
                assert np.array_equal(o, ref.draw_felt())
            elif op == 3:
                out = C.c_uint64()
                bound = int(rng.integers(1, 2**40))
                V.check(L.vs_channel_draw_number(ch.h, bound, C.byref(out)))
                assert out.value == ref.draw_number(bound)
            elif op == 4:
                n, log = 80 + step, 10 + step % 12
                o = np.empty(n, np.uint32)
                V.check(L.vs_channel_draw_query_indices(ch.h, log, n, o.ctypes.data))
                assert np.array_equal(o.astype(np.uint64), ref.draw_queries(log, n))
            elif op == 5:
                v = int(rng.integers(0, 2**63))
                V.check(L.vs_channel_mix_u64(ch.h, v))
                ref.mix_u64(v)
            else:
                bits = 5 + step % 20
                o = np.empty(8, np.uint32)
                V.check(L.vs_channel_pow_prefix(ch.h, bits, o.ctypes.data))
                assert np.array_equal(o, ref.pow_prefix(bits))
                nonce = O.pow_grind_min(ref.pow_prefix(6), 6, 0, 1 << 12)
                assert L.vs_channel_verify_pow_nonce(ch.h, 6, nonce) == int(ref.verify_pow(6, nonce)) == 1
            assert ch.state()[0] == ref.state_bytes()
    finally:
        ch.close()


def test_channel_rejects_bad_arguments(L):
    out = C.c_uint64()
    assert L.vs_channel_draw_number(None, 5, C.byref(out)) != 0
    assert L.vs_channel_verify_pow_nonce(None, 5, 1) == -1
    ch = Ch(L)
    try:
        assert L.vs_channel_draw_number(ch.h, 0, C.byref(out)) != 0
        assert L.vs_channel_draw_query_indices(ch.h, 33, 1, np.empty(1, np.uint32).ctypes.data) != 0
    finally:
        ch.close()
