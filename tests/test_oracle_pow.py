"""CPU: the oracle's proof-of-work grinding and channel helpers pinned to hashlib.

Follows the reference's Blake2s PoW (src/channel.rs:140-168, cuda/grind.cu,
cuda/grind_m31_output.cu): prefix = Blake2s(0x12345678_LE || 0^12 || state ||
pow_bits_LE); a nonce passes when the first 16 bytes of Blake2s(prefix || nonce_LE),
read as a little-endian u128 (each word reduced mod 2^31 - 1 first for the M31
variant), have at least pow_bits trailing zeros."""
import hashlib
import struct

import numpy as np
import pytest

import oracle_lib as O

P = 0x7FFFFFFF


def tz_hashlib(prefix_words, nonce, m31=False):
    d = hashlib.blake2s(np.asarray(prefix_words, np.uint32).tobytes() + struct.pack("<Q", nonce)).digest()
    words = list(struct.unpack("<8I", d))[:4]
    if m31:
        words = [w % P for w in words]
    v = sum(w << (32 * i) for i, w in enumerate(words))
    return 128 if v == 0 else (v & -v).bit_length() - 1


def fresh_channel(seed):
    ch = O.Channel()
    ch.mix_digest(np.arange(seed, seed + 8, dtype=np.uint32))
    return ch


def test_pow_prefix_matches_hashlib():
    ch = fresh_channel(3)
    for bits in (0, 5, 20):
        exp = hashlib.blake2s(struct.pack("<I", 0x12345678) + bytes(12) + ch.state_bytes() + struct.pack("<I", bits))
        assert ch.pow_prefix(bits).tobytes() == exp.digest()


@pytest.mark.parametrize("m31", [False, True])
def test_trailing_zeros_match_hashlib(m31):
    prefix = fresh_channel(9).pow_prefix(12)
    for nonce in [0, 1, 2, 1000, 2**32 + 5, 2**63 + 17]:
        assert O.pow_trailing_zeros(prefix, nonce, m31) == tz_hashlib(prefix, nonce, m31)


@pytest.mark.parametrize("m31", [False, True])
def test_grind_finds_the_smallest_valid_nonce(m31):
    prefix = fresh_channel(21).pow_prefix(10)
    n = O.pow_grind_min(prefix, 10, 0, 1 << 16, m31)
    assert n < (1 << 16)
    assert tz_hashlib(prefix, n, m31) >= 10
    assert all(tz_hashlib(prefix, k, m31) < 10 for k in range(n))
    assert O.pow_grind_min(prefix, 10, n + 1, 3, m31) in (2**64 - 1, n + 1, n + 2, n + 3)


def test_verify_pow_nonce_and_mix_u64():
    ch = fresh_channel(40)
    prefix = ch.pow_prefix(8)
    n = O.pow_grind_min(prefix, 8, 0, 1 << 14)
    assert ch.verify_pow(8, n) and not ch.verify_pow(8 + tz_hashlib(prefix, n) + 1, n)
    before = ch.state_bytes()
    ch.mix_u64(n)
    assert ch.state_bytes() == hashlib.blake2s(before + struct.pack("<Q", n)).digest()
