"""GPU parity: the device Fibonacci prover emits byte-identical KRAK proofs to the
oracle's restatement of the reference prover, and they verify."""
import ctypes as C

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


def gpu_prove(L, a, b, log_n) -> bytes:
    cap = 16 << 20
    buf = (C.c_uint8 * cap)()
    n = C.c_uint64(0)
    V.check(L.vs_prove_fib(a, b, log_n, buf, cap, C.byref(n), None), "vs_prove_fib")
    return bytes(buf[: n.value])


@pytest.mark.parametrize("log_n", [4, 5, 6, 8, 10, 11, 12, 14])
def test_prove_byte_identical(L, log_n):
    p = gpu_prove(L, 1, 1, log_n)
    assert p == O.prove(1, 1, log_n)
    assert O.verify(p) == (0, "")


@pytest.mark.parametrize("a,b", [(2, 3), (42, 99), (1000, 2000), (0x7FFFFFFE, 12345)])
def test_prove_inputs(L, a, b):
    assert gpu_prove(L, a, b, 6) == O.prove(a, b, 6)


def test_prove_log16_seeded(L):
    """log_n = 16 (65,536 rows), a1 seeded: the plain single-proof workload."""
    a1 = int(O.seeded_m31(0x56530000, 1)[0])
    p = gpu_prove(L, 1, a1, 16)
    assert p == O.prove(1, a1, 16)


def test_prove_deterministic_and_rejects_bad_args(L):
    assert gpu_prove(L, 5, 8, 7) == gpu_prove(L, 5, 8, 7)
    n = C.c_uint64(0)
    buf = (C.c_uint8 * 16)()
    assert L.vs_prove_fib(1, 1, 3, buf, 16, C.byref(n), None) == 1
    assert L.vs_prove_fib(0x7FFFFFFF, 1, 6, buf, 16, C.byref(n), None) == 1
    rc = L.vs_prove_fib(1, 1, 6, buf, 16, C.byref(n), None)  # buffer too small: length still reported
    assert rc == 1 and n.value > 16
