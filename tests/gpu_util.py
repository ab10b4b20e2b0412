"""Device-buffer helpers for the GPU parity tests (torch owns the memory; the
library is called through its C ABI with raw device pointers)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

P = 0x7FFFFFFF


def dev(a) -> torch.Tensor:
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return torch.from_numpy(a.view(np.int32).copy()).cuda()


def empty(n: int) -> torch.Tensor:
    return torch.empty(int(n), dtype=torch.int32, device="cuda")


def zeros(n: int) -> torch.Tensor:
    return torch.zeros(int(n), dtype=torch.int32, device="cuda")


def host(t: torch.Tensor) -> np.ndarray:
    torch.cuda.synchronize()
    return t.cpu().numpy().view(np.uint32)


# Every tensor whose raw pointer is handed to the library stays referenced here
# until the test has synchronised (tests/conftest.py clears it after each test):
# a temporary freed while a launch is queued would be recycled by torch's caching
# allocator and the kernel would read someone else's data.
KEEP: list = []


def ptr(t: torch.Tensor) -> int:
    KEEP.append(t)
    return t.data_ptr()


def ptr_array(ts) -> torch.Tensor:
    """Device array of device pointers (uint32_t**); keeps the columns alive too."""
    ts = list(ts)
    KEEP.extend(ts)
    arr = torch.tensor([t.data_ptr() for t in ts], dtype=torch.int64, device="cuda")
    KEEP.append(arr)
    return arr


def release() -> None:
    torch.cuda.synchronize()
    KEEP.clear()


def u32_host(vals) -> C.Array:
    vals = [int(v) for v in vals]
    return (C.c_uint32 * max(1, len(vals)))(*vals)


def rand_m31(rng: np.random.Generator, *shape) -> np.ndarray:
    return rng.integers(0, P, size=shape, dtype=np.uint64).astype(np.uint32)


# --- tiny exact QM31 helpers for small checks
def qm_mul(x, y):
    a, b, c, d = (int(v) for v in x)
    e, f, g, h = (int(v) for v in y)

    def cm(p, q, r, s):
        return ((p * r - q * s) % P, (p * s + q * r) % P)

    ac = cm(a, b, e, f)
    bd = cm(c, d, g, h)
    ad = cm(a, b, g, h)
    bc = cm(c, d, e, f)
    bdu = ((2 * bd[0] - bd[1]) % P, (bd[0] + 2 * bd[1]) % P)
    return [(ac[0] + bdu[0]) % P, (ac[1] + bdu[1]) % P, (ad[0] + bc[0]) % P, (ad[1] + bc[1]) % P]


def qm_add(x, y):
    return [(int(a) + int(b)) % P for a, b in zip(x, y)]
