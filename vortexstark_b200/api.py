"""Host API over libvstark for torch device tensors.

Names follow the reference's host API for this path: commitment of columns
(src/merkle.rs commit_root_only / cairo_air trace commit), FRI fold + commit
(src/fri.rs), Fibonacci prove / verify (src/prover.rs:192, src/verifier.rs:39).
Tensors are int32 views of u32 field words, on a CUDA device.
"""
from __future__ import annotations

import ctypes as C
import threading

import torch

from . import check, lib

PROOF_CAP = 32 << 20  # bytes; the largest proof (log_n = 28) is a few MB


def _stream(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def _ptr(t: torch.Tensor) -> int:
    if not t.is_cuda or t.dtype != torch.int32 or not t.is_contiguous():
        raise TypeError("expected a contiguous int32 CUDA tensor")
    return t.data_ptr()


def fill_uniform_m31(out: torch.Tensor, seed: int, offset: int = 0, stream=None) -> torch.Tensor:
    check(lib().vs_fill_uniform_m31(_ptr(out), out.numel(), seed, offset, _stream(stream)), "vs_fill_uniform_m31")
    return out


def lde_stwo(cols: torch.Tensor, log_n: int, blowup: int = 2, out: torch.Tensor | None = None, stream=None):
    """cols: (n_cols, 2^log_n) BRT-canonic evaluations -> (n_cols, 2^(log_n+blowup))."""
    n_cols = cols.shape[0]
    N = 1 << (log_n + blowup)
    if out is None:
        out = torch.empty((n_cols, N), dtype=torch.int32, device=cols.device)
    check(lib().vs_lde_stwo(_ptr(cols), 1 << log_n, _ptr(out), N, n_cols, log_n, blowup, _stream(stream)), "vs_lde_stwo")
    return out


def commit_columns(cols: torch.Tensor, log_n: int, blowup: int, lde: torch.Tensor, root: torch.Tensor, stream=None):
    """Commitment-layer step: stwo LDE of every column + row-packed Blake2s Merkle root."""
    check(lib().vs_commit_columns(_ptr(cols), cols.shape[0], log_n, blowup, _ptr(lde), _ptr(root), _stream(stream)),
          "vs_commit_columns")


def merkle_root_rowpacked(cols: torch.Tensor, root: torch.Tensor, stream=None):
    n_cols, n = cols.shape
    check(lib().vs_merkle_root_rowpacked(_ptr(cols), n, n_cols, n.bit_length() - 1, _ptr(root), _stream(stream)),
          "vs_merkle_root_rowpacked")


def merkle_root_capped(cols: torch.Tensor, root: torch.Tensor, stream=None):
    """Root over leaves of the first min(n_cols, 16) columns (the reference's native leaf)."""
    n_cols, n = cols.shape
    stride = cols.stride(0)
    if cols.stride(1) != 1 or not cols.is_cuda or cols.dtype != torch.int32:
        raise TypeError("expected int32 CUDA rows with unit stride")
    check(lib().vs_merkle_root_capped(cols.data_ptr(), stride, n_cols, n.bit_length() - 1, _ptr(root),
                                      _stream(stream)), "vs_merkle_root_capped")


def fri_fold_commit(src: torch.Tensor, log_n: int, alphas, work: torch.Tensor, roots: torch.Tensor,
                    last: torch.Tensor, stream=None):
    """src: (4, 2^log_n) SoA4 QM31; alphas: (log_n - 3) x 4 host words."""
    flat = [int(x) for row in alphas for x in row]
    arr = (C.c_uint32 * len(flat))(*flat)
    check(lib().vs_fri_fold_commit(_ptr(src), log_n, arr, _ptr(work), _ptr(roots), _ptr(last), _stream(stream)),
          "vs_fri_fold_commit")


_tls = threading.local()


def _proof_buffer():
    """One reusable host buffer per thread for proofs coming back from the library."""
    buf = getattr(_tls, "buf", None)
    if buf is None:
        buf = _tls.buf = (C.c_uint8 * PROOF_CAP)()
    return buf


def prove_fib(a: int, b: int, log_n: int, stream=None) -> bytes:
    """Fibonacci proof in the KRAK v1 wire format."""
    buf = _proof_buffer()
    n = C.c_uint64(0)
    check(lib().vs_prove_fib(a, b, log_n, buf, PROOF_CAP, C.byref(n), _stream(stream)), "vs_prove_fib")
    return C.string_at(buf, n.value)


def commit_seeded(log_n: int, n_cols: int, seed: int, blowup: int = 2, stream=None) -> bytes:
    """Root of n_cols seeded uniform-M31 columns of 2^log_n rows (stwo LDE + row-packed Merkle),
    one call at a time through the drop-in entry points."""
    dev = torch.device("cuda", torch.cuda.current_device())
    cols = fill_uniform_m31(torch.empty((n_cols, 1 << log_n), dtype=torch.int32, device=dev), seed, 0, stream)
    lde = torch.empty((n_cols, 1 << (log_n + blowup)), dtype=torch.int32, device=dev)
    root = torch.empty(8, dtype=torch.int32, device=dev)
    commit_columns(cols, log_n, blowup, lde, root, stream)
    return root.cpu().numpy().tobytes()


def verify_fib(proof: bytes) -> tuple[bool, str]:
    buf = (C.c_uint8 * max(1, len(proof))).from_buffer_copy(proof or b"\0")
    err = C.create_string_buffer(256)
    rc = lib().vs_verify_fib(buf, len(proof), err, 256)
    return rc == 0, err.value.decode()


def init_memory_pool(release_threshold_bytes: int = 2 << 30) -> None:
    """Keep this many bytes cached in the device's default stream-ordered pool
    (the reference's init_memory_pool keeps 2 GiB)."""
    check(lib().vs_init_memory_pool(release_threshold_bytes), "vs_init_memory_pool")


def launch_count() -> int:
    return int(lib().vs_launch_count())


# ---------------------------------------------------------------- batched / served proving
class Job(C.Structure):
    """vs_job: kind 0 = Fibonacci proof (log_n, a, b), 1 = column commitment (log_n, n_cols, seed)."""
    _fields_ = [("kind", C.c_uint32), ("log_n", C.c_uint32), ("a", C.c_uint32), ("b", C.c_uint32),
                ("n_cols", C.c_uint32), ("pad", C.c_uint32), ("seed", C.c_uint64)]


class JobResult(C.Structure):
    _fields_ = [("status", C.c_int), ("pad", C.c_uint32), ("out_len", C.c_uint64), ("t_submit", C.c_double),
                ("t_start", C.c_double), ("t_end", C.c_double)]


FIB, COMMIT = 0, 1


def fib_job(log_n: int, a: int, b: int) -> Job:
    return Job(FIB, log_n, a, b, 0, 0, 0)


def commit_job(log_n: int, n_cols: int, seed: int) -> Job:
    return Job(COMMIT, log_n, 0, 0, n_cols, 0, seed)


class Engine:
    """Slots of concurrent provers with FIFO admission against an HBM budget."""

    def __init__(self, slots: int, hbm_budget_bytes: int = 0, size_priority: bool = True):
        """size_priority: run small jobs on higher-priority CUDA streams (VS_ENGINE_FIFO_PRIORITY off)."""
        self.h = C.c_void_p()
        flags = 0 if size_priority else 1
        check(lib().vs_engine_create_ex(slots, hbm_budget_bytes, flags, C.byref(self.h)), "vs_engine_create_ex")
        self._buf = (C.c_uint8 * PROOF_CAP)()

    def prepare(self, job: Job) -> None:
        check(lib().vs_engine_prepare(self.h, C.byref(job)), "vs_engine_prepare")

    def submit(self, job: Job) -> int:
        t = C.c_uint64()
        check(lib().vs_engine_submit(self.h, C.byref(job), C.byref(t)), "vs_engine_submit")
        return t.value

    def wait(self, ticket: int):
        """Returns (result bytes, t_submit, t_start, t_end) in engine seconds."""
        r = JobResult()
        check(lib().vs_engine_wait(self.h, ticket, C.byref(r), self._buf, PROOF_CAP), "vs_engine_wait")
        return C.string_at(self._buf, r.out_len), r.t_submit, r.t_start, r.t_end

    def drain(self) -> None:
        lib().vs_engine_drain(self.h)

    def now(self) -> float:
        return lib().vs_engine_now(self.h)

    def close(self) -> None:
        if self.h:
            lib().vs_engine_destroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
