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


def ntt_plan(log_n: int) -> tuple[int, int, int]:
    """(lower pass layers, tiles per CTA, register-round radix) used for 2^log_n transforms."""
    v = [C.c_uint32() for _ in range(3)]
    check(lib().vs_ntt_plan_get(log_n, *[C.byref(x) for x in v]), "vs_ntt_plan_get")
    return tuple(int(x.value) for x in v)


def set_ntt_plan(log_n: int, lower: int = 0, items: int = 0, radix: int = 0) -> None:
    """Sets the launch shape of 2^log_n transforms (zeros restore the defaults)."""
    check(lib().vs_ntt_plan_set(log_n, lower, items, radix), "vs_ntt_plan_set")


def ntt_plan_candidates(log_n: int) -> list[tuple[int, int, int]]:
    n = C.c_uint32()
    check(lib().vs_ntt_plan_candidates(log_n, None, 0, C.byref(n)), "vs_ntt_plan_candidates")
    buf = (C.c_uint32 * max(1, 3 * n.value))()
    check(lib().vs_ntt_plan_candidates(log_n, buf, n.value, C.byref(n)), "vs_ntt_plan_candidates")
    return [tuple(buf[3 * i:3 * i + 3]) for i in range(n.value)]


def autotune_lde(log_n: int, n_cols: int = 34, blowup: int = 2, reps: int = 3, stream=None) -> dict:
    """Times every candidate plan of 2^log_n on an n_cols-column LDE, keeps the fastest
    and returns {"best": plan, "candidates": [(plan, ms per LDE), ...]}."""
    cands = ntt_plan_candidates(log_n)
    best = (C.c_uint32 * 3)()
    ms = (C.c_float * max(1, len(cands)))()
    check(lib().vs_autotune_lde(log_n, n_cols, blowup, reps, best, ms, len(cands), _stream(stream)),
          "vs_autotune_lde")
    return {"best": tuple(best), "candidates": [(c, float(ms[i])) for i, c in enumerate(cands)]}


def merkle_split() -> int:
    """First-level split of root-only Merkle trees (2^split roots per 1024-leaf tile)."""
    return int(lib().vs_merkle_split_get())


def set_merkle_split(split: int) -> None:
    check(lib().vs_merkle_split_set(split), "vs_merkle_split_set")


def autotune_merkle(log_leaves: int, n_cols: int = 34, reps: int = 3, stream=None) -> dict:
    """Times the row-packed root at every split, keeps the fastest; {"best": s, "ms": [...]}."""
    best = C.c_uint32()
    ms = (C.c_float * 9)()
    check(lib().vs_autotune_merkle(log_leaves, n_cols, reps, C.byref(best), ms, 9, _stream(stream)),
          "vs_autotune_merkle")
    return {"best": int(best.value), "ms": [float(x) for x in ms]}


def save_tuning(path, log_ns=range(5, 31)) -> None:
    """Writes the current NTT plans ({log_n: [lower, items, radix]}) and Merkle split as JSON."""
    import json
    with open(path, "w") as f:
        json.dump({"ntt": {str(l): list(ntt_plan(l)) for l in log_ns}, "merkle_split": merkle_split()}, f, indent=1)


def load_tuning(path) -> None:
    import json
    with open(path) as f:
        t = json.load(f)
    for k, v in t.get("ntt", {}).items():
        set_ntt_plan(int(k), *v)
    if "merkle_split" in t:
        set_merkle_split(int(t["merkle_split"]))


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


class EngineStats(C.Structure):
    """Mirror of vs_engine_stats (include/vstark.h)."""
    _fields_ = [("budget_bytes", C.c_uint64), ("resident_bytes", C.c_uint64), ("twiddle_bytes", C.c_uint64),
                ("peak_held_bytes", C.c_uint64), ("evictions", C.c_uint64), ("workspaces_created", C.c_uint64),
                ("idle_workspaces", C.c_uint32), ("busy_workspaces", C.c_uint32), ("queued", C.c_uint32),
                ("running", C.c_uint32)]


FIB, COMMIT = 0, 1
VS_ERR_BUDGET, VS_ERR_TIMEOUT, VS_ERR_CANCELLED, VS_ERR_BUSY, VS_ERR_OOM = 4, 5, 6, 7, 3


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

    def submit_many(self, jobs) -> list[int]:
        """Queues the jobs at once (slots then batch them fully); returns their tickets."""
        arr = (Job * max(1, len(jobs)))(*jobs)
        t = (C.c_uint64 * max(1, len(jobs)))()
        check(lib().vs_engine_submit_many(self.h, arr, len(jobs), t), "vs_engine_submit_many")
        return list(t)[:len(jobs)]

    def wait(self, ticket: int, timeout_s: float | None = None):
        """Returns (result bytes, t_submit, t_start, t_end) in engine seconds. With a
        timeout, raises VstarkError (status VS_ERR_TIMEOUT = 5) when the job is not
        done in time; the ticket stays valid."""
        r = JobResult()
        t = -1.0 if timeout_s is None else float(timeout_s)
        check(lib().vs_engine_wait_for(self.h, ticket, t, C.byref(r), self._buf, PROOF_CAP), "vs_engine_wait")
        return C.string_at(self._buf, r.out_len), r.t_submit, r.t_start, r.t_end

    def wait_status(self, ticket: int, timeout_s: float | None = None) -> tuple[int, bytes]:
        """(status, result bytes) without raising; status 0 = done."""
        r = JobResult()
        t = -1.0 if timeout_s is None else float(timeout_s)
        rc = lib().vs_engine_wait_for(self.h, ticket, t, C.byref(r), self._buf, PROOF_CAP)
        return rc, (C.string_at(self._buf, r.out_len) if rc == 0 else b"")

    def cancel(self, ticket: int) -> int:
        """0 when the queued job was cancelled; VS_ERR_BUSY (7) when it already runs or ran."""
        return int(lib().vs_engine_cancel(self.h, ticket))

    def set_batch_limit(self, max_jobs: int) -> None:
        """At most max_jobs proofs per batched graph launch (0: per-size default, 1: no batching)."""
        check(lib().vs_engine_set_batch_limit(self.h, max_jobs), "vs_engine_set_batch_limit")

    def workspace_bytes(self, job: Job) -> int:
        b = C.c_uint64()
        check(lib().vs_engine_workspace_bytes(self.h, C.byref(job), C.byref(b)), "vs_engine_workspace_bytes")
        return b.value

    def inject_alloc_failures(self, count: int) -> None:
        check(lib().vs_engine_inject_alloc_failures(self.h, count), "vs_engine_inject_alloc_failures")

    def stats(self) -> dict:
        st = EngineStats()
        check(lib().vs_engine_get_stats(self.h, C.byref(st)), "vs_engine_get_stats")
        return {f: getattr(st, f) for f, _ in EngineStats._fields_}

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


# ------------------------------------------------------------------ channel (src/channel.rs)
class Channel:
    """Fiat-Shamir transcript held by the library (vs_channel_*)."""

    def __init__(self):
        self.h = C.c_void_p()
        check(lib().vs_channel_create(C.byref(self.h)), "vs_channel_create")

    def mix_digest(self, words8) -> None:
        a = (C.c_uint32 * 8)(*[int(w) for w in words8])
        check(lib().vs_channel_mix_digest(self.h, a), "vs_channel_mix_digest")

    def mix_felts(self, felts) -> None:
        flat = [int(w) for f in felts for w in f]
        a = (C.c_uint32 * max(1, len(flat)))(*flat)
        check(lib().vs_channel_mix_felts(self.h, a, len(flat) // 4), "vs_channel_mix_felts")

    def mix_u64(self, v: int) -> None:
        check(lib().vs_channel_mix_u64(self.h, v), "vs_channel_mix_u64")

    def draw_felt(self) -> list[int]:
        o = (C.c_uint32 * 4)()
        check(lib().vs_channel_draw_felt(self.h, o), "vs_channel_draw_felt")
        return list(o)

    def draw_query_indices(self, log_domain: int, n: int) -> list[int]:
        o = (C.c_uint32 * max(1, n))()
        check(lib().vs_channel_draw_query_indices(self.h, log_domain, n, o), "vs_channel_draw_query_indices")
        return list(o)[:n]

    def grind_pow(self, pow_bits: int, max_nonces: int = 1 << 40, stream=None) -> int:
        nonce = C.c_uint64()
        check(lib().vs_channel_grind_pow(self.h, pow_bits, max_nonces, C.byref(nonce), _stream(stream)),
              "vs_channel_grind_pow")
        return nonce.value

    def state(self) -> tuple[bytes, int]:
        s = (C.c_uint8 * 32)()
        n = C.c_uint32()
        check(lib().vs_channel_state(self.h, s, C.byref(n)), "vs_channel_state")
        return bytes(s), n.value

    def close(self) -> None:
        if self.h:
            lib().vs_channel_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ Cairo trace commitment and tail
def commit_group_cairo(cols_hc: torch.Tensor, log_n: int, blind=None, coeffs: torch.Tensor | None = None,
                       eval_hc: torch.Tensor | None = None, tile_roots: torch.Tensor | None = None, stream=None):
    """One Cairo column group (<= 16 columns, half-coset natural order) -> BRT-canonic
    x4 LDE, blinded (cairo_air/prover.rs:899-1047). Returns (eval_cn, root)."""
    n_cols, stride = cols_hc.shape
    N = 4 << log_n
    eval_cn = torch.empty((n_cols, N), dtype=torch.int32, device=cols_hc.device)
    root = torch.empty(8, dtype=torch.int32, device=cols_hc.device)
    hb = (C.c_uint32 * n_cols)(*[int(b) for b in blind]) if blind is not None else None
    check(lib().vs_commit_group_cairo(_ptr(cols_hc), stride, n_cols, log_n, hb,
                                      _ptr(coeffs) if coeffs is not None else None, _ptr(eval_cn),
                                      _ptr(eval_hc) if eval_hc is not None else None, _ptr(root),
                                      _ptr(tile_roots) if tile_roots is not None else None, _stream(stream)),
          "vs_commit_group_cairo")
    return eval_cn, root


class CairoOodsFriIO(C.Structure):
    """Mirror of vs_cairo_oods_fri_io (include/vstark.h)."""
    _fields_ = [
        ("log_n", C.c_uint32), ("n_trace", C.c_uint32), ("n_interaction", C.c_uint32), ("pad", C.c_uint32),
        ("trace_coeffs", C.c_void_p), ("zk_scalars", C.c_void_p), ("trace_evals", C.c_void_p),
        ("interaction_evals", C.c_void_p), ("quotient_hc", C.c_void_p * 4), ("quotient_cn", C.c_void_p * 4),
        ("oods_quotient", C.c_void_p * 4), ("quotient_tile_roots", C.c_void_p), ("oods_tile_roots", C.c_void_p),
        ("trace_at_z", C.c_void_p), ("trace_at_z_next", C.c_void_p), ("interaction_at_z", C.c_void_p),
        ("interaction_at_z_next", C.c_void_p), ("quotient_root", C.c_uint32 * 8), ("oods_point", C.c_uint32 * 8),
        ("quotient_at_z", C.c_uint32 * 16), ("oods_alpha", C.c_uint32 * 4), ("oods_root", C.c_uint32 * 8),
        ("n_fri_roots", C.c_uint32), ("fri_roots", C.c_uint32 * 256), ("fri_alphas", C.c_uint32 * 128),
        ("last_layer", C.c_uint32 * 32), ("last_layer_coeffs", C.c_uint32 * 32),
    ]


def cairo_oods_fri(channel: Channel, log_n: int, trace_coeffs, trace_evals, interaction_evals, quotient_hc,
                   zk_scalars=None, quotient_cn=None, oods_quotient=None, quotient_tile_roots=None,
                   oods_tile_roots=None, stream=None) -> dict:
    """Cairo prover tail after the trace / interaction commitments
    (cairo_air/prover.rs:1937-2438). Column arguments are lists of CUDA tensors;
    the optional outputs are lists of 4 tensors (limbs) or one tensor (tile roots)."""
    nt, ni = len(trace_coeffs), len(interaction_evals)
    u64p = C.c_uint64
    tc = (u64p * nt)(*[_ptr(t) for t in trace_coeffs])
    te = (u64p * nt)(*[_ptr(t) for t in trace_evals])
    ie = (u64p * max(1, ni))(*[_ptr(t) for t in interaction_evals])
    zk = (C.c_uint32 * nt)(*[int(z) for z in zk_scalars]) if zk_scalars is not None else None
    host = {k: (C.c_uint32 * (4 * max(1, m)))() for k, m in
            (("trace_at_z", nt), ("trace_at_z_next", nt), ("interaction_at_z", ni), ("interaction_at_z_next", ni))}
    io = CairoOodsFriIO()
    io.log_n, io.n_trace, io.n_interaction = log_n, nt, ni
    io.trace_coeffs = C.cast(tc, C.c_void_p)
    io.trace_evals = C.cast(te, C.c_void_p)
    io.interaction_evals = C.cast(ie, C.c_void_p)
    io.zk_scalars = C.cast(zk, C.c_void_p) if zk is not None else None
    for k in range(4):
        io.quotient_hc[k] = _ptr(quotient_hc[k])
        io.quotient_cn[k] = _ptr(quotient_cn[k]) if quotient_cn is not None else None
        io.oods_quotient[k] = _ptr(oods_quotient[k]) if oods_quotient is not None else None
    io.quotient_tile_roots = _ptr(quotient_tile_roots) if quotient_tile_roots is not None else None
    io.oods_tile_roots = _ptr(oods_tile_roots) if oods_tile_roots is not None else None
    for k, a in host.items():
        setattr(io, k, C.cast(a, C.c_void_p))
    check(lib().vs_cairo_oods_fri(channel.h, C.byref(io), _stream(stream)), "vs_cairo_oods_fri")

    def q(arr, m):
        return [list(arr[4 * i:4 * i + 4]) for i in range(m)]
    return {
        "quotient_root": list(io.quotient_root), "oods_point": list(io.oods_point),
        "trace_at_z": q(host["trace_at_z"], nt), "trace_at_z_next": q(host["trace_at_z_next"], nt),
        "interaction_at_z": q(host["interaction_at_z"], ni),
        "interaction_at_z_next": q(host["interaction_at_z_next"], ni),
        "quotient_at_z": q(io.quotient_at_z, 4), "oods_alpha": list(io.oods_alpha), "oods_root": list(io.oods_root),
        "fri_roots": [list(io.fri_roots[8 * i:8 * i + 8]) for i in range(io.n_fri_roots)],
        "fri_alphas": q(io.fri_alphas, log_n - 1), "last_layer": q(io.last_layer, 8),
        "last_layer_coeffs": q(io.last_layer_coeffs, 8),
    }


# ------------------------------------------------------------------ stwo wire-format export (src/stwo_export.rs)
class StwoProofParts(C.Structure):
    """Mirror of vs_stwo_proof_parts (include/vstark.h)."""
    _fields_ = [
        ("log_trace_size", C.c_uint32), ("n_queries", C.c_uint32), ("query_indices", C.c_void_p),
        ("pow_nonce", C.c_uint64), ("commitments", (C.c_uint32 * 8) * 7), ("n_trace_cols", C.c_uint32),
        ("trace_values_at_queries", C.c_void_p), ("n_oods", C.c_uint32), ("n_oods_next", C.c_uint32),
        ("oods_trace_at_z", C.c_void_p), ("oods_trace_at_z_next", C.c_void_p),
        ("oods_interaction_at_z", ((C.c_uint32 * 4) * 4) * 3),
        ("oods_interaction_at_z_next", ((C.c_uint32 * 4) * 4) * 3),
        ("oods_quotient_at_z", (C.c_uint32 * 4) * 4), ("trace_auth_paths", C.c_void_p * 3),
        ("trace_auth_paths_next", C.c_void_p * 3), ("decom_values", C.c_void_p * 4),
        ("decom_auth_paths", C.c_void_p * 4), ("oods_quotient_commitment", C.c_uint32 * 8),
        ("oods_quotient_sibling_values", C.c_void_p), ("oods_quotient_auth_paths", C.c_void_p),
        ("n_fri", C.c_uint32), ("fri_commitments", C.c_void_p), ("fri_sibling_values", C.c_void_p),
        ("fri_auth_paths", C.c_void_p), ("n_last", C.c_uint32), ("last_layer_poly", C.c_void_p),
    ]


def stwo_proof_json(parts: dict) -> str:
    """The stwo-compatible JSON proof (cairo_proof_to_json) from proof parts given as
    numpy uint32 arrays (query_indices uint64): keys as in vs_stwo_proof_parts;
    trace_auth_paths / trace_auth_paths_next / decom_values / decom_auth_paths are
    lists (None entries allowed for the next-row paths); fri_sibling_values and
    fri_auth_paths are lists of per-layer arrays."""
    import numpy as np
    keep = []

    def arr(a, dtype=np.uint32):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype)
        keep.append(a)
        return a.ctypes.data

    p = StwoProofParts()
    q = np.ascontiguousarray(parts["query_indices"], np.uint64)
    p.log_trace_size, p.n_queries, p.query_indices = parts["log_trace_size"], len(q), arr(q, np.uint64)
    p.pow_nonce = int(parts.get("pow_nonce", 0))
    for t, h in enumerate(parts["commitments"]):
        p.commitments[t][:] = [int(x) for x in h]
    tv = np.ascontiguousarray(parts["trace_values_at_queries"], np.uint32)
    p.n_trace_cols, p.trace_values_at_queries = (tv.shape[1] if tv.ndim == 2 else 0), arr(tv)
    z, zn = parts.get("oods_trace_at_z"), parts.get("oods_trace_at_z_next")
    p.n_oods = 0 if z is None else len(z)
    p.n_oods_next = 0 if zn is None else len(zn)
    p.oods_trace_at_z, p.oods_trace_at_z_next = arr(z), arr(zn)
    for name in ("oods_interaction_at_z", "oods_interaction_at_z_next"):
        v = np.zeros((3, 4, 4), np.uint32) if parts.get(name) is None else np.asarray(parts[name], np.uint32)
        for a in range(3):
            for b in range(4):
                getattr(p, name)[a][b][:] = [int(x) for x in v[a, b]]
    qz = np.zeros((4, 4), np.uint32) if parts.get("oods_quotient_at_z") is None else np.asarray(parts["oods_quotient_at_z"])
    for a in range(4):
        p.oods_quotient_at_z[a][:] = [int(x) for x in qz[a]]
    for t in range(3):
        p.trace_auth_paths[t] = arr(parts["trace_auth_paths"][t])
        nxt = parts.get("trace_auth_paths_next")
        p.trace_auth_paths_next[t] = arr(nxt[t]) if nxt is not None else None
    for t in range(4):
        p.decom_values[t] = arr(parts["decom_values"][t])
        p.decom_auth_paths[t] = arr(parts["decom_auth_paths"][t])
    p.oods_quotient_commitment[:] = [int(x) for x in parts["oods_quotient_commitment"]]
    p.oods_quotient_sibling_values = arr(parts["oods_quotient_sibling_values"])
    p.oods_quotient_auth_paths = arr(parts["oods_quotient_auth_paths"])
    fc = parts.get("fri_commitments", [])
    p.n_fri, p.fri_commitments = len(fc), arr(np.asarray(fc, np.uint32).reshape(-1, 8) if len(fc) else None)
    sv = [arr(x) for x in parts.get("fri_sibling_values", [])]
    ap = [arr(x) for x in parts.get("fri_auth_paths", [])]
    sva, apa = (C.c_void_p * max(1, len(sv)))(*sv), (C.c_void_p * max(1, len(ap)))(*ap)
    p.fri_sibling_values, p.fri_auth_paths = C.cast(sva, C.c_void_p), C.cast(apa, C.c_void_p)
    last = parts.get("last_layer_poly")
    p.n_last, p.last_layer_poly = (0 if last is None else len(last)), arr(last)
    n = C.c_uint64()
    check(lib().vs_stwo_proof_json(C.byref(p), None, 0, C.byref(n)), "vs_stwo_proof_json")
    buf = C.create_string_buffer(n.value + 1)
    check(lib().vs_stwo_proof_json(C.byref(p), buf, n.value + 1, C.byref(n)), "vs_stwo_proof_json")
    return buf.raw[: n.value].decode()
