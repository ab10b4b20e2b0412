"""ctypes bindings to the CPU oracle (oracle/_build/liboracle.so).

Test infrastructure: the parity checker for the CUDA path and the CPU baseline.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
ORACLE_SO = ROOT / "oracle" / "_build" / "liboracle.so"
REF_SO = ROOT / "oracle" / "_ref" / "libvortex_ref.so"
P = 0x7FFFFFFF

_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists():
            build()
        _lib = C.CDLL(str(ORACLE_SO))
        _declare(_lib)
    return _lib


u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)
u8p = C.POINTER(C.c_uint8)


def _declare(L: C.CDLL) -> None:
    L.oracle_prove.restype = C.c_uint64
    L.oracle_ch_draw_number.restype = C.c_uint64
    L.oracle_pow_grind_min.restype = C.c_uint64
    L.oracle_pow_trailing_zeros.restype = C.c_uint32
    L.oracle_coset_vanishing_half_coset.restype = C.c_uint32
    L.oracle_m31_mul.restype = C.c_uint32
    L.oracle_m31_inv.restype = C.c_uint32
    L.oracle_bench_commit.restype = C.c_double
    L.oracle_bench_fri.restype = C.c_double
    L.oracle_verify.restype = C.c_int


def ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    if a.dtype == np.uint32:
        return a.ctypes.data_as(u32p)
    if a.dtype == np.uint64:
        return a.ctypes.data_as(u64p)
    if a.dtype == np.uint8:
        return a.ctypes.data_as(u8p)
    raise TypeError(a.dtype)


def ptr_array(arrs):
    """A C array of uint32_t* pointing at the given numpy arrays."""
    return (u32p * len(arrs))(*[ptr(a) for a in arrs])


# ----------------------------------------------------------------- field / circle
def coset(kind: int, log_n: int):
    o = np.zeros(4, np.uint32)
    lib().oracle_coset(kind, log_n, ptr(o))
    return [int(x) for x in o]


HALF_COSET, HALF_ODDS, SUBGROUP = 0, 1, 2


def seeded_m31(seed: int, n: int, offset: int = 0) -> np.ndarray:
    o = np.empty(n, np.uint32)
    lib().oracle_seeded_m31(C.c_uint64(seed), C.c_uint64(offset), C.c_uint64(n), ptr(o))
    return o


# ----------------------------------------------------------------- NTT
def native_twiddles(log_n: int, kind: int = HALF_COSET):
    n = 1 << log_n
    line = np.zeros(n - 1, np.uint32)
    iline = np.zeros(n - 1, np.uint32)
    circ = np.zeros(n // 2, np.uint32)
    icirc = np.zeros(n // 2, np.uint32)
    offs = np.zeros(max(log_n - 1, 1), np.uint32)
    sizes = np.zeros(max(log_n - 1, 1), np.uint32)
    lib().oracle_native_twiddles(kind, log_n, ptr(line), ptr(circ), ptr(iline), ptr(icirc), ptr(offs), ptr(sizes))
    return dict(line=line, circle=circ, iline=iline, icircle=icirc, offsets=offs[: log_n - 1], sizes=sizes[: log_n - 1])


def native_evaluate(d: np.ndarray, log_n: int) -> np.ndarray:
    d = np.ascontiguousarray(d, np.uint32).copy()
    lib().oracle_native_evaluate(ptr(d), log_n)
    return d


def native_interpolate(d: np.ndarray, log_n: int) -> np.ndarray:
    d = np.ascontiguousarray(d, np.uint32).copy()
    lib().oracle_native_interpolate(ptr(d), log_n)
    return d


def ntt_layer(d: np.ndarray, tw: np.ndarray, layer_idx: int, forward: bool) -> np.ndarray:
    d = np.ascontiguousarray(d, np.uint32).copy()
    lib().oracle_ntt_layer(ptr(d), C.c_uint64(d.size), ptr(np.ascontiguousarray(tw, np.uint32)), layer_idx, int(forward))
    return d


def stwo_twiddles(log_n: int):
    n = 1 << log_n
    f = np.zeros(n // 2, np.uint32)
    i = np.zeros(n // 2, np.uint32)
    lib().oracle_stwo_twiddles(log_n, ptr(f), ptr(i))
    return f, i


def stwo_evaluate(d: np.ndarray, log_n: int) -> np.ndarray:
    d = np.ascontiguousarray(d, np.uint32).copy()
    lib().oracle_stwo_evaluate(ptr(d), log_n)
    return d


def stwo_interpolate(d: np.ndarray, log_n: int) -> np.ndarray:
    d = np.ascontiguousarray(d, np.uint32).copy()
    lib().oracle_stwo_interpolate(ptr(d), log_n)
    return d


def stwo_lde_columns(cols: np.ndarray, log_n: int, blowup: int = 2, threads: int = 1) -> np.ndarray:
    cols = np.ascontiguousarray(cols, np.uint32)
    nc = cols.shape[0]
    out = np.empty((nc, 1 << (log_n + blowup)), np.uint32)
    lib().oracle_stwo_lde_columns(ptr(cols), nc, log_n, blowup, ptr(out), threads)
    return out


def zh_eval_domain(log_n: int) -> np.ndarray:
    """Z_H of half_coset(log_n) at the BRT-canonic points of the 4x evaluation domain."""
    out = np.empty(1 << (log_n + 2), np.uint32)
    lib().oracle_zh_eval_domain(log_n, ptr(out))
    return out


def coset_vanishing_half_coset(log_n: int, x: int, y: int) -> int:
    return int(lib().oracle_coset_vanishing_half_coset(log_n, x, y))


def commit_group_cairo(cols_hc: np.ndarray, log_n: int, blind=None, threads: int = 8) -> dict:
    """One Cairo column group: coefficients, blinded BRT-canonic LDE, its half-coset
    copy, the capped-leaf root and the 1024-leaf tile roots."""
    cols_hc = np.ascontiguousarray(cols_hc, np.uint32)
    nc, n = cols_hc.shape
    N = n << 2
    b = np.zeros(nc, np.uint32) if blind is None else np.ascontiguousarray(blind, np.uint32)
    coeffs = np.empty((nc, n), np.uint32)
    ev_cn, ev_hc = np.empty((nc, N), np.uint32), np.empty((nc, N), np.uint32)
    root = np.empty(8, np.uint32)
    tiles = np.empty((max(1, N // 1024), 8), np.uint32)
    lib().oracle_commit_group_cairo(ptr(cols_hc), nc, log_n, ptr(b), ptr(coeffs), ptr(ev_cn), ptr(ev_hc), ptr(root),
                                    ptr(tiles), threads)
    return {"coeffs": coeffs, "eval_cn": ev_cn, "eval_hc": ev_hc, "root": root, "tile_roots": tiles}


def tree_paths(kind: int, cols: np.ndarray, idx) -> np.ndarray:
    """Auth paths (n_idx, log_n, 8) of a capped-leaf (kind 0) or SoA4 (kind 1) tree."""
    cols = np.ascontiguousarray(cols, np.uint32)
    nc, n = cols.shape
    log_n = n.bit_length() - 1
    ix = np.ascontiguousarray(idx, np.uint64)
    out = np.zeros((len(ix), max(log_n, 1), 8), np.uint32)
    lib().oracle_tree_paths(kind, ptr(cols), nc, log_n, ptr(ix), len(ix), ptr(out), 1)
    return out[:, :log_n]


def bit_reverse(d: np.ndarray, log_n: int) -> np.ndarray:
    d = np.ascontiguousarray(d, np.uint32).copy()
    lib().oracle_bit_reverse(ptr(d), log_n)
    return d


def batch_inverse(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, np.uint32)
    o = np.empty_like(x)
    lib().oracle_batch_inverse(ptr(x), ptr(o), C.c_uint64(x.size))
    return o


def coset_points(init_x, init_y, step_x, step_y, n):
    ox = np.empty(n, np.uint32)
    oy = np.empty(n, np.uint32)
    lib().oracle_coset_points(init_x, init_y, step_x, step_y, C.c_uint64(n), ptr(ox), ptr(oy))
    return ox, oy


# ----------------------------------------------------------------- hashing / Merkle
def blake2s_words(w: np.ndarray) -> np.ndarray:
    w = np.ascontiguousarray(w, np.uint32)
    o = np.empty(8, np.uint32)
    lib().oracle_blake2s_words(ptr(w), C.c_uint64(w.size), ptr(o))
    return o


def blake2s_bytes(b: bytes) -> bytes:
    a = np.frombuffer(b, np.uint8).copy() if b else np.zeros(1, np.uint8)
    o = np.empty(32, np.uint8)
    lib().oracle_blake2s_bytes(ptr(a), C.c_uint64(len(b)), ptr(o))
    return o.tobytes()


def leaf_hashes_capped(cols: np.ndarray) -> np.ndarray:
    cols = np.ascontiguousarray(cols, np.uint32)
    nc, n = cols.shape
    o = np.empty((n, 8), np.uint32)
    lib().oracle_leaf_hashes_capped(ptr(cols), nc, C.c_uint64(n), ptr(o))
    return o


def hash_nodes(children: np.ndarray) -> np.ndarray:
    children = np.ascontiguousarray(children, np.uint32).reshape(-1)
    n_par = children.size // 16
    o = np.empty((n_par, 8), np.uint32)
    lib().oracle_hash_nodes(ptr(children), C.c_uint64(n_par), ptr(o))
    return o


def merkle_root_hashes(h: np.ndarray) -> np.ndarray:
    h = np.ascontiguousarray(h, np.uint32)
    o = np.empty(8, np.uint32)
    lib().oracle_merkle_root_hashes(ptr(h), C.c_uint64(h.size // 8), ptr(o))
    return o


def merkle_root_capped(cols: np.ndarray, threads: int = 1) -> np.ndarray:
    cols = np.ascontiguousarray(cols, np.uint32)
    o = np.empty(8, np.uint32)
    lib().oracle_merkle_root_capped(ptr(cols), cols.shape[0], C.c_uint64(cols.shape[1]), threads, ptr(o))
    return o


def merkle_root_rowpacked(cols: np.ndarray, threads: int = 1) -> np.ndarray:
    cols = np.ascontiguousarray(cols, np.uint32)
    o = np.empty(8, np.uint32)
    lib().oracle_merkle_root_rowpacked(ptr(cols), cols.shape[0], C.c_uint64(cols.shape[1]), threads, ptr(o))
    return o


def merkle_root_soa4(c: np.ndarray, threads: int = 1) -> np.ndarray:
    c = np.ascontiguousarray(c, np.uint32)
    o = np.empty(8, np.uint32)
    lib().oracle_merkle_root_soa4(ptr(c[0]), ptr(c[1]), ptr(c[2]), ptr(c[3]), C.c_uint64(c.shape[1]), threads, ptr(o))
    return o


def lifted_leaves(cols, col_logs, lifting_log) -> np.ndarray:
    cols = [np.ascontiguousarray(c, np.uint32) for c in cols]
    logs = np.asarray(col_logs, np.uint32)
    o = np.empty((1 << lifting_log, 8), np.uint32)
    lib().oracle_lifted_leaves(ptr_array(cols), ptr(logs), len(cols), lifting_log, ptr(o))
    return o


# ----------------------------------------------------------------- channel
class ChState(C.Structure):
    _fields_ = [("state", C.c_uint8 * 32), ("n_draws", C.c_uint32)]


class Channel:
    def __init__(self):
        self.s = ChState()

    def mix_digest(self, d):
        a = np.ascontiguousarray(d, np.uint32)
        lib().oracle_ch_mix_digest(C.byref(self.s), ptr(a))

    def mix_felts(self, felts):
        a = np.ascontiguousarray(felts, np.uint32).reshape(-1)
        lib().oracle_ch_mix_felts(C.byref(self.s), ptr(a), C.c_uint64(a.size // 4))

    def mix_u64(self, v):
        lib().oracle_ch_mix_u64(C.byref(self.s), C.c_uint64(v))

    def draw_felt(self):
        o = np.empty(4, np.uint32)
        lib().oracle_ch_draw_felt(C.byref(self.s), ptr(o))
        return o

    def draw_number(self, bound):
        return int(lib().oracle_ch_draw_number(C.byref(self.s), C.c_uint64(bound)))

    def draw_queries(self, log_domain, n):
        o = np.empty(n, np.uint64)
        lib().oracle_ch_draw_queries(C.byref(self.s), log_domain, C.c_uint64(n), ptr(o))
        return o

    def state_bytes(self) -> bytes:
        return bytes(self.s.state)

    def pow_prefix(self, pow_bits: int) -> np.ndarray:
        o = np.empty(8, np.uint32)
        lib().oracle_ch_pow_prefix(C.byref(self.s), pow_bits, ptr(o))
        return o

    def verify_pow(self, pow_bits: int, nonce: int) -> bool:
        return bool(lib().oracle_ch_verify_pow(C.byref(self.s), pow_bits, C.c_uint64(nonce)))

    def oods_point(self):
        o = np.empty(8, np.uint32)
        lib().oracle_oods_point(C.byref(self.s), ptr(o))
        return o


def cairo_oods_fri(ch: "Channel", log_n: int, trace_coeffs, zk, trace_evals, inter_evals, quot_hc,
                   threads: int = 8) -> dict:
    """Cairo prover tail (quotient commitment, OODS, DEEP quotient, FRI); advances ch."""
    n, N = 1 << log_n, 4 << log_n
    tc = np.ascontiguousarray(trace_coeffs, np.uint32).reshape(-1, n)
    nt = tc.shape[0]
    te = np.ascontiguousarray(trace_evals, np.uint32).reshape(nt, N)
    ie = np.ascontiguousarray(inter_evals, np.uint32).reshape(-1, N)
    ni = ie.shape[0]
    qh = np.ascontiguousarray(quot_hc, np.uint32).reshape(4, N)
    z = np.zeros(nt, np.uint32) if zk is None else np.ascontiguousarray(zk, np.uint32)
    nt_ = max(1, N // 1024)
    out = {
        "quotient_root": np.empty(8, np.uint32), "quotient_tiles": np.empty((nt_, 8), np.uint32),
        "oods_point": np.empty(8, np.uint32), "trace_at_z": np.empty((nt, 4), np.uint32),
        "trace_at_z_next": np.empty((nt, 4), np.uint32), "interaction_at_z": np.empty((max(ni, 1), 4), np.uint32),
        "interaction_at_z_next": np.empty((max(ni, 1), 4), np.uint32), "quotient_at_z": np.empty((4, 4), np.uint32),
        "oods_alpha": np.empty(4, np.uint32), "oods_quotient": np.empty((4, N), np.uint32),
        "oods_root": np.empty(8, np.uint32), "oods_tiles": np.empty((nt_, 8), np.uint32),
        "fri_roots": np.empty((max(log_n - 2, 1), 8), np.uint32), "fri_alphas": np.empty((log_n - 1, 4), np.uint32),
        "last_layer": np.empty((8, 4), np.uint32), "last_layer_coeffs": np.empty((8, 4), np.uint32),
    }
    o = out
    lib().oracle_cairo_oods_fri(C.byref(ch.s), log_n, ptr(tc), nt, ptr(z), ptr(te), ptr(ie if ni else np.zeros(1, np.uint32)),
                                ni, ptr(qh), ptr(o["quotient_root"]), ptr(o["quotient_tiles"]), ptr(o["oods_point"]),
                                ptr(o["trace_at_z"]), ptr(o["trace_at_z_next"]), ptr(o["interaction_at_z"]),
                                ptr(o["interaction_at_z_next"]), ptr(o["quotient_at_z"]), ptr(o["oods_alpha"]),
                                ptr(o["oods_quotient"]), ptr(o["oods_root"]), ptr(o["oods_tiles"]), ptr(o["fri_roots"]),
                                ptr(o["fri_alphas"]), ptr(o["last_layer"]), ptr(o["last_layer_coeffs"]), threads)
    out["interaction_at_z"] = out["interaction_at_z"][:ni]
    out["interaction_at_z_next"] = out["interaction_at_z_next"][:ni]
    out["fri_roots"] = out["fri_roots"][: log_n - 2]
    return out


def pow_trailing_zeros(prefix, nonce: int, m31_output: bool = False) -> int:
    a = np.ascontiguousarray(prefix, np.uint32)
    return int(lib().oracle_pow_trailing_zeros(ptr(a), C.c_uint64(nonce), int(m31_output)))


def pow_grind_min(prefix, pow_bits: int, offset: int, n: int, m31_output: bool = False, threads: int = 0) -> int:
    """Smallest nonce in [offset, offset + n) meeting pow_bits, or 2^64 - 1."""
    a = np.ascontiguousarray(prefix, np.uint32)
    return int(lib().oracle_pow_grind_min(ptr(a), pow_bits, C.c_uint64(offset), C.c_uint64(n), int(m31_output),
                                          threads or (os.cpu_count() or 1)))


# ----------------------------------------------------------------- FRI / quotient
def fold_twiddles(kind: int, log_n: int, extract_y: bool) -> np.ndarray:
    o = np.empty(1 << (log_n - 1), np.uint32)
    lib().oracle_fold_twiddles(kind, log_n, int(extract_y), ptr(o))
    return o


def canonic_domain_points(log_size: int):
    xs = np.empty(1 << log_size, np.uint32)
    ys = np.empty(1 << log_size, np.uint32)
    lib().oracle_canonic_domain_points(log_size, ptr(xs), ptr(ys))
    return xs, ys


def fold_twiddles_generic(ix, iy, sx, sy, log_n, extract_y) -> np.ndarray:
    o = np.empty(1 << (log_n - 1), np.uint32)
    lib().oracle_fold_twiddles_generic(ix, iy, sx, sy, log_n, int(extract_y), ptr(o))
    return o


def fold_circle_into_line(dst: np.ndarray, src: np.ndarray, tw, alpha, alpha_sq) -> np.ndarray:
    dst = np.ascontiguousarray(dst, np.uint32).copy()
    src = np.ascontiguousarray(src, np.uint32)
    a = np.asarray(alpha, np.uint32)
    a2 = np.asarray(alpha_sq, np.uint32)
    lib().oracle_fold_circle_into_line(ptr_array(list(dst)), ptr_array(list(src)), ptr(np.ascontiguousarray(tw, np.uint32)),
                                       ptr(a), ptr(a2), C.c_uint64(dst.shape[1]))
    return dst


def fold_line(src: np.ndarray, tw, alpha) -> np.ndarray:
    src = np.ascontiguousarray(src, np.uint32)
    out = np.zeros((4, src.shape[1] // 2), np.uint32)
    a = np.asarray(alpha, np.uint32)
    lib().oracle_fold_line(ptr_array(list(src)), ptr(np.ascontiguousarray(tw, np.uint32)), ptr_array(list(out)), ptr(a),
                           C.c_uint64(out.shape[1]))
    return out


def last_layer_poly_coeffs(evals) -> np.ndarray:
    e = np.ascontiguousarray(evals, np.uint32)
    o = np.empty((8, 4), np.uint32)
    lib().oracle_last_layer_poly_coeffs(ptr(e), C.c_uint64(e.shape[0]), ptr(o))
    return o


def eval_last_layer_poly(coeffs, idx, log_size) -> np.ndarray:
    c = np.ascontiguousarray(coeffs, np.uint32)
    o = np.empty(4, np.uint32)
    lib().oracle_eval_last_layer_poly(ptr(c), C.c_uint64(c.shape[0]), C.c_uint64(idx), log_size, ptr(o))
    return o


def fib_quotient(trace: np.ndarray, alpha) -> np.ndarray:
    trace = np.ascontiguousarray(trace, np.uint32)
    out = np.zeros((4, trace.size), np.uint32)
    lib().oracle_fib_quotient(ptr(trace), C.c_uint64(trace.size), ptr(np.asarray(alpha, np.uint32)), ptr_array(list(out)))
    return out


def accumulate_numerators(cols, col_idx, b, c, n_rows) -> np.ndarray:
    cols = [np.ascontiguousarray(x, np.uint32) for x in cols]
    out = np.zeros((4, n_rows), np.uint32)
    lib().oracle_accumulate_numerators(ptr_array(cols), ptr(np.asarray(col_idx, np.uint32)),
                                       ptr(np.ascontiguousarray(b, np.uint32)), ptr(np.ascontiguousarray(c, np.uint32)),
                                       len(col_idx), C.c_uint64(n_rows), ptr_array(list(out)))
    return out


def quotients_combine(spx, spy, fla, numers, acc_logs, dxs, dys, lifting_log) -> np.ndarray:
    n_rows = dxs.size
    out = np.zeros((4, n_rows), np.uint32)
    numers = [np.ascontiguousarray(x, np.uint32) for x in numers]
    n0 = ptr_array([x[0] for x in numers])
    n1 = ptr_array([x[1] for x in numers])
    n2 = ptr_array([x[2] for x in numers])
    n3 = ptr_array([x[3] for x in numers])
    lib().oracle_quotients_combine(ptr(np.ascontiguousarray(spx, np.uint32)), ptr(np.ascontiguousarray(spy, np.uint32)),
                                   ptr(np.ascontiguousarray(fla, np.uint32)), n0, n1, n2, n3,
                                   ptr(np.asarray(acc_logs, np.uint32)), len(numers), ptr(dxs), ptr(dys), lifting_log,
                                   C.c_uint64(n_rows), ptr_array(list(out)))
    return out


def eval_at_oods(coeffs, z8) -> np.ndarray:
    c = np.ascontiguousarray(coeffs, np.uint32)
    o = np.empty(4, np.uint32)
    lib().oracle_eval_at_oods(ptr(c), C.c_uint64(c.size), ptr(np.ascontiguousarray(z8, np.uint32)), ptr(o))
    return o


def line_coeffs(z8, v):
    a = np.empty(4, np.uint32)
    b = np.empty(4, np.uint32)
    lib().oracle_line_coeffs(ptr(np.ascontiguousarray(z8, np.uint32)), ptr(np.ascontiguousarray(v, np.uint32)), ptr(a), ptr(b))
    return a, b


# ----------------------------------------------------------------- prover
def fib_trace(a, b, log_n) -> np.ndarray:
    o = np.empty(1 << log_n, np.uint32)
    lib().oracle_fib_trace(a, b, log_n, ptr(o))
    return o


def prove(a: int, b: int, log_n: int, threads: int = 0) -> bytes:
    threads = threads or (os.cpu_count() or 1)
    cap = 32 << 20  # every proof up to log_n = 30 fits; proving twice would double the cost
    buf = np.empty(cap, np.uint8)
    n = lib().oracle_prove(a, b, log_n, threads, ptr(buf), C.c_uint64(cap))
    if n > cap:
        buf = np.empty(n, np.uint8)
        lib().oracle_prove(a, b, log_n, threads, ptr(buf), C.c_uint64(n))
    return buf[:n].tobytes()


def verify(proof: bytes):
    a = np.frombuffer(proof, np.uint8).copy()
    err = C.create_string_buffer(256)
    rc = lib().oracle_verify(ptr(a), C.c_uint64(a.size), err, C.c_uint64(256))
    return rc, err.value.decode()


# --- stwo Backend adapter kernels (gather.cu, barycentric_eval.cu, accumulate_lift.cu, pack_leaves.cu)
def gather_u32(src: np.ndarray, idx: np.ndarray) -> np.ndarray:
    src = np.ascontiguousarray(src, np.uint32)
    idx = np.ascontiguousarray(idx, np.uint32)
    out = np.zeros(max(idx.size, 1), np.uint32)
    lib().oracle_gather_u32(ptr(src), ptr(idx), ptr(out), C.c_uint64(idx.size))
    return out[: idx.size]


def gather_u256(src: np.ndarray, idx: np.ndarray) -> np.ndarray:
    src = np.ascontiguousarray(src, np.uint32)
    idx = np.ascontiguousarray(idx, np.uint32)
    out = np.zeros(max(8 * idx.size, 1), np.uint32)
    lib().oracle_gather_u256(ptr(src), ptr(idx), ptr(out), C.c_uint64(idx.size))
    return out[: 8 * idx.size]


def barycentric_partials(evals: np.ndarray, weights: np.ndarray, n_blocks: int) -> np.ndarray:
    """(n_blocks, 4) partial sums; weights are QM31 AoS (4 words per element)."""
    evals = np.ascontiguousarray(evals, np.uint32)
    weights = np.ascontiguousarray(weights, np.uint32)
    out = np.zeros((max(n_blocks, 1), 4), np.uint32)
    lib().oracle_barycentric_partials(ptr(evals), ptr(weights), C.c_uint64(evals.size), C.c_uint32(n_blocks), ptr(out))
    return out[:n_blocks]


def accumulate_lift(col: np.ndarray, curr: np.ndarray, log_ratio: int) -> np.ndarray:
    """col (col_n*4 words, QM31 AoS) after col[i] += curr[src(i)]; returns a new array."""
    col = np.ascontiguousarray(col, np.uint32).copy()
    curr = np.ascontiguousarray(curr, np.uint32)
    lib().oracle_accumulate_lift(ptr(col), ptr(curr), C.c_uint64(col.size // 4), C.c_uint32(log_ratio))
    return col


def pack_leaves(cols: np.ndarray) -> np.ndarray:
    """cols (4, n) -> (64, ceil(n/16)); words past the end of a short last group stay 0."""
    cols = np.ascontiguousarray(cols, np.uint32)
    n = cols.shape[1]
    out_len = (n + 15) // 16
    out = np.zeros((64, max(out_len, 1)), np.uint32)
    lib().oracle_pack_leaves(ptr(cols), C.c_uint64(n), ptr(out), C.c_uint64(max(out_len, 1)))
    return out[:, :out_len]
