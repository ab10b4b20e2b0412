#!/usr/bin/env python3
"""Generates tests/golden/ref_golden.npz from the reference's own CUDA kernels.

Runs on a CUDA machine with oracle/_ref/libvortex_ref.so (built from the
reference's kernel sources by oracle/build_ref.sh). It records the reference
kernels' outputs on seeded inputs, and whole Fibonacci proofs produced by a
Python restatement of the reference prover's stage order (src/prover.rs:1721-1978)
that calls only reference kernels for the arithmetic and hashlib Blake2s for the
Fiat-Shamir channel (src/channel.rs). tests/test_golden.py checks the CPU oracle
against these fixtures without a GPU.

    python tests/golden/gen_ref_golden.py [out.npz]
"""
from __future__ import annotations

import ctypes as C
import hashlib
import struct
import sys
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
REF_SO = ROOT / "oracle" / "_ref" / "libvortex_ref.so"
P = 0x7FFFFFFF
G = (2, 1268011823)

R = None


def u32(v):
    return C.c_uint32(int(v))


KEEP = []  # tensors whose raw pointers were handed to a kernel (see keep-alive note in main)


def vp(t):
    KEEP.append(t)
    return C.c_void_p(t.data_ptr())


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.uint32).view(np.int32).copy()).cuda()


def empty(n):
    return torch.empty(int(max(n, 1)), dtype=torch.int32, device="cuda")


def zeros(n):
    return torch.zeros(int(max(n, 1)), dtype=torch.int32, device="cuda")


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy().view(np.uint32).copy()


def hostarr(vals):
    vals = [int(v) for v in vals]
    return (C.c_uint32 * len(vals))(*vals)


def ptrs(ts):
    ts = list(ts)
    KEEP.extend(ts)
    return torch.tensor([t.data_ptr() for t in ts], dtype=torch.int64, device="cuda")


# ------------------------------------------------------------------ circle group (circle.rs)
def pmul(a, b):
    return ((a[0] * b[0] - a[1] * b[1]) % P, (a[0] * b[1] + a[1] * b[0]) % P)


def rdouble(p, k):
    for _ in range(k):
        p = pmul(p, p)
    return p


def ppow(p, e):
    r = (1, 0)
    while e:
        if e & 1:
            r = pmul(r, p)
        p = pmul(p, p)
        e >>= 1
    return r


def half_coset(l):
    return rdouble(G, 30 - l), rdouble(G, 31 - l)


def half_odds(l):
    return rdouble(G, max(0, 29 - l)), rdouble(G, 31 - l)


def seeded(seed, n):
    rng = np.random.default_rng(seed)
    return rng.integers(0, P, n, dtype=np.uint64).astype(np.uint32)


# ------------------------------------------------------------------ reference host orchestration
def native_twiddles(log_n):
    """circle.rs:277-340 with the reference kernels."""
    (ix, iy), (sx, sy) = half_coset(log_n)
    n = 1 << log_n
    dx, dy = empty(n), empty(n)
    R.cuda_compute_coset_points(u32(ix), u32(iy), u32(sx), u32(sy), vp(dx), vp(dy), u32(n))
    line = zeros(n - 1)
    cur, cur_n, off, offs = dx, n, 0, []
    for _ in range(log_n - 1):
        ls = cur_n // 2
        sq = empty(ls)
        offs.append(off)
        R.cuda_extract_and_squash(vp(cur), C.c_void_p(line.data_ptr() + 4 * off), vp(sq), u32(ls))
        off += ls
        cur, cur_n = sq, ls
    iline, icirc = empty(n - 1), empty(n // 2)
    circ = dy[: n // 2].clone()
    R.cuda_batch_inverse_m31(vp(line), vp(iline), u32(n - 1))
    R.cuda_batch_inverse_m31(vp(circ), vp(icirc), u32(n // 2))
    torch.cuda.synchronize()
    return line, circ, iline, icirc, offs


def fold_twiddles(coset, log_n, extract_y):
    (ix, iy), (sx, sy) = coset
    half = 1 << (log_n - 1)
    src, out = empty(half), empty(half)
    R.cuda_compute_fold_twiddle_sources(u32(ix), u32(iy), u32(sx), u32(sy), vp(src), u32(1 << log_n), u32(log_n),
                                        C.c_int(int(extract_y)))
    R.cuda_batch_inverse_m31(vp(src), vp(out), u32(half))
    return out


def b2s(data: bytes) -> bytes:
    return hashlib.blake2s(data, digest_size=32).digest()


class Channel:  # channel.rs:15-185
    def __init__(self):
        self.state, self.n = bytes(32), 0

    def mix_digest(self, words):
        self.state = b2s(self.state + struct.pack("<8I", *words))
        self.n = 0

    def mix_felts(self, felts):
        self.state = b2s(self.state + b"".join(struct.pack("<4I", *f) for f in felts))
        self.n = 0

    def squeeze(self):
        out = b2s(self.state + struct.pack("<I", self.n) + b"\x00")
        self.n += 1
        return out

    def draw_felt(self):
        while True:
            w = struct.unpack("<8I", self.squeeze())
            if all(x < 2 * P for x in w):
                return [x % P for x in w[:4]]

    def draw_number(self, bound):
        return struct.unpack("<Q", self.squeeze()[:8])[0] % bound


def commit_layers(leaf_fn, n):
    """MerkleTree::commit layout (merkle.rs:28-104): returns host layers leaves..root."""
    leaves = empty(8 * n)
    leaf_fn(leaves)
    layers = [leaves]
    cur, size = leaves, n
    while size > 1:
        par = empty(8 * (size // 2))
        R.cuda_merkle_hash_nodes(vp(cur), vp(par), u32(size // 2))
        layers.append(par)
        cur, size = par, size // 2
    return [host(l).reshape(-1, 8) for l in layers]


def path(layers, idx):
    out = []
    for lay in layers[:-1]:
        out.append([int(x) for x in lay[idx ^ 1]])
        idx //= 2
    return out


def soa4_leaf_fn(cols):
    def fn(out):
        R.cuda_merkle_hash_leaves(vp(ptrs(cols)), vp(out), u32(4), u32(cols[0].numel()))
    return fn


def ref_prove(a, b, log_n):
    """src/prover.rs prove_with_cache stage order with reference kernels; KRAK bytes."""
    log_eval = log_n + 2
    n, N = 1 << log_n, 1 << log_eval
    tr = np.zeros(n, np.uint32)
    tr[0], tr[1] = a, b
    for i in range(2, n):
        tr[i] = (int(tr[i - 1]) + int(tr[i - 2])) % P
    d = dev(tr)
    _, _, il, ic, offs = native_twiddles(log_n)
    R.cuda_circle_ntt_interpolate(vp(d), vp(il), vp(ic), hostarr(offs), hostarr(offs), u32(log_n - 1), u32(n))
    ev = empty(N)
    R.cuda_zero_pad(vp(d), vp(ev), u32(n), u32(N))
    fl, fc, _, _, eoffs = native_twiddles(log_eval)
    R.cuda_circle_ntt_evaluate(vp(ev), vp(fl), vp(fc), hostarr(eoffs), hostarr(eoffs), u32(log_eval - 1), u32(N))
    trace_layers = commit_layers(lambda out: R.cuda_merkle_hash_leaves(vp(ptrs([ev])), vp(out), u32(1), u32(N)), N)
    ch = Channel()
    ch.mix_digest(trace_layers[-1][0])
    alpha = ch.draw_felt()
    q = [empty(N) for _ in range(4)]
    R.cuda_fibonacci_quotient(vp(ev), *[vp(x) for x in q], hostarr(alpha), u32(N))
    quot_layers = commit_layers(soa4_leaf_fn(q), N)
    ch.mix_digest(quot_layers[-1][0])
    fri_vals, fri_layers, fri_roots = [], [], []
    cur = log_eval
    src = q
    while cur > 3:
        fa = ch.draw_felt()
        half = 1 << (cur - 1)
        dst = [zeros(half) for _ in range(4)]
        if cur == log_eval:
            tw = fold_twiddles(half_coset(cur), cur, True)
            a2 = [int(x) for x in gpu_qmul(fa, fa)]
            R.cuda_fold_circle_into_line_soa(*[vp(x) for x in dst], *[vp(x) for x in src], vp(tw), hostarr(fa),
                                             hostarr(a2), u32(half))
        else:
            tw = fold_twiddles(half_odds(cur), cur, False)
            R.cuda_fold_line_soa(*[vp(x) for x in src], vp(tw), *[vp(x) for x in dst], hostarr(fa), u32(half))
        lay = commit_layers(soa4_leaf_fn(dst), half)
        fri_roots.append([int(x) for x in lay[-1][0]])
        ch.mix_digest(lay[-1][0])
        fri_layers.append(lay)
        fri_vals.append(np.stack([host(x) for x in dst]))
        src = dst
        cur -= 1
    last = [[int(x) for x in fri_vals[-1][:, i]] for i in range(8)]
    ch.mix_felts(last)
    queries = [ch.draw_number(N) for _ in range(80)]
    e_h = host(ev)
    q_h = np.stack([host(x) for x in q])
    w = bytearray()

    def w32(*vals):
        for v in vals:
            w.extend(struct.pack("<I", int(v)))

    def wpaths(ps):
        for p in ps:
            w32(len(p))
            for hh in p:
                w32(*hh)

    w32(0x4B52414B, 1, log_n, a, b, *trace_layers[-1][0], *quot_layers[-1][0], len(fri_roots))
    for r in fri_roots:
        w32(*r)
    w32(len(last))
    for v in last:
        w32(*v)
    w32(len(queries), *queries)
    w32(80, *[e_h[i] for i in queries], *[e_h[i ^ 1] for i in queries])
    wpaths([path(trace_layers, i) for i in queries])
    wpaths([path(trace_layers, i ^ 1) for i in queries])

    def w4(vals, layers, idx):
        w32(80)
        for i in idx:
            w32(*vals[:, i])
        for i in idx:
            w32(*vals[:, i ^ 1])
        wpaths([path(layers, i) for i in idx])
        wpaths([path(layers, i ^ 1) for i in idx])

    w4(q_h, quot_layers, queries)
    w32(len(fri_layers))
    folded = [i // 2 for i in queries]
    for vals, lay in zip(fri_vals, fri_layers):
        w4(vals, lay, folded)
        folded = [i // 2 for i in folded]
    return bytes(w)


def gpu_qmul(x, y):
    a, b, c, d = (int(v) for v in x)
    e, f, g, h = (int(v) for v in y)

    def cm(p, q, r, s):
        return ((p * r - q * s) % P, (p * s + q * r) % P)

    ac, bd, ad, bc = cm(a, b, e, f), cm(c, d, g, h), cm(a, b, g, h), cm(c, d, e, f)
    bdu = ((2 * bd[0] - bd[1]) % P, (bd[0] + 2 * bd[1]) % P)
    return [(ac[0] + bdu[0]) % P, (ac[1] + bdu[1]) % P, (ad[0] + bc[0]) % P, (ad[1] + bc[1]) % P]


def main(out_path: Path):
    global R
    R = C.CDLL(str(REF_SO))
    fx = {}
    # native twiddles and NTT
    for log_n in (6, 9):
        line, circ, il, ic, _ = native_twiddles(log_n)
        fx[f"tw{log_n}_line"], fx[f"tw{log_n}_circle"] = host(line), host(circ)
        fx[f"tw{log_n}_iline"], fx[f"tw{log_n}_icircle"] = host(il), host(ic)
    x = seeded(1, 1 << 9)
    line, circ, il, ic, offs = native_twiddles(9)
    d = dev(x)
    R.cuda_circle_ntt_evaluate(vp(d), vp(line), vp(circ), hostarr(offs), hostarr(offs), u32(8), u32(512))
    fx["ntt9_in"], fx["ntt9_eval"] = x, host(d)
    # fold twiddles
    fx["foldtw_hc8"] = host(fold_twiddles(half_coset(8), 8, True))
    fx["foldtw_ho7"] = host(fold_twiddles(half_odds(7), 7, False))
    # batch inverse with zeros
    z = seeded(2, 300)
    z[[0, 5, 64, 100, 299]] = 0
    o = empty(300)
    R.cuda_batch_inverse_m31(vp(dev(z)), vp(o), u32(300))
    fx["binv_in"], fx["binv_out"] = z, host(o)
    # Merkle leaves / tiles
    cols = seeded(3, 20 * 64).reshape(20, 64)
    for nc in (1, 4, 16, 20):
        out = empty(8 * 64)
        R.cuda_merkle_hash_leaves(vp(ptrs([dev(c) for c in cols[:nc]])), vp(out), u32(nc), u32(64))
        fx[f"leaves_c{nc}"] = host(out).reshape(64, 8)
    fx["leaf_cols"] = cols
    s4 = seeded(4, 4 * 2048).reshape(4, 2048)
    tiles = empty(16)
    R.cuda_merkle_tiled_soa4(*[vp(dev(c)) for c in s4], vp(tiles), u32(2048))
    fx["soa4_in"], fx["soa4_tiles"] = s4, host(tiles).reshape(2, 8)
    # folds
    src = seeded(5, 4 * 256).reshape(4, 256)
    alpha = seeded(6, 4)
    tw = fold_twiddles(half_odds(8), 8, False)
    outs = [empty(128) for _ in range(4)]
    R.cuda_fold_line_soa(*[vp(dev(c)) for c in src], vp(tw), *[vp(o) for o in outs], hostarr(alpha), u32(128))
    fx["fold_src"], fx["fold_alpha"], fx["fold_line"] = src, alpha, np.stack([host(o) for o in outs])
    # quotient
    t = seeded(7, 1024)
    outs = [empty(1024) for _ in range(4)]
    R.cuda_fibonacci_quotient(vp(dev(t)), *[vp(o) for o in outs], hostarr(alpha), u32(1024))
    fx["quot_trace"], fx["quot_out"] = t, np.stack([host(o) for o in outs])
    # whole proofs
    for log_n, a, b in ((4, 1, 1), (5, 2, 3), (6, 1, 1), (8, 42, 99)):
        fx[f"proof_{log_n}_{a}_{b}"] = np.frombuffer(ref_prove(a, b, log_n), np.uint8)
    np.savez_compressed(out_path, **fx)
    print(f"wrote {out_path} ({len(fx)} arrays)")


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else HERE / "ref_golden.npz")
