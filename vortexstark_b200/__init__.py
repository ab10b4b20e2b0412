"""vortexstark_b200 — B200-native (sm_100a) VortexSTARK polynomial-commitment path.

The compute lives in libvstark.so (CUDA kernels + C ABI, declared in
include/vstark.h). This package binds that library with ctypes and mirrors the
reference's host API for the hot path (src/ntt.rs, src/merkle.rs, src/fri.rs,
src/prover.rs, src/verifier.rs) on top of torch device tensors.

There is no CPU fallback: if the library is missing or no CUDA device is
present, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from pathlib import Path

# The slot engine keeps up to 24 streams busy (8 slots x 3 priorities); CUDA maps
# streams onto CUDA_DEVICE_MAX_CONNECTIONS hardware queues (8 by default), and
# streams that share a queue serialise, so a small job could wait behind a large
# one. 32 gives each stream its own queue. CUDA reads it when the context is
# created, so this only takes effect when the package is imported first.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
HEADER = ROOT / "include" / "vstark.h"
LIB_PATH = PKG / "libvstark.so"
P = 0x7FFFFFFF

__all__ = ["lib", "declared_functions", "VstarkError", "check", "P"]


class VstarkError(RuntimeError):
    pass


_CTYPES = {
    "void": None,
    "int": C.c_int,
    "uint32_t": C.c_uint32,
    "uint64_t": C.c_uint64,
    "size_t": C.c_size_t,
    "vs_stream_t": C.c_void_p,
    "const char*": C.c_char_p,
    "char*": C.c_char_p,
    "double": C.c_double,
}


def _ctype(decl: str):
    t = " ".join(decl.replace("const", " const ").split())
    t = re.sub(r"\s*\*\s*", "*", t)
    if t in ("const char*", "char*"):
        return C.c_char_p
    if "*" in t:
        return C.c_void_p
    base = t.replace("const ", "").strip()
    if base not in _CTYPES:
        raise ValueError(f"unmapped C type {decl!r}")
    return _CTYPES[base]


def declared_functions() -> dict[str, tuple[str, list[str]]]:
    """Parse include/vstark.h: name -> (return type, [argument types])."""
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    text = re.sub(r"^\s*#[^\n]*", "", text, flags=re.M)
    text = text.replace('extern "C" {', "").replace("}", ";")
    out = {}
    for stmt in text.split(";"):
        stmt = " ".join(stmt.split())
        m = re.fullmatch(r"((?:const )?[A-Za-z_]\w*(?: ?\*)*) ?\b(\w+) ?\((.*)\)", stmt)
        if not m or stmt.startswith(("typedef", "enum")):
            continue
        ret, name, args = m.group(1).strip(), m.group(2), m.group(3).strip()
        arg_types = []
        if args and args != "void":
            for a in args.split(","):
                a = a.strip()
                arg_types.append(re.sub(r"\s*\b\w+$", "", a) if re.search(r"[\w\*]\s+\w+$", a) else a)
        out[name] = (ret, arg_types)
    return out


_lib = None


def lib() -> C.CDLL:
    """Load libvstark.so and declare every function of include/vstark.h."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise VstarkError(f"{LIB_PATH} is missing: build it with `python -m vortexstark_b200.build`")
    L = C.CDLL(str(LIB_PATH))
    for name, (ret, args) in declared_functions().items():
        fn = getattr(L, name)  # AttributeError here means the library lacks a declared symbol
        fn.restype = _ctype(ret)
        fn.argtypes = [_ctype(a) for a in args]
    _lib = L
    return L


def check(status: int, what: str = "") -> None:
    if status != 0:
        msg = lib().vs_last_error().decode(errors="replace")
        raise VstarkError(f"{what or 'vstark'} failed with status {status}: {msg}")
