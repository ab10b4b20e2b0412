"""Builds libvstark.so (sm_100a) in-tree from vortexstark_b200/csrc/*.cu.

    python -m vortexstark_b200.build [--force] [--verbose]

Objects go to vortexstark_b200/_build/, the library to vortexstark_b200/libvstark.so.
Each translation unit is compiled in parallel and only when its sources changed.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "_build"
LIB = PKG / "libvstark.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I", str(ROOT / "include"), "-I", str(CSRC)]


def _digest(paths) -> str:
    h = hashlib.sha256()
    for p in sorted(paths):
        h.update(p.name.encode())
        h.update(p.read_bytes())
    h.update(" ".join(FLAGS + ARCH).encode())
    return h.hexdigest()[:16]


def build(force: bool = False, verbose: bool = False, extra_flags: list[str] | None = None) -> Path:
    OUT.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    sources = sorted(CSRC.glob("*.cu"))
    flags = FLAGS + (extra_flags or [])

    def compile_one(src: Path) -> Path:
        obj = OUT / (src.stem + ".o")
        stamp = OUT / (src.stem + ".stamp")
        dig = _digest([src] + headers)
        if not force and obj.exists() and stamp.exists() and stamp.read_text() == dig:
            return obj
        cmd = [NVCC, *ARCH, *flags, "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr.strip():
            print(r.stderr, file=sys.stderr)
        stamp.write_text(dig)
        return obj

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(compile_one, sources))
    newest = max(o.stat().st_mtime for o in objs)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        # --no-undefined: a declaration left without a definition fails the link
        # instead of producing a library that breaks at load or call time
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-Xlinker", "--no-undefined", *map(str, objs),
               "-o", str(LIB)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
