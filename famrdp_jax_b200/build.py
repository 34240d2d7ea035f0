"""Builds libfamrdp_cuda.so in-tree with nvcc for sm_100a.

    python -m famrdp_jax_b200.build            # build if sources are newer
    python -m famrdp_jax_b200.build --force    # always rebuild

The library lands in ``famrdp_jax_b200/_lib/`` so it travels with the source
tree; it links the CUDA runtime statically and has no torch dependency.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
LIBDIR = PKG / "_lib"
LIB = LIBDIR / "libfamrdp_cuda.so"
OBJDIR = LIBDIR / "obj"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-Xptxas", "-warn-spills"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libfamrdp_cuda.so")
    return cand


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _stale(obj: Path, src: Path, hdr_mtime: float) -> bool:
    if not obj.exists():
        return True
    m = obj.stat().st_mtime
    return m < src.stat().st_mtime or m < hdr_mtime


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> Path:
    nvcc = _nvcc()
    OBJDIR.mkdir(parents=True, exist_ok=True)
    srcs = sources()
    hdr_mtime = max((h.stat().st_mtime for h in _headers()), default=0.0)
    procs = []
    objs = []
    for src in srcs:
        obj = OBJDIR / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, src, hdr_mtime):
            cmd = [nvcc, *ARCH_FLAGS, *CFLAGS, "-I", str(INCLUDE), "-I", str(CSRC), "-c",
                   str(src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd), flush=True)
            procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
            max_jobs = jobs or max(1, os.cpu_count() or 1)
            while len([p for _, p in procs if p.poll() is None]) >= max_jobs:
                procs[0][1].wait()
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        text = out.decode(errors="replace")
        if p.returncode != 0:
            failed.append((src, text))
        elif verbose and text.strip():
            print(text)
    if failed:
        msg = "\n".join(f"--- {s.name}\n{t}" for s, t in failed)
        raise RuntimeError(f"nvcc failed:\n{msg}")
    lib_mtime = LIB.stat().st_mtime if LIB.exists() else 0.0
    if force or not LIB.exists() or any(o.stat().st_mtime > lib_mtime for o in objs):
        cmd = [nvcc, *ARCH_FLAGS, "-shared", "-o", str(LIB), *map(str, objs), "-cudart", "static"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout.decode(errors="replace"))
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    lib = build(force=a.force, verbose=a.verbose)
    print(lib)
    return 0


if __name__ == "__main__":
    sys.exit(main())
