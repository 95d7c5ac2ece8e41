"""Build libdmrgb200.so in-tree with nvcc for sm_100a (no torch, no JIT cache).

Usage: ``python dmrjtensor.jl_b200/build.py`` (or ``__graft_entry__.build()``).
The shared library lands next to this file so it travels with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "libdmrgb200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xcompiler", "-fvisibility=hidden"]

SOURCES = ["gemm_f64.cu", "gemm_tf32.cu", "vec_kernels.cu", "jacobi.cu", "jacobi_block.cu", "syevt.cu", "syevt_mid.cu", "noalloc.cu", "engine_layout.cpp", "engine_eig.cpp",
           "engine_contract.cpp", "engine_sweep.cpp", "engine_3s.cpp", "engine_tdvp.cpp", "engine_meas.cpp", "abi.cpp", "server.cpp", "batch.cpp"]


def _needs_build(objs_src):
    if not OUT.exists():
        return True
    t = OUT.stat().st_mtime
    deps = list(CSRC.glob("*")) + [HERE.parent / "include" / "dmrg_b200.h", Path(__file__)]
    return any(p.stat().st_mtime > t for p in deps if p.exists())


def build(force: bool = False, verbose: bool = False, jobs: int = 8) -> Path:
    """Compile every source for sm_100a and link ``libdmrgb200.so``. Returns its path."""
    if not force and not _needs_build(SOURCES):
        return OUT
    objdir = HERE / "_build"
    objdir.mkdir(exist_ok=True)
    procs = []
    objs = []
    for src in SOURCES:
        obj = objdir / (src + ".o")
        objs.append(obj)
        extra = ["-x", "cu"] if src.endswith(".cu") else []
        cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", str(CSRC / src), "-o", str(obj),
               "-I", str(HERE.parent / "include")]
        if src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if verbose else []
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        if len(procs) >= jobs:
            _drain(procs)
    _drain(procs)
    link = [NVCC, *ARCH, "-shared", "-o", str(OUT), *map(str, objs), "-lcudart"]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return OUT


def _drain(procs):
    errs = []
    for src, p in procs:
        out, _ = p.communicate()
        text = out.decode(errors="replace")
        if p.returncode != 0:
            errs.append(f"--- {src}\n{text}")
        elif text.strip() and os.environ.get("DMRG_BUILD_VERBOSE"):
            sys.stderr.write(text)
    procs.clear()
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
