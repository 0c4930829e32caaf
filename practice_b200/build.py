"""Builds libcrystal_b200.so in-tree: nvcc for the sm_100a kernels, g++ for the
host runtime (plan reader, code generator, NVRTC compiler, executor).

Run as ``python -m practice_b200.build`` or through ``__graft_entry__.build()``.
The library links the CUDA runtime statically and NVRTC dynamically; it needs
no libcuda at link time, so it loads on machines without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libcrystal_b200.so"
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = CUDA_HOME / "bin" / "nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

HOST_SOURCES = ["cx_plan.cpp", "cx_codegen.cpp", "cx_runtime.cpp", "cx_server.cpp", "cx_sycl.cpp"]
CUDA_SOURCES = ["cx_kernels.cu", "cx_finalize.cu"]
EMBEDDED = ["crystal_sm100.cuh", "cx_args.h"]


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"build step failed ({proc.returncode}): {' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _embed(out: Path) -> None:
    """Writes the device headers as C++ raw strings for NVRTC's in-memory includes."""
    names = {"crystal_sm100.cuh": "kCxEmbeddedCrystalHeader", "cx_args.h": "kCxEmbeddedArgsHeader"}
    parts = ["// Generated by practice_b200/build.py; do not edit.\n#pragma once\n"]
    for fname in EMBEDDED:
        text = (CSRC / fname).read_text()
        if ")CXHDR\"" in text:
            raise RuntimeError(f"{fname} contains the raw-string delimiter")
        parts.append(f'static const char {names[fname]}[] = R"CXHDR({text})CXHDR";\n')
    content = "".join(parts)
    if not out.exists() or out.read_text() != content:
        out.write_text(content)


def build(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    embed = BUILD / "cx_embedded.inc"
    _embed(embed)
    headers = sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + [PKG.parent / "include" / "crystal_b200.h", embed]
    objs: list[Path] = []
    for src in CUDA_SOURCES:
        obj = BUILD / (src + ".o")
        if _stale(obj, [CSRC / src] + headers):
            _run([str(NVCC), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-c",
                  str(CSRC / src), "-o", str(obj)])
        objs.append(obj)
    for src in HOST_SOURCES:
        obj = BUILD / (src + ".o")
        if _stale(obj, [CSRC / src] + headers):
            _run(["g++", "-O2", "-g", "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-function",
                  f"-I{CUDA_HOME / 'include'}", f"-I{BUILD}", "-c", str(CSRC / src), "-o", str(obj)])
        objs.append(obj)
    if _stale(LIB, objs):
        _run(["g++", "-shared", "-o", str(LIB), *map(str, objs), f"-L{CUDA_HOME / 'lib64'}",
              "-lcudart_static", "-lnvrtc", "-ldl", "-lpthread", "-lrt",
              f"-Wl,-rpath,{CUDA_HOME / 'lib64'}"])
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(verbose=True)
    sys.exit(0)
