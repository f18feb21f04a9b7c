"""Builds libgprm_b200.so in-tree with nvcc for sm_100a (no JIT, no torch
extension machinery: the library is a plain C-ABI shared object)."""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
OUT = os.path.join(PKG, "libgprm_b200.so")
SOURCES = ["gprm_api.cu", "gprm_batch.cu", "gprm_kernels.cu", "gprm_mlp.cu", "gprm_nbr.cu", "gprm_graph.cu", "gprm_sample.cu"]
HEADERS = ["gprm_device.cuh", "gprm_host.h", "gprm_internal.h", "gprm_sincos64.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    # IEEE single precision everywhere, no FMA contraction: the FP32 kernels
    # reproduce the reference's operation-by-operation rounding.
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC", "-shared", "-ccbin", "/usr/bin/g++",
]


def nvcc() -> str:
    for c in ("/usr/local/cuda/bin/nvcc", "nvcc"):
        if os.path.isabs(c) and os.path.exists(c):
            return c
    return "nvcc"


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(PKG, "..", "include", "gprm_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False, out: str = OUT,
          defines=()) -> str:
    """Compiles every source to an object in parallel (one nvcc per file,
    objects under a build folder beside `out`), then links the shared
    library."""
    if not force and out == OUT and not needs_build():
        return OUT
    from concurrent.futures import ThreadPoolExecutor
    objdir = os.path.join(os.path.dirname(os.path.abspath(out)), "_build",
                          os.path.splitext(os.path.basename(out))[0])
    os.makedirs(objdir, exist_ok=True)
    flags = NVCC_FLAGS[:]
    flags.remove("-shared")
    extra = (["-Xptxas", "-v"] if ptxas_info else []) + [f"-D{d}" for d in defines]

    def compile_one(f):
        obj = os.path.join(objdir, f.replace(".cu", ".o"))
        cmd = [nvcc()] + flags + extra + ["-c", "-o", obj, os.path.join(CSRC, f)]
        if verbose:
            print(" ".join(cmd), flush=True)
        return obj, subprocess.run(cmd, capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    for obj, r in results:
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc failed compiling " + os.path.basename(obj))
        if verbose or ptxas_info:
            sys.stderr.write(r.stderr)
    link = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-fPIC", "-ccbin",
            "/usr/bin/g++", "-o", out] + [o for o, _ in results]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed linking libgprm_b200.so")
    return out


if __name__ == "__main__":
    build(verbose=True, force=True, ptxas_info="-v" in sys.argv)
