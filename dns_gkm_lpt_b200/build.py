"""Build libgkm_b200.so in-tree with nvcc for sm_100a.

    python -m dns_gkm_lpt_b200.build          (or __graft_entry__.build())

The library lands in dns_gkm_lpt_b200/lib/ so it travels with the source tree
(no JIT cache).  Objects are compiled in parallel and only when their sources
changed.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
OBJDIR = os.path.join(PKG, "lib", "obj")
LIB = os.path.join(LIBDIR, "libgkm_b200.so")

SOURCES = ["sweep.cu", "sweep_mixed.cu", "lagrangian.cu", "probe.cu", "noalloc.cu", "gkm_capi.cu", "gkm_ensemble.cu", "output.cu"]
HEADERS = ["gkm_numerics.cuh", "gkm_internal.h", "gkm_handle.h", "sweep_impl.cuh", "sweep_ws.cuh", "f32x2.cuh"]
# per-file extra flags: the single-precision sweeps use fast float math
EXTRA = {"sweep_mixed.cu": ["-use_fast_math", "-DGKM_UNROLL_SIDES=0"]}

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-std=c++17", "-lineinfo",
    "-Xcompiler", "-fPIC,-ffp-contract=off",
    "-ccbin", "g++",
    "-I" + os.path.join(ROOT, "include"),
    "-I" + CSRC,
]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _stale(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    nvcc = _nvcc()
    deps_common = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "gkm.h")]
    jobs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJDIR, src.replace(".cu", ".o"))
        if _stale(o, [s] + deps_common) or ptxas_info:
            cmd = [nvcc] + NVCC_FLAGS + EXTRA.get(src, []) + (["-Xptxas", "-v"] if ptxas_info else []) + [
                "-c", s, "-o", o]
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with cf.ThreadPoolExecutor(max_workers=len(jobs) or 1) as ex:
        for cmd, r in ex.map(run, jobs):
            if verbose or ptxas_info or r.returncode:
                sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            if r.returncode:
                raise RuntimeError(f"nvcc failed for {cmd[-3]}")
    objs = [os.path.join(OBJDIR, s.replace(".cu", ".o")) for s in SOURCES]
    if jobs or not os.path.exists(LIB):
        cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-ccbin", "g++", "-cudart", "static",
               "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv))
