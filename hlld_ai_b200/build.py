"""Build libhlld_b200.so in place with nvcc for sm_100a.

``python -m hlld_ai_b200.build`` (or ``build()``) compiles csrc/*.cu into
object files under ``_build/`` and links the shared library next to this
file, where ``hlld_ai_b200._lib`` loads it.  The FP64-exact variant is the
same source as the FP64 one compiled with ``-fmad=false``; the mixed and
FP32 variants are the same source with float real types.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "libhlld_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                 "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), "-I", CSRC]
# (source, extra flags)
UNITS = [
    ("capi.cu", []),
    ("variant_fp64.cu", []),
    ("variant_exact.cu", ["-fmad=false"]),
    ("variant_mixed.cu", ["-ftz=true", "-prec-div=false", "-prec-sqrt=false"]),
    ("variant_fp32.cu", ["-ftz=true"]),
    ("noalloc.cu", []),
    ("adjoint_fp64.cu", []),
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    hs = [os.path.join(ROOT, "include", "hlld_b200.h")]
    hs += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    return hs


def build(verbose: bool = False, ptxas_info: bool = False, force: bool = False) -> str:
    """Compile and link; returns the library path.  Raises on failure."""
    nvcc = _nvcc()
    os.makedirs(BUILD, exist_ok=True)
    hdrs = _headers()
    jobs = []
    for src, extra in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        if force or ptxas_info or _stale(o, [s] + hdrs):
            cmd = [nvcc] + COMMON + extra + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", s, "-o", o]
            jobs.append((src, cmd))
    objs = [os.path.join(BUILD, u.replace(".cu", ".o")) for u, _ in UNITS]

    def run(job):
        src, cmd = job
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, r

    with cf.ThreadPoolExecutor(max_workers=len(jobs) or 1) as ex:
        for src, r in ex.map(run, jobs):
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
            if ptxas_info or verbose:
                sys.stdout.write(r.stderr)
    if force or jobs or _stale(LIB, objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv,
                force="--force" in sys.argv))
