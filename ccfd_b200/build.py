"""Build the in-tree native library ``ccfd_b200/lib/libccfd_b200.so``.

Sources: the C host layer (``csrc/host/*.c``, gcc), the locality ordering
(``csrc/*.cpp``, g++) and the CUDA kernels plus C ABI (``csrc/*.cu``, nvcc for
``sm_100a`` only).  Floating-point contraction is disabled everywhere
(``-ffp-contract=off`` / ``-fmad=false``) so the FP64 path performs exactly the
operations written in the reference's C source.

    python -m ccfd_b200.build          # incremental
    python -m ccfd_b200.build --force  # rebuild everything
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "lib")
OBJ = os.path.join(OUT, "obj")
INC = os.path.join(ROOT, "include")
LIB = os.path.join(OUT, "libccfd_b200.so")
DRIVER = os.path.join(OUT, "ccfd_run")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build ccfd_b200")


def _headers() -> list[str]:
    return (glob.glob(os.path.join(CSRC, "**", "*.h"), recursive=True)
            + glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True)
            + glob.glob(os.path.join(CSRC, "**", "*.inc"), recursive=True)
            + glob.glob(os.path.join(INC, "*.h")))


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def _compile(src: str, force: bool) -> str:
    rel = os.path.relpath(src, CSRC).replace(os.sep, "_")
    obj = os.path.join(OBJ, rel + ".o")
    deps = [src] + _headers()
    if not force and not _stale(obj, deps):
        return obj
    inc = ["-I", INC, "-I", CSRC, "-I", os.path.join(CSRC, "host")]
    if src.endswith(".cu"):
        # FP64 code keeps every multiply and add separately rounded (as the
        # reference); the mixed-precision kernels may contract them
        fmad = "-fmad=true" if src.endswith("_mixed.cu") else "-fmad=false"
        cmd = [_nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", fmad,
               "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-ffp-contract=off",
               *inc, "-c", src, "-o", obj]
    elif src.endswith(".cpp"):
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", *inc, "-c", src, "-o", obj]
    else:
        cmd = ["gcc", "-O2", "-std=c11", "-D_POSIX_C_SOURCE=200809L", "-fPIC",
               "-ffp-contract=off", "-Wall", *inc, "-c", src, "-o", obj]
    _run(cmd)
    return obj


def build(force: bool = False, verbose: bool = True) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = (sorted(glob.glob(os.path.join(CSRC, "*.cu")))
            + sorted(glob.glob(os.path.join(CSRC, "*.cpp")))
            + sorted(glob.glob(os.path.join(CSRC, "host", "*.c"))))
    driver_src = os.path.join(CSRC, "driver", "ccfd_run.c")
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
    if force or _stale(LIB, objs):
        _run([_nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart", "-lm"])
        if verbose:
            print(f"built {os.path.relpath(LIB, ROOT)}")
    if os.path.exists(driver_src) and (force or _stale(DRIVER, [driver_src, LIB])):
        _run(["gcc", "-O2", "-std=c11", "-D_POSIX_C_SOURCE=200809L", "-Wall",
              "-I", INC, driver_src, "-o", DRIVER, "-L", OUT, "-lccfd_b200",
              "-Wl,-rpath,$ORIGIN", "-lm"])
        if verbose:
            print(f"built {os.path.relpath(DRIVER, ROOT)}")
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args(argv)
    try:
        build(force=a.force)
    except RuntimeError as e:
        print(e, file=sys.stderr)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
