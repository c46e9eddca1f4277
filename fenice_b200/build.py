"""Builds the CUDA library of the package in-tree: fenice_b200/libfenice_gpu.so (sm_100a only).

    python -m fenice_b200.build            # or: python fenice_b200/build.py

The library is plain nvcc output with a C ABI (include/fenice_gpu.h); it does not link PyTorch. The floating-point
flags are part of the numerics: --fmad=false keeps every multiply and add separately rounded (the reference is built
with -ffp-contract=off), and double division and square root are IEEE-rounded, so the FP64 kernels give the
reference's bits.
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libfenice_gpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = ["runtime.cu", "mixed.cu", "batch.cu", "batch_mixed.cu", "sensor.cu", "expr.cu", "cells.cu"]
HEADERS = ["physics.cuh", "grid.cuh", "stage.cuh", "viscous.cuh", "hancock.cuh", "mixed.cuh", "mixed_api.h", "batch.cuh", "batch_api.h", "host_common.h", "ibm.cuh", "ibm_host.h", "sensor.cuh", "sensor_api.h", "expr.h", "expr.cuh", "fourth.cuh", "tma.cuh", "tc.cuh"]

COMMON_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "-I" + os.path.join(ROOT, "include"),
]
# per translation unit: the FP64 path keeps every operation IEEE-rounded and uncontracted (the reference's bits); the
# mixed-precision kernels use fast single-precision math
UNIT_FLAGS = {
    "runtime.cu": ["--fmad=false", "-prec-div=true", "-prec-sqrt=true"],
    "mixed.cu": ["--use_fast_math"],
    "batch.cu": ["--fmad=false", "-prec-div=true", "-prec-sqrt=true"],
    "batch_mixed.cu": ["--use_fast_math"],
    "sensor.cu": ["--use_fast_math"],
    "expr.cu": ["--fmad=false", "-prec-div=true", "-prec-sqrt=true"],
    "cells.cu": ["--fmad=false", "-prec-div=true", "-prec-sqrt=true"],
}


def _deps(obj):
    """The files an object was compiled from, from the dependency file nvcc wrote beside it (-MD); None if absent."""
    try:
        with open(obj + ".d") as f:
            text = f.read().replace("\\\n", " ")
    except OSError:
        return None
    return [d for d in text.split(":", 1)[1].split() if d] if ":" in text else None


def _obj_stale(src, obj):
    if not os.path.exists(obj):
        return True
    deps = _deps(obj)
    if deps is None:
        deps = [src] + [os.path.join(SRC, h) for h in HEADERS]
    t = os.path.getmtime(obj)
    return any(not os.path.exists(d) or os.path.getmtime(d) > t for d in deps + [__file__])


def _stale():
    if not os.path.exists(LIB):
        return True
    objdir = os.path.join(HERE, "_build")
    objs = [os.path.join(objdir, f.replace(".cu", ".o")) for f in SOURCES]
    t = os.path.getmtime(LIB)
    return any(_obj_stale(os.path.join(SRC, f), o) for f, o in zip(SOURCES, objs)) or any(os.path.getmtime(o) > t for o in objs if os.path.exists(o))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed: " + " ".join(cmd))
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)


def build(force=False, verbose=False, extra=()):
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = [os.path.join(objdir, f.replace(".cu", ".o")) for f in SOURCES]
    # only the translation units whose sources or included headers changed since their object was built (all with --force)
    cmds = [[NVCC] + COMMON_FLAGS + UNIT_FLAGS[f] + list(extra) + ["-MD", "-MF", o + ".d", "-c", os.path.join(SRC, f), "-o", o]
            for f, o in zip(SOURCES, objs) if force or extra or _obj_stale(os.path.join(SRC, f), o)]
    # the translation units compile in parallel
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, len(cmds))) as pool:
        for fut in [pool.submit(_run, c, verbose) for c in cmds]:
            fut.result()
    _run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "--cudart", "static", "-shared", "-o", LIB] + objs, verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, extra=[a for a in sys.argv[1:] if a != "--force"])
