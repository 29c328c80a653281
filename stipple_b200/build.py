"""Build librdb_b200.so (the sm_100a engines + C ABI) in-tree.

    python -m stipple_b200.build [--verbose-ptxas]

Device code compiles with -fmad=false so no multiply-add is contracted (the
exact engines reproduce the reference's double arithmetic operation by
operation); host code with -ffp-contract=off for the same reason.  No fast-math
anywhere: the IEEE float divide and the float/double conversions are part of
the numeric contract.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build", "rdb")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "librdb_b200.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler",
          "-ffp-contract=off", "-Xcompiler", "-fno-fast-math", "-I", os.path.join(ROOT, "include")]
DEVICE = ["-fmad=false", "--ftz=false", "--prec-div=true", "--prec-sqrt=true"]

SOURCES = [
    "rdb_octree.cpp",
    "rdb_plan.cpp",
    "rdb_runtime.cpp",
    "rdb_capi.cpp",
    "rdb_serve.cpp",
    "rdb_palette_file.cpp",
    "rdb_palette_png.cpp",
    "rdb_curve.cu",
    "rdb_walk_seq.cu",
    "rdb_walk_blocks.cu",
    "rdb_jacobi.cu",
    "rdb_ssw.cu",
    "rdb_tsw.cu",
    "rdb_uniform.cu",
    "rdb_probe.cu",
    "rdb_cand.cu",
    "rdb_octree_dev.cu",
]


def _obj(src: str) -> str:
    return os.path.join(BUILD, src + ".o")


def _compile(src: str, ptxas_verbose: bool) -> tuple[str, str]:
    path = os.path.join(CSRC, src)
    cmd = [NVCC, *ARCH, *COMMON, *DEVICE, "-c", path, "-o", _obj(src)]
    if ptxas_verbose and src.endswith(".cu"):
        cmd.append("-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return src, r.stderr


def _stale(src: str) -> bool:
    o = _obj(src)
    if not os.path.exists(o):
        return True
    t = os.path.getmtime(o)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(ROOT, "include", "rdb.h"))
    deps.append(__file__)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _lib_current() -> bool:
    """The shipped library is newer than every source (object files need not exist)."""
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps += [os.path.join(ROOT, "include", "rdb.h"), __file__]
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


# The reference-facing C++ layer (stipple_b200/dropin) is compiled against
# the reference's own headers, where that tree is present; elsewhere the
# libraries built here earlier are used as they are.
# The reference checkout: $RDB_REFERENCE, else a sibling of this repository
# named "reference".
REFERENCE = os.environ.get("RDB_REFERENCE",
                           os.path.normpath(os.path.join(ROOT, os.pardir, "reference")))
DROPIN = os.path.join(HERE, "dropin")
DROPIN_LIB = os.path.join(LIBDIR, "librd_b200_dropin.so")
PLUGIN_LIB = os.path.join(LIBDIR, "librd_b200_plugin.so")


def build_dropin() -> bool:
    """Builds librd_b200_dropin.so (the seven engine symbols of
    rd_riemersma.h) and librd_b200_plugin.so (the "riemersma-b200" registry
    entry).  Returns False when the reference headers are absent."""
    inc = os.path.join(REFERENCE, "include")
    if not os.path.isdir(inc):
        return False
    common = ["g++", "-std=c++20", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-I", inc,
              "-I", os.path.join(ROOT, "include"), "-Wl,-rpath,$ORIGIN"]
    steps = [
        (DROPIN_LIB, [os.path.join(DROPIN, "rd_b200_dropin.cpp")],
         ["-L", LIBDIR, "-lrdb_b200"]),
        (PLUGIN_LIB, [os.path.join(DROPIN, "rd_b200_plugin.cpp")],
         ["-L", LIBDIR, "-lrd_b200_dropin"]),
    ]
    for out, srcs, libs in steps:
        if os.path.exists(out) and all(os.path.getmtime(x) <= os.path.getmtime(out)
                                       for x in srcs + [LIB]):
            continue
        r = subprocess.run(common + ["-o", out] + srcs + libs, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"drop-in build failed ({out}):\n{r.stdout}\n{r.stderr}")
    return True


def build(ptxas_verbose: bool = False, force: bool = False) -> str:
    if not force and not ptxas_verbose and _lib_current():
        build_dropin()
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    todo = [s for s in SOURCES if force or _stale(s)]
    logs = []
    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            for src, log in ex.map(lambda s: _compile(s, ptxas_verbose), todo):
                if log.strip():
                    logs.append(f"--- {src}\n{log}")
    if todo or not os.path.exists(LIB):
        # zlib: the PNG form of palette files.
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *[_obj(s) for s in SOURCES], "-lcudart", "-lz"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if logs and ptxas_verbose:
        print("\n".join(logs))
    build_dropin()
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose_ptxas, a.force))
    sys.exit(0)
