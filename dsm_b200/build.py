"""Builds the engine: dsm_b200/libdsm.so (C ABI of include/dsm.h) and the
CDSM command line dsm_b200/bin/CDSM, for sm_100a with nvcc.

    python dsm_b200/build.py            # incremental
    python dsm_b200/build.py --clean
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdsm.so")
CLI = os.path.join(HERE, "bin", "CDSM")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a", "-Wno-deprecated-gpu-targets"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include")]
CU_FLAGS = ARCH + COMMON + ["--expt-relaxed-constexpr", "-Xptxas", "-O3"]
CXX_FLAGS = COMMON

LIB_SOURCES = [
    "engine/kernels.cu",
    "engine/match.cu",
    "engine/filter.cu",
    "engine/engine.cu",
    "engine/batch.cu",
    "engine/serve.cu",
    "engine/snapshot.cu",
    "engine/abi.cu",
    "engine/noalloc.cu",
    "host/gen.cpp",
    "host/textio.cpp",
    "host/binio.cpp",
    "host/query_plan.cpp",
]
CLI_SOURCES = ["cli/cdsm.cpp"]


def _headers():
    out = []
    for d, _, fs in os.walk(CSRC):
        out += [os.path.join(d, f) for f in fs if f.endswith((".h", ".cuh"))]
    out.append(os.path.join(ROOT, "include", "dsm.h"))
    return out


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src, verbose=False):
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, src.replace("/", "_") + ".o")
    if not _stale(obj, [path] + _headers()):
        return obj
    flags = CU_FLAGS if src.endswith(".cu") else CXX_FLAGS
    cmd = [NVCC] + flags + ["-c", path, "-o", obj]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src}\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip() and verbose:
        print(r.stderr)
    return obj


def build(clean=False, verbose=False):
    if clean and os.path.isdir(BUILD):
        shutil.rmtree(BUILD)
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    srcs = [s for s in LIB_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    cli_srcs = [os.path.join(CSRC, s) for s in CLI_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    if cli_srcs and _stale(CLI, cli_srcs + [LIB] + _headers()):
        cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-o", CLI] + cli_srcs + [
            "-L", HERE, "-ldsm", "-Wl,-rpath,$ORIGIN/..", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"CLI build failed\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    try:
        print(build(a.clean, a.verbose))
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
