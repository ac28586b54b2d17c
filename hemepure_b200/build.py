"""Build libhemeb200.so in-tree (nvcc for sm_100a + g++ for the host front-end).

Usage: python -m hemepure_b200.build [--force]
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libhemeb200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# FP64 kernels: no FMA contraction, so results follow the reference's rounding.
CU_SOURCES = {
    "kernels_f64.cu": ["-fmad=false"],
    "kernels_mixed.cu": [],
    "noalloc.cu": [],
    "kernels_batch.cu": [],
    "gmy_device.cu": [],
    "shard.cu": [],
    "layout_device.cu": [],
    # the selectors' float arithmetic as the host rounds it
    "extract.cu": ["-fmad=false"],
}
CPP_SOURCES = ["xml.cpp", "config.cpp", "layout.cpp", "shard.cpp", "solver.cpp", "extraction.cpp", "batch.cpp", "capi.cpp"]
HEADERS = ["hb_common.h", "f64_site.cuh", "xml.h", "config.h", "layout.h", "device.h", "solver.h", "extraction.h", "mixed_site.cuh", "batch.h", "batch_dev.h", "shard.h", "setup_pool.h"]


def _deps_mtime() -> float:
    paths = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "hemeb200.h"), __file__]
    return max(os.path.getmtime(p) for p in paths if os.path.exists(p))


def _local_includes(path: str, seen: set) -> None:
    """The quoted #include files of `path` within the source tree, transitively."""
    if path in seen or not os.path.exists(path):
        return
    seen.add(path)
    with open(path) as fh:
        for line in fh:
            t = line.strip()
            if t.startswith("#include") and '"' in t:
                inc = t.split('"')[1]
                _local_includes(os.path.normpath(os.path.join(os.path.dirname(path), inc)), seen)


def _stale(src: str, obj: str, hdr_mtime: float) -> bool:
    """An object is stale when it is older than its source, one of the source's
    own headers (followed through quoted includes) or this script."""
    if not os.path.exists(obj):
        return True
    deps: set = set()
    _local_includes(src, deps)
    newest = max([os.path.getmtime(d) for d in deps] + [os.path.getmtime(__file__)])
    return os.path.getmtime(obj) < newest


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hm = _deps_mtime()
    jobs = []
    objs = []
    for src, extra in CU_SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if force or _stale(s, o, hm):
            jobs.append([NVCC, *ARCH, "-O3", "-std=c++17", "-lineinfo", "-Xptxas", "-v", *extra,
                         "-Xcompiler", "-fPIC", "-c", s, "-o", o])
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if force or _stale(s, o, hm):
            jobs.append(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wno-unused-function",
                         "-I" + os.path.join(CUDA, "include"), "-c", s, "-o", o])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=max(2, os.cpu_count() or 2)) as ex:
            for out in ex.map(_run, jobs):
                if verbose and out:
                    print(out)
    if force or jobs or not os.path.exists(LIB):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB + ".tmp", *objs, "-lz"])
        os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
