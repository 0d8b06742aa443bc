"""Build libkumo_b200.so in-tree (CUDA kernels for sm_100a + C++20 host core + C ABI).

    python chem-kumo_b200/build.py [--force] [--jobs N]

Objects go to chem-kumo_b200/_build/, the library to chem-kumo_b200/lib/.
Each translation unit is rebuilt only when it or a header changed.
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
BUILD = os.path.join(HERE, "_build")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libkumo_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INCLUDES = ["-I" + os.path.join(HERE, "include"), "-I" + os.path.join(ROOT, "include"),
            "-I" + os.path.join(HERE, "csrc")]
HOST_CXX = "g++"

# Translation units and their extra flags.
CUDA_UNITS = {
    "csrc/cuda/ao_build_f64.cu": ["-fmad=false"],
    "csrc/cuda/ao_mixed.cu": [],
    "csrc/cuda/contract_f64.cu": [],
    "csrc/cuda/contract_mixed.cu": [],
    "csrc/cuda/contract_p_mixed.cu": [],
    "csrc/cuda/esp.cu": [],
    "csrc/host/device_state.cu": [],
    "csrc/host/evaluator.cu": [],
    "csrc/host/capi.cu": [],
    "csrc/host/profile.cu": [],
    "csrc/host/noalloc.cu": [],
    "csrc/host/server.cu": [],
    "csrc/cuda/isosurface.cu": [],
    "csrc/host/surface.cu": [],
}
CXX_UNITS = [
    "csrc/host/fchk.cpp",
    "csrc/host/basis.cpp",
    "csrc/host/molecule.cpp",
    "csrc/host/grid.cpp",
    "csrc/host/cube.cpp",
]


def _headers():
    hs = []
    for pat in ("csrc/**/*.cuh", "csrc/**/*.hpp", "include/**/*.hpp"):
        hs += glob.glob(os.path.join(HERE, pat), recursive=True)
    hs.append(os.path.join(ROOT, "include", "kumo_b200.h"))
    return hs


def _stale(src: str, obj: str, headers) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return os.path.getmtime(src) > t or any(os.path.getmtime(h) > t for h in headers)


def _compile(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compilation failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stderr


def build(force: bool = False, jobs: int = 0, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    headers = _headers()
    cmds = []
    objs = []
    ccbin = shutil.which(HOST_CXX) or HOST_CXX
    for rel, extra in CUDA_UNITS.items():
        src = os.path.join(HERE, rel)
        obj = os.path.join(BUILD, rel.replace("/", "_") + ".o")
        objs.append(obj)
        if force or _stale(src, obj, headers):
            cmds.append([NVCC, "-ccbin", ccbin, "-std=c++20", *ARCH, "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
                         "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr", *INCLUDES, *extra,
                         "-c", src, "-o", obj])
    for rel in CXX_UNITS:
        src = os.path.join(HERE, rel)
        obj = os.path.join(BUILD, rel.replace("/", "_") + ".o")
        objs.append(obj)
        if force or _stale(src, obj, headers):
            cmds.append([ccbin, "-std=c++20", "-O2", "-fPIC", "-ffp-contract=off", "-Wall",
                         "-I/usr/local/cuda/include", *INCLUDES, "-c", src, "-o", obj])
    if cmds:
        with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
            for out in ex.map(_compile, cmds):
                if verbose and out:
                    print(out, file=sys.stderr)
    if cmds or not os.path.exists(LIB):
        _compile([NVCC, "-ccbin", ccbin, *ARCH, "-shared", "-o", LIB, *objs, "-lz", "-Xcompiler", "-fPIC"])
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=0)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.jobs, a.verbose))


if __name__ == "__main__":
    main()
