"""Builds the C-ABI libraries in-tree for sm_100a.

    astaroth_b200/lib/libastaroth_sp.so     AcReal = float,  FP32 kernels
    astaroth_b200/lib/libastaroth_dp.so     AcReal = double, FP64 kernels
    astaroth_b200/lib/libastaroth_mixed.so  AcReal = float,  compensated state

Each library exports the whole of include/astaroth.h, include/astaroth_utils.h
and include/astaroth_b200.h. Usage: python -m astaroth_b200.build [-j N] [--force]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(REPO, "include")
LIBDIR = os.path.join(HERE, "lib")
BUILD = os.path.join(HERE, "_build")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
# the system compiler carries libgomp (a CC/CXX from the environment may not)
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

FLAVOURS = {
    "sp": ["-DAC_DOUBLE_PRECISION=0", "-DACB_MIXED=0"],
    "dp": ["-DAC_DOUBLE_PRECISION=1", "-DACB_MIXED=0"],
    "mixed": ["-DAC_DOUBLE_PRECISION=0", "-DACB_MIXED=1"],
}
CU_SOURCES = ["device.cu", "ensemble.cu", "reduce_noalloc.cu"]
CXX_SOURCES = ["node.cc", "host_utils.cc", "host_model.cc", "forcing.cc"]
HEADERS = ["common.cuh", "tma.cuh", "solve.cuh", "halo.cuh", "reduce.cuh", "internal.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xptxas", "-v",
    f"-ccbin={CXX}",
]
CXX_FLAGS = ["-O3", "-fPIC", "-std=c++17", "-fopenmp", f"-I{CUDA_HOME}/include"]


def lib_path(flavour: str) -> str:
    return os.path.join(LIBDIR, f"libastaroth_{flavour}.so")


def _deps() -> list[str]:
    files = [os.path.join(CSRC, f) for f in CU_SOURCES + CXX_SOURCES + HEADERS]
    files += [os.path.join(INC, f) for f in os.listdir(INC) if f.endswith(".h")]
    return files


def _stale(target: str) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in _deps())


def _run(cmd: list[str], log: str) -> None:
    with open(log, "w") as f:
        f.write(" ".join(cmd) + "\n")
        f.flush()
        r = subprocess.run(cmd, stdout=f, stderr=subprocess.STDOUT)
    if r.returncode != 0:
        with open(log) as f:
            sys.stderr.write(f.read()[-8000:])
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ... (log {log})")


def build_flavour(flavour: str, force: bool = False) -> str:
    target = lib_path(flavour)
    if not force and not _stale(target):
        return target
    odir = os.path.join(BUILD, flavour)
    os.makedirs(odir, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    defs = FLAVOURS[flavour]
    objs = []
    jobs = []
    for src in CU_SOURCES:
        obj = os.path.join(odir, src + ".o")
        cmd = [NVCC, *NVCC_FLAGS, *defs, f"-I{INC}", f"-I{CSRC}", "-c", os.path.join(CSRC, src),
               "-o", obj]
        jobs.append((cmd, obj + ".log"))
        objs.append(obj)
    for src in CXX_SOURCES:
        obj = os.path.join(odir, src + ".o")
        cmd = [CXX, *CXX_FLAGS, *defs, f"-I{INC}", f"-I{CSRC}", "-c", os.path.join(CSRC, src),
               "-o", obj]
        jobs.append((cmd, obj + ".log"))
        objs.append(obj)
    with cf.ThreadPoolExecutor(max_workers=len(jobs)) as ex:
        for fut in [ex.submit(_run, c, l) for c, l in jobs]:
            fut.result()
    tmp = target + ".tmp"
    link = [CXX, "-shared", "-o", tmp, *objs, f"-L{CUDA_HOME}/lib64", "-lcudart", "-fopenmp",
            f"-Wl,-rpath,{CUDA_HOME}/lib64", "-Wl,--no-undefined"]
    _run(link, os.path.join(odir, "link.log"))
    os.replace(tmp, target)
    return target


def build_all(flavours=None, force: bool = False, jobs: int = 3) -> list[str]:
    flavours = list(flavours or FLAVOURS)
    with cf.ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        futs = [ex.submit(build_flavour, f, force) for f in flavours]
        return [f.result() for f in futs]


def ptxas_report(flavour: str) -> str:
    """The -Xptxas -v lines (registers, spills, shared memory) of the last build."""
    log = os.path.join(BUILD, flavour, "device.cu.o.log")
    if not os.path.exists(log):
        return ""
    with open(log) as f:
        return "".join(line for line in f if "ptxas" in line or "registers" in line
                       or "spill" in line)


def main(argv=None) -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=3)
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("flavours", nargs="*")
    a = ap.parse_args(argv)
    if a.clean:
        shutil.rmtree(BUILD, ignore_errors=True)
    for p in build_all(a.flavours or None, a.force, a.j):
        print("built", p)


if __name__ == "__main__":
    main()
