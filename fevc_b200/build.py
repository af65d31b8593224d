"""Build ``libfevc_b200.so`` in-tree for sm_100a.

Host C++ (preparation, C ABI) is compiled with g++, device code with nvcc
(``-gencode arch=compute_100a,code=sm_100a``), and everything is linked into one
shared library next to this file, with the CUDA runtime linked statically so
the library needs only the driver at run time.
"""

from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
BUILD = HERE / "_build"
LIB = HERE / "libfevc_b200.so"

CXX_SOURCES = ["prep.cpp", "abi.cpp", "hybrid.cpp", "cmg_host.cpp", "abi_unsupported.cpp", "numerical.cpp",
               "projection.cpp"]
CU_SOURCES = ["engine.cu", "multigrid.cu", "noalloc.cu", "learned.cu", "devmem.cu"]
GENCODE = "-gencode=arch=compute_100a,code=sm_100a"


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build fevc_b200")


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + [INCLUDE / "fevc_b200.h"]


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    newest = max([src.stat().st_mtime] + [h.stat().st_mtime for h in _headers()])
    return obj.stat().st_mtime < newest


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + proc.stdout + proc.stderr)


def build(verbose: bool = False, ptxas_info: bool = False) -> Path:
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    jobs = []
    objs = []
    for name in CXX_SOURCES:
        src, obj = CSRC / name, BUILD / (name + ".o")
        objs.append(obj)
        if _stale(obj, src):
            jobs.append([nvcc, "-x", "c++", "-std=c++17", "-O3", "-Xcompiler", "-fPIC,-Wall,-fopenmp",
                         f"-I{CSRC}", f"-I{INCLUDE}", "-c", str(src), "-o", str(obj)])
    for name in CU_SOURCES:
        src, obj = CSRC / name, BUILD / (name + ".o")
        objs.append(obj)
        if _stale(obj, src):
            cmd = [nvcc, GENCODE, "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp",
                   "--expt-relaxed-constexpr", f"-I{CSRC}", f"-I{INCLUDE}", "-c", str(src), "-o", str(obj)]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as pool:
        for cmd, _ in zip(jobs, pool.map(_run, jobs)):
            if verbose:
                print(" ".join(cmd))
    if jobs or not LIB.exists():
        tmp = LIB.with_suffix(".so.tmp")
        _run([nvcc, GENCODE, "-shared", "-cudart", "static", "-o", str(tmp)] + [str(o) for o in objs]
             + ["-Xcompiler", "-fopenmp", "-Xlinker", "--no-undefined",
                # every kernel launch passes through these two runtime calls;
                # the wrappers in devmem.cu count them
                "-Xlinker", "--wrap=cudaLaunchKernel", "-Xlinker", "--wrap=cudaLaunchCooperativeKernel"])
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))
