"""Ahead-of-time build of libhippie_b200.so for sm_100a (B200).

Every CUDA source is compiled with
    nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3 -fmad=false
(-fmad=false: the kernels spell out each fused multiply-add they want, so
that a CPU restatement can reproduce their results bit for bit; k_refarith.cu
is compiled with -use_fast_math, see FILE_FLAGS) and the host
sources with g++ -ffp-contract=off. Objects go to hippie_b200/_build/, the
shared library to hippie_b200/libhippie_b200.so. Rebuilds are incremental
(by modification time of sources and headers).

Usage: python -m hippie_b200.build [--force] [--jobs N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libhippie_b200.so"
CLI_SRC = PKG / "cli" / "bench_main.cpp"
CLI = PKG / "hippie_b200_bench"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-fopenmp",
              "--expt-relaxed-constexpr", "-I", str(INCLUDE)] + ARCH
CXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-fopenmp", "-ffp-contract=off", "-I", str(INCLUDE)]
# k_refarith.cu holds the reference-arithmetic kernels, compiled with the
# reference's own -use_fast_math (approximate quotient, denormals flushed,
# compiler contraction; the flag comes after -fmad=false and overrides it).
FILE_FLAGS = {"k_refarith.cu": ["-use_fast_math", "-fmad=true"]}


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found")
    return cand


def _cuda_include() -> str:
    nvcc = Path(_nvcc()).resolve()
    return str(nvcc.parent.parent / "include")


def _sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers_mtime() -> float:
    hs = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _compile(src: Path, force: bool, hdr_mtime: float) -> Path:
    obj = BUILD / (src.name + ".o")
    if not force and obj.exists():
        if obj.stat().st_mtime >= max(src.stat().st_mtime, hdr_mtime):
            return obj
    if src.suffix == ".cu":
        cmd = [_nvcc()] + NVCC_FLAGS + FILE_FLAGS.get(src.name, []) + ["-c", str(src), "-o", str(obj)]
    else:
        cmd = ["g++"] + CXX_FLAGS + ["-I", _cuda_include(), "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    hdr = _headers_mtime()
    srcs = _sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, hdr), srcs))
    newest = max(o.stat().st_mtime for o in objs)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [_nvcc()] + ARCH + ["-shared", "-o", str(tmp)] + [str(o) for o in objs] + \
              ["-Xcompiler", "-fopenmp", "-lgomp"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
        if verbose:
            print(f"built {LIB}")
    _build_cli(force, verbose)
    return LIB


def _build_cli(force: bool, verbose: bool) -> None:
    """The C++ bench CLI (hippie_b200_bench) over the C++ facade of the C ABI."""
    deps = [CLI_SRC, LIB, INCLUDE / "hippie_b200.hpp", INCLUDE / "hippie_b200.h"]
    if not force and CLI.exists() and CLI.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return
    cuda = Path(_cuda_include()).parent
    cmd = ["g++", "-std=c++17", "-O2", "-I", str(INCLUDE), "-I", _cuda_include(), str(CLI_SRC), "-o", str(CLI),
           "-L", str(PKG), "-lhippie_b200", "-L", str(cuda / "lib64"), "-lcudart_static", "-ldl", "-lrt",
           "-lpthread", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"CLI build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(f"built {CLI}")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    a = ap.parse_args(argv)
    build(force=a.force, jobs=a.jobs, verbose=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
