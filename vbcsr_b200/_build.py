"""In-tree build of the native parts of vbcsr_b200.

Produces, next to this file:
  libvbcsr_b200.so     CUDA kernels + the C ABI of include/vbcsr_b200.h (nvcc, sm_100a)
  vbcsr_core*.so       the pybind11 host core that mirrors the reference's
                       `vbcsr_core` extension on top of that C ABI

Run ``python -m vbcsr_b200._build`` (or ``__graft_entry__.build()``).  nvcc
cross-compiles for sm_100a without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
LIB = HERE / "libvbcsr_b200.so"

CUDA_SOURCES = [
    "vbg_matrix.cu",
    "vbg_apply.cu",
    "vbg_vec.cu",
    "vbg_algebra.cu",
    "vbg_spgemm.cu",
    "vbg_sddmm.cu",
    "vbg_struct.cu",
]
HOST_SOURCES = ["core_module.cpp"]

NVCC_FLAGS = [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, cwd=str(CSRC), capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:4]) + " ...")


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def build_cuda(force: bool = False, verbose: bool = False) -> Path:
    srcs = [CSRC / s for s in CUDA_SOURCES if (CSRC / s).exists()]
    deps = srcs + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "vbcsr_b200.h"]
    if not force and not _stale(LIB, deps):
        return LIB
    objs = []
    for src in srcs:
        obj = CSRC / (src.stem + ".o")
        if force or _stale(obj, [src] + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "vbcsr_b200.h"]):
            cmd = [_nvcc(), *NVCC_FLAGS, "-c", src.name, "-o", obj.name]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
        objs.append(obj.name)
    _run([_nvcc(), "-shared", "-Xcompiler", "-fPIC", *[o for o in objs], "-o", str(LIB), "-lcudart"])
    return LIB


def core_module_path() -> Path:
    suffix = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    return HERE / ("vbcsr_core" + suffix)


def build_host(force: bool = False, verbose: bool = False) -> Path | None:
    srcs = [CSRC / s for s in HOST_SOURCES if (CSRC / s).exists()]
    if not srcs:
        return None
    target = core_module_path()
    deps = srcs + [ROOT / "include" / "vbcsr_b200.h", LIB]
    if not force and not _stale(target, deps):
        return target
    import pybind11

    cuda_inc = "/usr/local/cuda/include"
    cmd = [
        "g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
        f"-I{pybind11.get_include()}", f"-I{sysconfig.get_paths()['include']}", f"-I{cuda_inc}",
        f"-I{ROOT / 'include'}",
        *[str(s) for s in srcs],
        "-o", str(target),
        f"-L{HERE}", "-lvbcsr_b200", "-Wl,-rpath,$ORIGIN",
        "-L/usr/local/cuda/lib64", "-lcudart",
    ]
    if verbose:
        print(" ".join(cmd))
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError("host core build failed")
    return target


def build(force: bool = False, verbose: bool = False) -> None:
    build_cuda(force=force, verbose=verbose)
    build_host(force=force, verbose=verbose)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
