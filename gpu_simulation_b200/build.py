"""In-tree build of the engine for sm_100a.

Produces
  gpu_simulation_b200/librsv.so                  C ABI (include/rsv.h): CUDA kernels + host scheduler
  standalone_backend/_cuda_backend<EXT_SUFFIX>   pybind11 drop-in for the reference's
                                                 standalone_backend._cuda_backend

Usage: python -m gpu_simulation_b200.build [--verbose]
"""

from __future__ import annotations

import os
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "librsv.so"
DROPIN_DIR = ROOT / "standalone_backend"
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["rsv_kernels.cu", "rsv_pass.cu", "rsv_pass_half.cu", "rsv_layer0.cu", "rsv_mps.cu", "rsv_noalloc.cu", "rsv_pass_tma.cu", "rsv_batch.cu", "rsv_mlp.cu", "rsv_gate.cu", "rsv_dense.cu", "rsv_shard.cu"]
CPP_SOURCES = ["rsv_backend.cpp", "rsv_mlp_host.cpp"]
HEADERS = ["rsv_device.cuh", "rsv_types.h", "rsv_launch.h", "rsv_workspace.h", "rsv_tma.h", "rsv_tile.cuh", "rsv_batch.h", "rsv_mlp.h", "rsv_gate.h", "rsv_dense.h"]


def _ext_suffix() -> str:
    return sysconfig.get_config_var("EXT_SUFFIX") or ".so"


def dropin_path() -> Path:
    return DROPIN_DIR / f"_cuda_backend{_ext_suffix()}"


def _newer(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> str:
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    return res.stdout + res.stderr


def build(verbose: bool = False, ptxas_verbose: bool = False) -> Path:
    """Compile librsv.so and the drop-in module if any source changed."""
    BUILD.mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [ROOT / "include" / "rsv.h", ROOT / "include" / "rsv_shard.h"]
    jobs = []
    objs = []
    for src in CU_SOURCES:
        obj = BUILD / (Path(src).stem + ".o")
        objs.append(obj)
        if _newer(obj, [CSRC / src, *headers]) or ptxas_verbose:
            cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                   "-c", str(CSRC / src), "-o", str(obj)]
            if ptxas_verbose:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)
    for src in CPP_SOURCES:
        obj = BUILD / (Path(src).stem + ".o")
        objs.append(obj)
        if _newer(obj, [CSRC / src, *headers]):
            jobs.append(["g++", "-O2", "-std=c++17", "-fPIC", "-Wall", f"-I{CUDA_HOME / 'include'}",
                         "-c", str(CSRC / src), "-o", str(obj)])
    logs = []
    if jobs:
        with ThreadPoolExecutor(max_workers=max(1, len(jobs))) as ex:
            logs = list(ex.map(lambda c: _run(c, verbose), jobs))
    if _newer(LIB, objs):
        _run(["g++", "-shared", "-o", str(LIB), *map(str, objs), f"-L{CUDA_HOME / 'lib64'}",
              "-lcudart", f"-Wl,-rpath,{CUDA_HOME / 'lib64'}"], verbose)
    _build_dropin(verbose)
    if ptxas_verbose:
        for log in logs:
            print(log)
    return LIB


def _build_dropin(verbose: bool) -> Path:
    import pybind11

    src = CSRC / "cuda_backend_pybind.cpp"
    out = dropin_path()
    if not _newer(out, [src, LIB, ROOT / "include" / "rsv.h"]):
        return out
    py_inc = sysconfig.get_paths()["include"]
    rel = os.path.relpath(PKG, DROPIN_DIR)
    _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", f"-I{py_inc}", f"-I{pybind11.get_include()}",
          f"-I{ROOT / 'include'}", str(src), "-o", str(out), f"-L{PKG}", "-lrsv",
          f"-Wl,-rpath,$ORIGIN/{rel}"], verbose)
    return out


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, ptxas_verbose="--ptxas" in sys.argv)
    print(LIB)
    print(dropin_path())
