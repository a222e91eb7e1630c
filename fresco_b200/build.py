"""Builds the fresco_b200 CUDA library in-tree with nvcc for sm_100a.

``python fresco_b200/build.py`` (or ``build()``) compiles every ``csrc/*.cu``
to an object under ``fresco_b200/_build/`` (rebuilt only when the source or a
header changed) and links ``fresco_b200/libfresco_b200.so`` against cuFFT and
the CUDA runtime.  No JIT cache is involved, so the built library travels with
the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "libfresco_b200.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "--expt-relaxed-constexpr",
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-fvisibility=hidden",
] + ARCH


def _cuda_home() -> Path:
    env = os.environ.get("CUDA_HOME") or os.environ.get("CUDA_PATH")
    if env:
        return Path(env)
    nvcc = shutil.which("nvcc")
    if nvcc:
        return Path(nvcc).resolve().parent.parent
    return Path("/usr/local/cuda")


def _nvcc() -> str:
    return str(_cuda_home() / "bin" / "nvcc")


def _newest_header() -> float:
    hs = list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _compile(src: Path, verbose: bool) -> Path:
    obj = OBJ / (src.stem + ".o")
    if obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, _newest_header()):
        return obj
    cmd = [_nvcc(), *NVCC_FLAGS, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    OBJ.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu"))
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    newest = max(o.stat().st_mtime for o in objs)
    if LIB.exists() and LIB.stat().st_mtime >= newest:
        return LIB
    cuda = _cuda_home()
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [
        _nvcc(),
        *ARCH,
        "-shared",
        "-o",
        str(tmp),
        *map(str, objs),
        "-L",
        str(cuda / "lib64"),
        "-lcufft",
        "-lcudart",
        "-Xlinker",
        f"-rpath={cuda / 'lib64'}",
    ]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


TORCH_OPS_SRC = CSRC / "torch_ops.cpp"
TORCH_LIB = PKG / "libfresco_torch.so"


def build_torch_ops(verbose: bool = False) -> Path:
    """Compiles the PyTorch operator library (csrc/torch_ops.cpp) against the
    installed torch's headers and libfresco_b200.so into
    fresco_b200/libfresco_torch.so."""
    newest = max(TORCH_OPS_SRC.stat().st_mtime, LIB.stat().st_mtime, _newest_header())
    if TORCH_LIB.exists() and TORCH_LIB.stat().st_mtime >= newest:
        return TORCH_LIB
    import torch
    from torch.utils import cpp_extension

    torch_lib = Path(torch.__file__).resolve().parent / "lib"
    tmp = TORCH_LIB.with_suffix(".so.tmp")
    cmd = [
        os.environ.get("CXX", "g++"),
        "-O2",
        "-std=c++17",
        "-fPIC",
        "-shared",
        f"-D_GLIBCXX_USE_CXX11_ABI={int(torch._C._GLIBCXX_USE_CXX11_ABI)}",
        *[f"-I{p}" for p in cpp_extension.include_paths()],
        f"-I{_cuda_home() / 'include'}",
        f"-I{INCLUDE}",
        str(TORCH_OPS_SRC),
        "-o",
        str(tmp),
        f"-L{torch_lib}",
        "-lc10",
        "-lc10_cuda",
        "-ltorch_cpu",
        f"-L{PKG}",
        "-lfresco_b200",
        "-Wl,-rpath,$ORIGIN",
    ]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"torch operator build failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, TORCH_LIB)
    return TORCH_LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
    print(build_torch_ops(verbose="-v" in sys.argv))
