"""Builds libturbo_b200.so in-tree with nvcc for sm_100a, and the thin libtorch autograd
wrapper of its differentiable decoder (turbo_cpp_b200/lib/torch_ext/turbo_torch*.so), which the
scale-training harness imports; both are built here once and loaded from their files."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libturbo_b200.so")
SOURCES = ["decoder.cu", "chain.cu", "noalloc.cu", "adjoint.cu", "generate.cu", "lte_codec.cpp", "capi.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def build(verbose: bool = False, extra: list[str] | None = None) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--shared", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "-Xcompiler", "-Wall",
           "-I", os.path.join(HERE, "..", "include"), *srcs, "-o", LIB + ".tmp", "-lcudart"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    cmd += list(extra or [])
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


TORCH_EXT_DIR = os.path.join(LIB_DIR, "torch_ext")
TORCH_EXT_NAME = "turbo_torch"


def build_torch(verbose: bool = False) -> str:
    """Compiles csrc/torch_adjoint.cpp against libtorch and libturbo_b200.so (found next to the
    extension through its run path, so the same library copy as the ctypes mirror is used)."""
    from torch.utils import cpp_extension

    os.makedirs(TORCH_EXT_DIR, exist_ok=True)
    cpp_extension.load(
        name=TORCH_EXT_NAME, sources=[os.path.join(CSRC, "torch_adjoint.cpp")],
        extra_include_paths=[os.path.join(HERE, "..", "include")],
        extra_cflags=["-O2"],
        extra_ldflags=[f"-L{LIB_DIR}", "-lturbo_b200", "-Wl,-rpath,'$$ORIGIN/..'"],
        build_directory=TORCH_EXT_DIR, with_cuda=True, verbose=verbose)
    return torch_ext_path()


def torch_ext_path() -> str:
    import glob

    found = sorted(glob.glob(os.path.join(TORCH_EXT_DIR, TORCH_EXT_NAME + "*.so")))
    if not found:
        raise ImportError(f"the torch extension is missing from {TORCH_EXT_DIR}: run "
                          "`python turbo_cpp_b200/build.py`")
    return found[0]


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
    if "--no-torch" not in sys.argv:
        print(build_torch(verbose="-v" in sys.argv))
