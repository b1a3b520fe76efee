"""Build libippi_lbm.so (the C-ABI library) in-tree for sm_100a.

    python build.py [--force] [-j N]

Every .cu under csrc/ is compiled by nvcc with
    -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo -std=c++17
into csrc/_build/*.o (in parallel), then linked with the CUDA runtime
(static) into ./libippi_lbm.so next to this file.  Incremental: a unit is
rebuilt when it or any header under csrc/ or include/ is newer than its
object.  nvcc cross-compiles, so this runs without a GPU.

Then the C++ host layer (host/: the reference's Mesh / Lattice classes and
its main.cpp driver over the C ABI) is compiled with the host compiler into
./ippi_main, linked against ./libippi_lbm.so, and the libtorch extension
(torch_ext/ippi_autograd.cpp: torch::autograd::Function wrappers of the
adjoint over the C ABI) into ./torch_ext/_build/ippi_autograd.so with
torch.utils.cpp_extension, in-tree.
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
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(CSRC, "_build")
LIB = os.path.join(HERE, "libippi_lbm.so")
HOST = os.path.join(HERE, "host")
MAIN = os.path.join(HERE, "ippi_main")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
         "-I", os.path.join(REPO, "include")]
# Units whose arithmetic is FP32 (populations stored as FP32/FP16/BF16) use
# the hardware reciprocal and square root: their error (< 2 ulp) is far below
# the FP32 parity tolerance.  The FP64 unit keeps IEEE division and sqrt.
FAST_FP32 = {"kernels_f32.cu", "kernels_f16.cu", "kernels_bf16.cu"}
FAST_FLAGS = ["-ftz=true", "-prec-div=false", "-prec-sqrt=false"]
# Units whose FP64 results must equal a sequential CPU restatement bit for
# bit: no FMA contraction.
NO_FMA = {"tau_scan.cu"}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newest_header() -> float:
    hdrs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(REPO, "include", "*.h"))
    return max(os.path.getmtime(h) for h in hdrs)


def _compile(src: str, force: bool) -> str:
    obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src),
                                                                           _newest_header()):
        return obj
    extra = FAST_FLAGS if os.path.basename(src) in FAST_FP32 else []
    if os.path.basename(src) in NO_FMA:
        extra = extra + ["-fmad=false"]
    cmd = [nvcc(), *ARCH, *FLAGS, *extra, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
    return obj


def build(force: bool = False, jobs: int | None = None) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    build_host(force)
    build_torch_ext(force)
    return LIB


def cxx() -> str:
    for cand in (os.environ.get("IPPI_CXX"), "/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("g++ not found")


def build_host(force: bool = False) -> str:
    """ippi_main: host/*.cpp (Mesh, Lattice, the driver) against libippi_lbm.so."""
    srcs = sorted(glob.glob(os.path.join(HOST, "*.cpp")))
    deps = srcs + glob.glob(os.path.join(HOST, "*.h")) + [LIB, os.path.join(REPO, "include", "ippi_lbm.h")]
    if not force and os.path.exists(MAIN) and os.path.getmtime(MAIN) >= max(map(os.path.getmtime, deps)):
        return MAIN
    cmd = [cxx(), "-std=c++17", "-O2", "-Wall", "-I", os.path.join(REPO, "include"), "-I", HOST, *srcs,
           "-o", MAIN, "-L", HERE, "-lippi_lbm", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"host build failed:\n{r.stderr}")
    return MAIN


TORCH_EXT = os.path.join(HERE, "torch_ext")
TORCH_EXT_SO = os.path.join(TORCH_EXT, "_build", "ippi_autograd.so")


def build_torch_ext(force: bool = False) -> str:
    """torch_ext/_build/ippi_autograd.so: the libtorch extension (C++, no
    device code of its own) linked against libippi_lbm.so."""
    src = os.path.join(TORCH_EXT, "ippi_autograd.cpp")
    deps = [src, LIB, os.path.join(REPO, "include", "ippi_lbm.h")]
    if not force and os.path.exists(TORCH_EXT_SO) and os.path.getmtime(TORCH_EXT_SO) >= max(map(os.path.getmtime, deps)):
        return TORCH_EXT_SO
    from torch.utils import cpp_extension

    bdir = os.path.dirname(TORCH_EXT_SO)
    os.makedirs(bdir, exist_ok=True)
    cpp_extension.load(name="ippi_autograd", sources=[src], build_directory=bdir, with_cuda=False,
                       extra_cflags=["-O2"], extra_include_paths=[os.path.join(REPO, "include")],
                       extra_ldflags=[f"-L{HERE}", "-lippi_lbm", f"-Wl,-rpath,{HERE}"], verbose=False)
    os.utime(TORCH_EXT_SO, None)
    return TORCH_EXT_SO


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    a = ap.parse_args()
    print(build(a.force, a.j))
    sys.exit(0)
