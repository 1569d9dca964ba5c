"""Build libmrsim_acq_cuda.so in-tree for sm_100a (nvcc; no JIT, no torch extension).

The library is plain CUDA C++ behind a C ABI: nvcc compiles every .cu/.cpp under csrc/ with
`-gencode arch=compute_100a,code=sm_100a -lineinfo`, links the CUDA runtime statically, and
writes the shared object next to this file, where the ctypes loader finds it.
"""
from __future__ import annotations

import os
import pathlib
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = pathlib.Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OBJ = HERE / "_build"
LIB = HERE / "libmrsim_acq_cuda.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


# Files whose FP64 arithmetic must round as the reference's does: no multiply-add contraction in
# device or host code.
NO_CONTRACT = {"spin_history.cu", "tseg_fit.cu"}


def _flags(src: pathlib.Path) -> list[str]:
    extra = ["-fmad=false", "-Xcompiler", "-ffp-contract=off"] if src.name in NO_CONTRACT else []
    common = extra + ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "-I", str(HERE.parent / "include")]
    if src.suffix == ".cu":
        return common + ARCH + ["-lineinfo", "-Xptxas", "-O3"]
    return common + ["-x", "cu"] + ARCH


def build(verbose: bool = False, force: bool = False) -> pathlib.Path:
    OBJ.mkdir(exist_ok=True)
    srcs = sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))
    headers = list(CSRC.glob("*.h")) + list((HERE.parent / "include").glob("*.h"))
    newest_header = max((h.stat().st_mtime for h in headers), default=0.0)
    exe = nvcc()

    def compile_one(src: pathlib.Path) -> pathlib.Path:
        obj = OBJ / (src.name + ".o")
        if not force and obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, newest_header):
            return obj
        cmd = [exe, "-c", str(src), "-o", str(obj)] + _flags(src)
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr.strip():
            print(r.stderr, file=sys.stderr)
        return obj

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, srcs))
    if force or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [exe, "-shared", "-o", str(LIB)] + [str(o) for o in objs] + ARCH + [
            "-cudart", "static", "-Xcompiler", "-fvisibility=hidden", "-lpthread", "-lz"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
