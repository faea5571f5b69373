"""Builds the CUDA library in-tree: ice_b200/lib/libice_gpu.so for sm_100a.

    python -m ice_b200.build [--verbose] [--force]

Each closure's stage kernels are their own translation unit (csrc/ice_fam_*.cu), compiled in
parallel; csrc/ice_gpu.cu holds the C ABI. --fmad=false keeps every product and sum rounded on
its own, as the Fortran source writes them: the plain FP64 form then reproduces the reference's
order of operations.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
SRC = PKG / "csrc"
OBJ = PKG / "lib" / "obj"
OUT = PKG / "lib" / "libice_gpu.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
UNITS = ["ice_gpu.cu", "ice_noalloc.cu", "ice_mlp_f32.cu", "ice_fam_mk.cu", "ice_fam_ig.cu", "ice_fam_ag.cu"] + [
    f"ice_stage_{c}_{p}.cu" for c in ("mk", "ig", "ag") for p in ("f64", "f32")]
# -prec-div=false -prec-sqrt=false -ftz=true act on single precision only: the FP32-flux form
# divides and takes roots at hardware speed; every FP64 operation stays IEEE and unfused.
FLAGS = ["-O3", "-std=c++17", "--fmad=false", "-prec-div=false", "-prec-sqrt=false", "-ftz=true", "-lineinfo",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def headers():
    return sorted(SRC.glob("*.cuh")) + sorted(SRC.glob("*.h")) + [PKG.parent / "include" / "ice_gpu.h"]


def _newer(target: Path, deps) -> bool:
    return target.exists() and all(p.stat().st_mtime <= target.stat().st_mtime for p in deps)


def flags_of(unit: str):
    """The FP32-flux units (*_f32.cu) keep no bit-for-bit tie to the reference's order of operations:
    they contract a*b + c into fused multiply-adds and take single-precision divisions, square roots
    and elementary functions at hardware speed (--use_fast_math, which leaves double precision
    alone). Every other unit keeps --fmad=false."""
    if unit.endswith("_f32.cu"):
        return [f if f != "--fmad=false" else "--fmad=true" for f in FLAGS] + ["--use_fast_math"]
    return FLAGS


def _compile(unit: str, verbose: bool, extra) -> str:
    src = SRC / unit
    obj = OBJ / (unit[:-3] + ".o")
    cmd = [nvcc(), *ARCH, *flags_of(unit), "-c", "-o", str(obj), str(src), *extra]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {unit}:\n{r.stdout}{r.stderr}")
    return r.stderr


def build(force: bool = False, verbose: bool = False, extra=()) -> Path:
    OBJ.mkdir(parents=True, exist_ok=True)
    hs = headers()
    todo = [u for u in UNITS if force or not _newer(OBJ / (u[:-3] + ".o"), [SRC / u, *hs])]
    if todo:
        with ThreadPoolExecutor(max_workers=min(len(todo), os.cpu_count() or 4)) as ex:
            logs = list(ex.map(lambda u: _compile(u, verbose, extra), todo))
        if verbose:
            for u, log in zip(todo, logs):
                sys.stderr.write(f"== {u}\n{log}")
    objs = [OBJ / (u[:-3] + ".o") for u in UNITS]
    if force or todo or not _newer(OUT, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(OUT), *map(str, objs), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}{r.stderr}")
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print(OUT)
