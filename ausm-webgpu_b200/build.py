"""Build libausm.so (sm_100a) in-tree: ausm-webgpu_b200/lib/libausm.so.

    python ausm-webgpu_b200/build.py [--force] [--verbose]

Each .cu file under csrc/ is compiled by nvcc for sm_100a only, and with -fmad=false:
the compiler contracts no multiply and add on its own.  The reference-shaped engine
and the grid/force/layout kernels thereby keep the reference's float arithmetic
operation by operation; the fused engines write each fused multiply-add explicitly
(fmaf, packed f32x2), so every expression rounds the same way in every kernel that
inlines it.  The CUDA runtime is linked statically so the library has no torch or
Python dependency.  ptxas resource usage (-Xptxas -v) goes to lib/ptxas.log.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "lib"
OUT = LIB / "libausm.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include"), "-I", str(CSRC),
          "-Xptxas", "-v", "--expt-relaxed-constexpr", "-fmad=false"]


def sources():
    return sorted(CSRC.glob("*.cu"))


def _deps():
    return sources() + sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "ausm.h", Path(__file__)]


def up_to_date() -> bool:
    if not OUT.exists():
        return False
    t = OUT.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in _deps())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and up_to_date():
        return OUT
    LIB.mkdir(exist_ok=True)
    objdir = LIB / "obj"
    objdir.mkdir(exist_ok=True)

    def compile_one(src: Path):
        obj = objdir / (src.stem + ".o")
        flags = list(COMMON)
        cmd = [NVCC, *ARCH, *flags, "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
        return obj, r.stderr

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(compile_one, sources()))
    (LIB / "ptxas.log").write_text("".join(log for _, log in results))
    objs = [str(o) for o, _ in results]
    cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", *objs, "-o", str(OUT)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print((LIB / "ptxas.log").read_text())
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
