"""ORACLE — test infrastructure only: build recipe for the CPU checkers.

  oracle/_build/libausm_oracle.so  the restatement (ausm_oracle.cpp), float + double
  oracle/_ref/libausm_ref.so       the reference's own WGSL compute shaders, translated to
                                   C++ by wgsl_ref/translate.py from the reference tree and
                                   driven by wgsl_ref/ref_harness.cpp (main.js dispatch order)

Both are built with -ffp-contract=off so float arithmetic is plain IEEE single precision
without fused multiply-add.  The reference tree is only read when it is present (it is
absent on GPU hosts, which use the prebuilt libraries that travel with the repository).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build"
REF_OUT = HERE / "_ref"
# The reference tree: AUSM_REFERENCE_ROOT, else where this build recipe finds it in the
# build container.  This recipe is the one place that names that location.
REF_SRC = Path(os.environ.get("AUSM_REFERENCE_ROOT", "/root/reference"))

CXXFLAGS = ["-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-Wall", "-Wno-unused"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(map(str, cmd))}\n{r.stdout}\n{r.stderr}")


def _newer(out: Path, deps) -> bool:
    if not out.exists():
        return False
    t = out.stat().st_mtime
    return all(Path(d).stat().st_mtime <= t for d in deps)


def build_oracle(force: bool = False, contract: bool = False) -> Path:
    """The restatement; contract=True builds it with fused multiply-add contraction
    (-ffp-contract=fast -mfma) into oracle/_build_fma/, a second float32 rounding of the
    same arithmetic (for the float32 spread of long runs)."""
    out_dir = HERE / "_build_fma" if contract else BUILD
    out_dir.mkdir(exist_ok=True)
    out = out_dir / "libausm_oracle.so"
    src = HERE / "ausm_oracle.cpp"
    flags = [f for f in CXXFLAGS if f != "-ffp-contract=off"] + ["-ffp-contract=fast", "-mfma"] if contract else CXXFLAGS
    if force or not _newer(out, [src, __file__]):
        _run(["g++", "-std=c++17", *flags, "-shared", str(src), "-o", str(out)])
    return out


def build_ref(force: bool = False, contract: bool = False) -> Path | None:
    """Translate and compile the reference's shaders; returns None when the tree is absent.
    contract=True builds the same sources with fused multiply-add contraction
    (-ffp-contract=fast -mfma) into oracle/_ref_fma/: a second float32 rounding of the
    reference's own arithmetic, used to measure how far two float32 builds of the
    reference drift apart on a long run."""
    out_dir = HERE / "_ref_fma" if contract else REF_OUT
    out = out_dir / "libausm_ref.so"
    if not (REF_SRC / "src" / "shaders" / "ausm.js").exists():
        return out if out.exists() else None
    sys.path.insert(0, str(HERE / "wgsl_ref"))
    import translate  # noqa: E402

    deps = [HERE / "wgsl_ref" / f for f in ("translate.py", "wgsl_rt.h", "ref_harness.cpp")] + [Path(__file__)]
    deps += list((REF_SRC / "src").rglob("*.js"))
    if not force and _newer(out, deps):
        return out
    gen = out_dir / "gen"
    objdir = out_dir / "obj"
    objdir.mkdir(parents=True, exist_ok=True)
    sources = translate.translate_reference(REF_SRC, gen) + [HERE / "wgsl_ref" / "ref_harness.cpp"]
    inc = ["-I", str(HERE / "wgsl_ref"), "-I", str(gen)]
    flags = [f for f in CXXFLAGS if f != "-ffp-contract=off"] + ["-ffp-contract=fast", "-mfma"] if contract else CXXFLAGS

    def compile_one(s: Path):
        o = objdir / (s.stem + ".o")
        _run(["g++", "-std=c++20", *flags, *inc, "-c", str(s), "-o", str(o)])
        return o

    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        objs = list(ex.map(compile_one, sources))
    _run(["g++", "-shared", "-fopenmp", *map(str, objs), "-o", str(out)])
    return out


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    print(build_ref(force="--force" in sys.argv))
