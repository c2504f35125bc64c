"""Builds lib/libnepheline_b200.so from csrc/*.cu for sm_100a (nvcc, no JIT).

The solver's translation units are compiled without FMA contraction and with IEEE division
and square root (-fmad=false -prec-div=true -prec-sqrt=true -ftz=false): the results must
round as the reference's SSE/AVX arithmetic does.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "lib"
LIB = LIB_DIR / "libnepheline_b200.so"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
EXACT = ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"]
HOST = ["-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale() -> bool:
    if not LIB.exists():
        return True
    built = LIB.stat().st_mtime
    deps = list(CSRC.glob("*")) + list(INCLUDE.glob("*.h")) + [Path(__file__)]
    return any(p.stat().st_mtime > built for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles every CUDA source into the shared library (only when a source changed)."""
    if not force and not _stale():
        return LIB
    LIB_DIR.mkdir(exist_ok=True)
    objs = []
    build_dir = PKG / "_build"
    build_dir.mkdir(exist_ok=True)
    for src in sources():
        obj = build_dir / (src.stem + ".o")
        cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", *EXACT, *HOST,
               f"-I{INCLUDE}", f"-I{CSRC}", "-c", str(src), "-o", str(obj)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart"], check=True)
    os.replace(tmp, LIB)
    return LIB


# Where the reference's sources lie in the build container (NPH_REFERENCE overrides); the GPU
# machines only use the libraries built from them.
REFERENCE = Path(os.environ.get("NPH_REFERENCE", "/root/reference"))


def build_oracle() -> None:
    """The checkers under oracle/ (the reference library only where its sources exist)."""
    cmd = ["make", "-s", "-C", str(ROOT / "oracle"), "-j8"]
    if (REFERENCE / "engine" / "physics" / "src" / "solver.c").exists():
        cmd.append(f"REF={REFERENCE}")
    subprocess.run(cmd, check=True)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    if "--oracle" in sys.argv:
        build_oracle()
    print(LIB)
