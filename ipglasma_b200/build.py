"""Build recipe of the CUDA library (sm_100a) and the host executable.

    python -m ipglasma_b200.build            # library + executable
    python -m ipglasma_b200.build --verbose  # also print -Xptxas -v

Outputs, in-tree so they travel with the repository snapshot:
    ipglasma_b200/libipglasma_b200.so   the C-ABI library (include/ipglasma_b200.h)
    ipglasma_b200/ipglasma_b200         the drop-in executable
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
HOST = PKG / "host"
LIB = PKG / "libipglasma_b200.so"
EXE = PKG / "ipglasma_b200"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC"]
CU_SOURCES = ["api.cu", "evolve.cu", "init.cu", "poisson.cu", "observables.cu", "reduce.cu",
              "noalloc.cu", "adjoint.cu", "nuclei.cu", "writers_gpu.cu", "gaugefix.cu"]
# the GPU writer rounds every sum and product on its own, as the host writer
# (g++ -ffp-contract=off) does, so its text is byte-identical
CU_EXTRA_FLAGS = {"writers_gpu.cu": ["-fmad=false"]}
CPP_SOURCES = ["writers.cpp"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd: list[str]) -> str:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"command failed ({res.returncode}): {' '.join(cmd)}\n"
                           f"{res.stdout}\n{res.stderr}")
    return res.stdout + res.stderr


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build_library(verbose: bool = False, force: bool = False) -> Path:
    deps = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + \
        sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cpp")) + \
        [ROOT / "include" / "ipglasma_b200.h"]
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    nvcc = _nvcc()
    objs = []
    for src in CU_SOURCES:
        obj = objdir / (Path(src).stem + ".o")
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, *CU_EXTRA_FLAGS.get(src, []), "-I",
               str(ROOT / "include"), "-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        out = _run(cmd)
        if verbose and out:
            print(out)
        objs.append(str(obj))
    # host-only sources (writers): plain g++, no FP contraction, so the text
    # output is computed with the reference's operation order and rounding
    cxx = shutil.which("g++") or "g++"
    for src in CPP_SOURCES:
        obj = objdir / (Path(src).stem + ".o")
        _run([cxx, "-O2", "-std=c++17", "-fPIC", "-pthread", "-ffp-contract=off", "-I",
              str(ROOT / "include"), "-c", str(CSRC / src), "-o", str(obj)])
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    _run([nvcc, *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart"])
    tmp.replace(LIB)
    return LIB


def build_executable(force: bool = False) -> Path | None:
    srcs = sorted(HOST.glob("*.cpp"))
    if not srcs:
        return None
    deps = srcs + sorted(HOST.glob("*.h")) + [ROOT / "include" / "ipglasma_b200.h", LIB]
    if not force and not _stale(EXE, deps):
        return EXE
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-O2", "-std=c++17", "-I", str(ROOT / "include"), *map(str, srcs),
           "-o", str(EXE), "-L", str(PKG), "-lipglasma_b200",
           "-Wl,-rpath,$ORIGIN", "-lm"]
    _run(cmd)
    return EXE


def main(argv: list[str]) -> int:
    verbose = "--verbose" in argv
    force = "--force" in argv
    lib = build_library(verbose=verbose, force=force)
    exe = build_executable(force=force)
    print(f"built {lib}" + (f" and {exe}" if exe else ""))
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
