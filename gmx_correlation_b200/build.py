"""In-tree build of libgmxcorr_b200.so (CUDA kernels for sm_100a + C ABI +
C++ drop-in) and the standalone CLI.

    python -m gmx_correlation_b200.build [--force] [--verbose]

Objects go to gmx_correlation_b200/_build/, the library and CLI next to this
file, so they travel with the source tree.  Incremental: a target is rebuilt
when any of its sources or the shared headers is newer.
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libgmxcorr_b200.so"
CLI = PKG / "gmx_correlation_b200"
INCLUDE = ROOT / "include"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
# The system compilers; the image's CC/CXX wrappers lack OpenMP specs.
CXX = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "--expt-relaxed-constexpr", "-ccbin", CXX,
                     f"-I{INCLUDE}", f"-I{CSRC}", f"-I{CSRC / 'dropin'}"]
CXX_FLAGS = ["-O2", "-fPIC", "-std=c++17", "-ffp-contract=off", f"-I{INCLUDE}", f"-I{CSRC}",
             f"-I{CSRC / 'dropin'}", f"-I{CUDA_HOME / 'include'}"]

# Extra preprocessor definitions for both compilers (build-time settings of
# the kernels, e.g. GC_EXTRA_DEFS="-DGC_BAND_CAP=16"); empty for the product.
EXTRA_DEFS = os.environ.get("GC_EXTRA_DEFS", "").split()
NVCC_FLAGS += EXTRA_DEFS
CXX_FLAGS += EXTRA_DEFS

CU_SOURCES = sorted(CSRC.glob("*.cu"))
CPP_SOURCES = sorted(CSRC.glob("*.cpp")) + sorted((CSRC / "dropin").glob("*.cpp"))
HEADERS = (sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))
           + sorted((CSRC / "dropin").glob("*.h")))


def _newer(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    res = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} ... {cmd[-1]}")
    return res.stdout + res.stderr


def build(force: bool = False, verbose: bool = False, ptxas_report: Path | None = None) -> Path:
    """Compile every CUDA and host source and link the shared library."""
    if shutil.which(NVCC) is None and not Path(NVCC).exists():
        raise RuntimeError(f"nvcc not found at {NVCC}")
    BUILD.mkdir(exist_ok=True)
    objs = []
    reports = []
    for src in CU_SOURCES:
        obj = BUILD / (src.stem + ".cu.o")
        objs.append(obj)
        if force or _newer(obj, [src, *HEADERS]):
            extra = ["-Xptxas", "-v"] if ptxas_report is not None else []
            out = _run([NVCC, *NVCC_FLAGS, *extra, "-c", src, "-o", obj], verbose)
            if ptxas_report is not None:
                reports.append(f"== {src.name}\n{out}")
    for src in CPP_SOURCES:
        obj = BUILD / (src.stem + ".cpp.o")
        objs.append(obj)
        if force or _newer(obj, [src, *HEADERS]):
            _run([CXX, *CXX_FLAGS, "-c", src, "-o", obj], verbose)
    if force or _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-ccbin", CXX, "-Xlinker", "-Bsymbolic", "-o", LIB, *objs,
              "-lcudart_static", "-lrt", "-lpthread", "-ldl"], verbose)
    cli_src = CSRC / "cli" / "main.cpp"
    if cli_src.exists() and (force or _newer(CLI, [cli_src, LIB, *HEADERS])):
        _run([CXX, *CXX_FLAGS, cli_src, "-o", CLI, f"-L{PKG}", "-lgmxcorr_b200",
              f"-Wl,-rpath,$ORIGIN"], verbose)
    if ptxas_report is not None and reports:
        ptxas_report.write_text("\n".join(reports))
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", type=Path, default=None, help="write -Xptxas -v output here")
    a = ap.parse_args(argv)
    lib = build(force=a.force or a.ptxas is not None, verbose=a.verbose, ptxas_report=a.ptxas)
    print(lib)


if __name__ == "__main__":
    main()
