"""Build libpsycles_cuda.so in-tree for sm_100a.

    python -m psycles_b200.build          # or psycles_b200.build.build()

The CUDA sources are compiled by nvcc with -gencode arch=compute_100a,
code=sm_100a, no fast math and no FMA contraction (-fmad=false: the
kernels spell out every fused operation the reference prescribes); the
host translation unit by g++ with -ffp-contract=off, so host tables are
bit-identical to the reference's construction.
"""

from __future__ import annotations

import os
import pathlib
import shutil
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "libpsycles_cuda.so"
BUILD = HERE / "_build"

CUDA_HOME = pathlib.Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
              "-ftz=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
              "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall", "-Wextra"]

SOURCES_CU = ["psy_kernels.cu", "psy_static.cu"]
SOURCES_CPP = ["psy_host.cpp", "psy_light_tree.cpp", "psy_engine.cpp", "psy_batch.cpp", "psy_server.cpp"]


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target: pathlib.Path, deps: list[pathlib.Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose_ptxas: bool = False, defines: tuple[str, ...] = (),
          out: pathlib.Path | None = None, build_dir: pathlib.Path | None = None) -> pathlib.Path:
    """Compiles the library; `defines` (NAME=VALUE) set the kernel tuning
    macros, `out` / `build_dir` redirect the artefacts."""
    global OUT, BUILD
    out_path, build_path = OUT, BUILD
    if out is not None:
        OUT, BUILD = pathlib.Path(out), pathlib.Path(build_dir or pathlib.Path(out).parent / "_build")
    try:
        return _build(force, verbose_ptxas, [f"-D{d}" for d in defines])
    finally:
        OUT, BUILD = out_path, build_path


def _build(force: bool, verbose_ptxas: bool, defs: list[str]) -> pathlib.Path:
    BUILD.mkdir(exist_ok=True, parents=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [HERE.parent / "include" / "psycles_cuda.h"]
    objects = []
    for src in SOURCES_CU:
        obj = BUILD / (src + ".o")
        objects.append(obj)
        if force or _stale(obj, [CSRC / src] + headers):
            extra = ["-Xptxas", "-v"] if verbose_ptxas else []
            _run([NVCC, *ARCH, *NVCC_FLAGS, *defs, *extra, "-c", str(CSRC / src), "-o", str(obj)])
    cxx = shutil.which("g++") or "g++"
    for src in SOURCES_CPP:
        obj = BUILD / (src + ".o")
        objects.append(obj)
        if force or _stale(obj, [CSRC / src] + headers):
            _run([cxx, *CXX_FLAGS, *defs, f"-I{CUDA_HOME / 'include'}", "-c", str(CSRC / src), "-o", str(obj)])
    if force or _stale(OUT, objects):
        _run([NVCC, *ARCH, "-shared", "-o", str(OUT), *map(str, objects), "-lcudart"])
    return OUT


def main(argv: list[str]) -> None:
    """`--force`, `--ptxas`, `-D NAME=VALUE` (repeatable: a kernel tuning
    macro or the build option PSY_BVH_WIDTH=8) and `--out PATH` (a variant
    library beside the default one; load it with PSYCLES_CUDA_LIB=PATH)."""
    import argparse
    ap = argparse.ArgumentParser(prog="python -m psycles_b200.build")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true")
    ap.add_argument("-D", dest="defines", action="append", default=[])
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    out = pathlib.Path(a.out).resolve() if a.out else None
    build(force=a.force, verbose_ptxas=a.ptxas, defines=tuple(a.defines), out=out)


if __name__ == "__main__":
    main(sys.argv[1:])
