"""Build the CUDA library and CLI in-tree with nvcc (sm_100a).

Outputs:
  purinecfd_b200/libjst_gpu.so   the C-ABI library (include/jst_gpu.h)
  purinecfd_b200/bin/jst         the `jst` command-line front end

The strict FP64 passes path (passes.cu) is compiled with --fmad=false so no
a*b+c is contracted; the fused path keeps contraction on.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libjst_gpu.so"
CLI = PKG / "bin" / "jst"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-warn-spills",
          f"-I{ROOT / 'include'}", f"-I{CSRC}"]

# source -> extra flags
UNITS = {
    "passes.cu": ["--fmad=false"],
    "fused.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
    "api.cu": [],
    "noalloc.cu": [],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _newer(out: Path, deps) -> bool:
    if not out.exists():
        return False
    t = out.stat().st_mtime
    return all(Path(d).stat().st_mtime <= t for d in deps)


def _headers():
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "jst_gpu.h", Path(__file__)]


def compile_unit(src: str, flags, verbose=False) -> Path:
    obj = BUILD / (Path(src).stem + ".o")
    deps = [CSRC / src] + _headers()
    if _newer(obj, deps):
        return obj
    cmd = [nvcc(), *ARCH, *COMMON, *flags, "-c", str(CSRC / src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stderr.strip() or r.stdout.strip()):
        print(r.stdout + r.stderr)
    return obj


def build(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    with ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        objs = list(ex.map(lambda kv: compile_unit(kv[0], kv[1], verbose), UNITS.items()))
    if not _newer(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(LIB), *map(str, objs)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    CLI.parent.mkdir(exist_ok=True)
    cli_src = CSRC / "cli.cpp"
    if cli_src.exists() and not _newer(CLI, [cli_src, LIB]):
        cmd = [nvcc(), "-O2", "-std=c++17", f"-I{ROOT / 'include'}", str(cli_src), "-o", str(CLI),
               f"-L{PKG}", "-ljst_gpu", "-Xlinker", "-rpath=$ORIGIN/.."]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"CLI build failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(f"built {LIB}")
