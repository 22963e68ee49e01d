"""Build the native libraries in-tree (no GPU needed: nvcc cross-compiles for sm_100a).

    python -m specann_b200.build            # both libraries
    python -m specann_b200.build --verbose  # also print ptxas resource usage

Outputs (next to this file):
  libspecann_b200.so   CUDA kernels + the C-ABI of include/specann_b200.h (sm_100a only)
  libspecann_graphs.so seeded synthetic graph generators and the instance loader (host C++, OpenMP)
"""
import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
CUDA_LIB = "libspecann_b200.so"
GRAPH_LIB = "libspecann_graphs.so"
CU_SOURCES = ["capi.cu", "alpha.cu", "ls.cu", "batch.cu", "adjoint.cu", "noalloc.cu", "panel.cu", "split.cu", "coo.cu",
              "guard.cu"]
HEADERS = ["common.cuh", "handle.cuh", "spmv.cuh", "policy.cuh", "alpha_body.cuh", "ls_body.cuh", "panel.cuh"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: Path, sources) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(s).stat().st_mtime > t for s in sources)


NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "--extended-lambda", "-Xcompiler", "-fPIC"]


def build_cuda(verbose: bool = False, force: bool = False) -> Path:
    """Compile every .cu to an object in parallel (build/ under the package), then link."""
    from concurrent.futures import ThreadPoolExecutor
    out = PKG / CUDA_LIB
    srcs = [CSRC / s for s in CU_SOURCES]
    common = [CSRC / h for h in HEADERS] + [ROOT / "include" / "specann_b200.h"]
    if not force and not _stale(out, srcs + common):
        return out
    objdir = PKG / "build"
    objdir.mkdir(exist_ok=True)
    nvcc = nvcc_path()

    def compile_one(src: Path) -> Path:
        obj = objdir / (src.stem + ".o")
        if force or _stale(obj, [src] + common):
            cmd = [nvcc] + NVCC_FLAGS + [f"-I{ROOT / 'include'}", "-c", "-o", str(obj), str(src)]
            if verbose:
                cmd += ["-Xptxas", "-v"]
            subprocess.run(cmd, check=True)
        return obj

    with ThreadPoolExecutor(max_workers=len(srcs)) as ex:
        objs = list(ex.map(compile_one, srcs))
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(out)]
                   + [str(o) for o in objs], check=True)
    return out


def build_graphs(force: bool = False) -> Path:
    """Host library: seeded graph generators and the native instance loader."""
    out = PKG / GRAPH_LIB
    srcs = [CSRC / "graphgen.cpp", CSRC / "loader.cpp", CSRC / "coloring.cpp"]
    if not force and not _stale(out, srcs):
        return out
    cxx = shutil.which("g++") or "g++"
    subprocess.run([cxx, "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-o", str(out)] + [str(s) for s in srcs],
                   check=True)
    return out


def build_all(verbose: bool = False, force: bool = False):
    return build_graphs(force), build_cuda(verbose, force)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    for p in build_all(a.verbose, a.force):
        print(p)
    sys.exit(0)
