"""Build the oracle's native helper (TEST INFRASTRUCTURE ONLY): oracle/_bin/ba_graph, the stand-alone
graph writer the CPU baseline runs so that its own process loads none of the product's libraries.

    python -m oracle.build_tools
"""
import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
BIN = HERE / "_bin" / "ba_graph"
SOURCES = [HERE / "ba_graph_main.cpp", ROOT / "specann_b200" / "csrc" / "graphgen.cpp"]


def build(force: bool = False) -> Path:
    if not force and BIN.exists() and all(BIN.stat().st_mtime >= s.stat().st_mtime for s in SOURCES):
        return BIN
    BIN.parent.mkdir(exist_ok=True)
    cxx = shutil.which("g++") or "g++"
    subprocess.run([cxx, "-O3", "-std=c++17", "-fopenmp", "-o", str(BIN)] + [str(s) for s in SOURCES], check=True)
    return BIN


if __name__ == "__main__":
    print(build(force=True))
