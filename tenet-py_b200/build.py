"""Build ``tenet/libtenet_b200.so`` from ``csrc/*.cu`` for sm_100a (in-tree, no JIT cache).

    python tenet-py_b200/build.py

nvcc cross-compiles without a GPU, so this runs on the CPU build machine; the built
library travels with the source tree.
"""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
SOURCES = sorted([*(PKG / "csrc").glob("*.cu"), *(PKG / "csrc").glob("*.cpp")])
OUT = PKG / "tenet" / "libtenet_b200.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared", "-rdc=true", "--expt-relaxed-constexpr",
]


def build(verbose: bool = False) -> Path:
    newest = max(p.stat().st_mtime for p in [*SOURCES, *(PKG / "csrc").glob("*.cuh"),
                                             ROOT / "include" / "tenet_b200.h"])
    if OUT.exists() and OUT.stat().st_mtime >= newest:
        return OUT
    cmd = ["nvcc", *NVCC_FLAGS, f"-I{ROOT / 'include'}", *map(str, SOURCES), "-o", str(OUT)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed:\n{res.stdout}\n{res.stderr}")
    if verbose:
        print(res.stderr)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
