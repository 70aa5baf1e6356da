"""Builds libgjxl_b200.so in-tree with nvcc for sm_100a.

Every .cu and .cpp under gjxl_b200/csrc is compiled separately (objects in
gjxl_b200/_build) and linked into gjxl_b200/libgjxl_b200.so. Objects are
rebuilt when their source or any header in csrc/ or include/ is newer.

All device code uses --fmad=false so that multiply-add pairs round twice, as
in the reference's x86 build; fused multiply-adds are written explicitly.
"""

from __future__ import annotations

import concurrent.futures
import os
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
CSRC = PACKAGE / "csrc"
INCLUDE = ROOT / "include"
BUILD = PACKAGE / "_build"
LIBRARY = PACKAGE / "libgjxl_b200.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC",
          "-Xcompiler", "-ffp-contract=off",
          "-Xcompiler", "-fvisibility=hidden", "-I", str(INCLUDE), "-I", str(CSRC)]


def _headers_mtime() -> float:
    paths = (list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.inc"))
             + list(INCLUDE.glob("*.h")))
    return max((p.stat().st_mtime for p in paths), default=0.0)


def _compile(source: Path, verbose: bool) -> Path:
    obj = BUILD / (source.name + ".o")
    newest = max(source.stat().st_mtime, _headers_mtime(), Path(__file__).stat().st_mtime)
    if obj.exists() and obj.stat().st_mtime >= newest:
        return obj
    cmd = [NVCC, *ARCH, *COMMON, "-c", str(source), "-o", str(obj)]
    if source.suffix == ".cu":
        cmd[1:1] = ["-Xptxas", "-warn-spills"]
    if verbose:
        print(" ".join(cmd), flush=True)
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"nvcc failed for {source.name}:\n{result.stdout}\n{result.stderr}")
    if result.stderr.strip() and verbose:
        print(result.stderr, file=sys.stderr)
    return obj


def build(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as pool:
        objects = list(pool.map(lambda s: _compile(s, verbose), sources))
    newest = max(o.stat().st_mtime for o in objects)
    if not LIBRARY.exists() or LIBRARY.stat().st_mtime < newest:
        cmd = [NVCC, *ARCH, "-shared", "-o", str(LIBRARY), *map(str, objects),
               "-lcudart", "-Xlinker", "--no-undefined"]
        if verbose:
            print(" ".join(cmd), flush=True)
        result = subprocess.run(cmd, capture_output=True, text=True)
        if result.returncode != 0:
            raise RuntimeError(f"link failed:\n{result.stdout}\n{result.stderr}")
    return LIBRARY


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
