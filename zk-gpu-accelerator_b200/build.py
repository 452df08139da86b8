"""Build libzkb200.so (the sm_100a kernels and their C ABI) in-tree.

    python zk-gpu-accelerator_b200/build.py [--force]

Each csrc/*.cu compiles to an object with nvcc for sm_100a only, in
parallel; the objects link into zkgpu/libzkb200.so next to the Python
package that loads it. A source or header newer than the library triggers a
rebuild.
"""

from __future__ import annotations

import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
OUT = HERE / "zkgpu" / "libzkb200.so"
OBJ_DIR = HERE / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-diag-suppress", "177"]


def _nvcc() -> str:
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libzkb200.so")
    return nvcc


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _inputs() -> list[Path]:
    return sources() + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))


def up_to_date() -> bool:
    if not OUT.exists():
        return False
    built = OUT.stat().st_mtime
    return all(p.stat().st_mtime <= built for p in _inputs())


def _compile(nvcc: str, src: Path) -> Path:
    obj = OBJ_DIR / (src.stem + ".o")
    cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stdout}\n{res.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile every csrc/*.cu for sm_100a and link zkgpu/libzkb200.so; returns its path."""
    if not force and up_to_date():
        return OUT
    nvcc = _nvcc()
    OBJ_DIR.mkdir(exist_ok=True)
    srcs = sources()
    workers = min(len(srcs), os.cpu_count() or 1)
    with concurrent.futures.ThreadPoolExecutor(max_workers=workers) as pool:
        objs = list(pool.map(lambda s: _compile(nvcc, s), srcs))
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    tmp.replace(OUT)
    if verbose:
        print(f"built {OUT}", file=sys.stderr)
    return OUT


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--force", action="store_true", help="rebuild even if up to date")
    args = ap.parse_args()
    print(build(force=args.force, verbose=True))


if __name__ == "__main__":
    main()
