"""Builds libsincgpu.so (CUDA, sm_100a) in-tree with nvcc.

The library is compiled from v1-1_b200/csrc/*.cu into v1-1_b200/sincgpu/.
No JIT cache is used: the .so travels with the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
CSRC = PKG_DIR.parent / "csrc"
REPO = PKG_DIR.parent.parent
LIB = PKG_DIR / "libsincgpu.so"
BUILD_DIR = PKG_DIR.parent / "_build"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
    "-I", str(REPO / "include"),
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _compile(src: Path, obj: Path, extra: list[str]) -> str:
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    return r.stderr


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    deps = sources() + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + list((REPO / "include").glob("*.h"))
    return all(p.stat().st_mtime <= t for p in deps)


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> Path:
    if not force and up_to_date():
        return LIB
    BUILD_DIR.mkdir(exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_v else []
    objs = []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        futs = {}
        for src in sources():
            obj = BUILD_DIR / (src.stem + ".o")
            objs.append(obj)
            futs[ex.submit(_compile, src, obj, extra)] = src
        for f in cf.as_completed(futs):
            msg = f.result()
            if verbose and msg:
                print(f"--- {futs[f].name}\n{msg}", file=sys.stderr)
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(tmp), *map(str, objs)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_v="-v" in sys.argv)
    print(LIB)
