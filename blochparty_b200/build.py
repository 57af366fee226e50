"""Builds ``libblochparty_b200.so`` in-tree from ``csrc/`` with nvcc for sm_100a (no GPU needed).

    python -m blochparty_b200.build [--verbose]    # -Xptxas -v register / spill report with --verbose
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
LIB = PKG / "libblochparty_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is needed to build the sm_100a library")
    return cand


def sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    deps = list(CSRC.glob("*")) + [ROOT / "include" / "blochparty_b200.h"]
    return all(p.stat().st_mtime <= t for p in deps)


def build(verbose: bool = False, force: bool = False) -> Path:
    if not force and up_to_date():
        return LIB
    nvcc = _nvcc()
    objdir = ROOT / "_build"
    objdir.mkdir(exist_ok=True)
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Wno-deprecated-gpu-targets", f"-I{ROOT / 'include'}"]

    def compile_one(src: Path) -> str:
        obj = objdir / (src.stem + ".o")
        if src.suffix == ".cu":
            cmd = [nvcc, *ARCH, "-lineinfo", *common, "-c", str(src), "-o", str(obj)]
            if verbose:
                cmd += ["-Xptxas", "-v"]
        else:
            cmd = [nvcc, *common, "-x", "c++", "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr:
            print(r.stderr, file=sys.stderr)
        return str(obj)

    # one nvcc per source, in parallel (the sources are independent translation units)
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        objs = list(pool.map(compile_one, sources()))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force=True)
    print(LIB)
