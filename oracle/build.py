"""Builds the C oracle ``oracle/liboracle_bloch.so`` from ``oracle/bloch_c.c`` with gcc (OpenMP, float64, no
fast-math) — TEST INFRASTRUCTURE ONLY, like everything under ``oracle/``.

    python -m oracle.build
"""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "bloch_c.c"
LIB = HERE / "liboracle_bloch.so"


def build(force: bool = False) -> Path:
    if not force and LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        raise RuntimeError("no C compiler (gcc) for the oracle")
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [cc, "-O2", "-std=c11", "-fopenmp", "-fPIC", "-shared", "-fno-fast-math", "-ffp-contract=off", str(SRC),
           "-o", str(tmp), "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"gcc failed on {SRC.name}:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
