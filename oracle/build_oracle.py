"""Compile the oracle's C helper (TEST INFRASTRUCTURE).

oracle/fd_apply.c -> oracle/liboracle_fd.so with gcc and OpenMP.  Only the
oracle loads the library; the product never does.  Plain x86-64 code (no
-march flags), so the library built here also runs on other hosts.

Usage: python oracle/build_oracle.py
"""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "fd_apply.c"
LIB = HERE / "liboracle_fd.so"


def needs_build() -> bool:
    return not LIB.exists() or LIB.stat().st_mtime < SRC.stat().st_mtime


def build(force: bool = False) -> Path:
    if not force and not needs_build():
        return LIB
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        raise RuntimeError("no C compiler found for the oracle helper")
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [cc, "-O3", "-fopenmp", "-fPIC", "-shared", "-o", str(tmp), str(SRC)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle helper build failed:\n{res.stdout}\n{res.stderr}")
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
