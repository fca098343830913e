"""Build the oracle's C restatement (CPU baseline) into oracle/_build/ -- test infrastructure."""
from __future__ import annotations

import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "cpu_energy.c"
OUT = HERE / "_build" / "libcpuenergy.so"


def build(force: bool = False) -> Path:
    if OUT.exists() and not force and OUT.stat().st_mtime >= SRC.stat().st_mtime:
        return OUT
    OUT.parent.mkdir(exist_ok=True)
    cmd = ["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", str(SRC), "-o", str(OUT)]
    subprocess.run(cmd, check=True)
    return OUT
