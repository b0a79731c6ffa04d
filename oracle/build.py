"""Build recipe of the CPU oracle (test infrastructure): g++ -O2 -fopenmp on oracle.cpp
into oracle/_build/liboracle.so."""
from __future__ import annotations

import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "oracle.cpp"
OUT = HERE / "_build" / "liboracle.so"


def build(force: bool = False) -> Path:
    if not force and OUT.exists() and OUT.stat().st_mtime >= SRC.stat().st_mtime:
        return OUT
    OUT.parent.mkdir(exist_ok=True)
    tmp = OUT.with_suffix(".so.tmp")
    subprocess.run(["g++", "-O2", "-fopenmp", "-fPIC", "-shared", "-std=c++17", str(SRC), "-o", str(tmp)], check=True)
    tmp.replace(OUT)
    return OUT


if __name__ == "__main__":
    print(build(force=True))
