"""Build the C oracle (test infrastructure) into ``oracle/_build/libswe_oracle.so``.

    python oracle/build.py

gcc flags: ``-O3 -march=x86-64-v3 -fopenmp -ffp-contract=off`` -- no fast-math
and no FMA contraction, so every float operation is rounded on its own, in the
order the reference NumPy solver performs it.
"""

from __future__ import annotations

import pathlib
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
OUT = HERE / "_build" / "libswe_oracle.so"
SOURCES = [HERE / "swe_oracle.c"]
DEPS = SOURCES + [HERE / "swe_oracle_impl.h"]


def build(force: bool = False) -> pathlib.Path:
    """Compile the oracle if it is missing or older than its sources."""
    if not force and OUT.exists() and all(OUT.stat().st_mtime >= p.stat().st_mtime for p in DEPS):
        return OUT
    OUT.parent.mkdir(parents=True, exist_ok=True)
    cmd = [
        "gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
        "-fPIC", "-shared", "-std=c11", "-Wall", "-Wno-unknown-pragmas",
        *map(str, SOURCES), "-o", str(OUT), "-lm",
    ]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
