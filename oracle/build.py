"""Build recipe of the CPU oracle (test infrastructure only): oracle/liblworacle.so from lw_oracle.cpp.

-ffp-contract=off keeps every float expression rounded as written (the GPU library is built with -fmad=false),
so the integer outputs of the two agree bit for bit. OpenMP is used when the compiler supports it; the oracle's
results do not depend on the thread count except for the float64 summation order of the ICP accumulator.
"""

from __future__ import annotations

import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "lw_oracle.cpp"
OUT = HERE / "liblworacle.so"
FLAGS = ["-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math"]


def compilers():
    for c in ("/usr/bin/g++", shutil.which("g++"), shutil.which("c++")):
        if c:
            yield c


def build(force: bool = False) -> Path:
    if not force and OUT.exists() and OUT.stat().st_mtime >= SRC.stat().st_mtime:
        return OUT
    err = ""
    for cxx in compilers():
        for extra in (["-fopenmp"], []):
            r = subprocess.run([cxx, *FLAGS, *extra, str(SRC), "-o", str(OUT)], capture_output=True, text=True)
            if r.returncode == 0:
                return OUT
            err = r.stderr
    raise RuntimeError("oracle build failed:\n" + err)


if __name__ == "__main__":
    print(build("--force" in sys.argv))
