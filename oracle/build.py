"""Build the CPU oracle (liboracle.so) and, when the reference sources are
present, the reference's own code under oracle/_ref/ (see build_ref.py).

The oracle is compiled with -ffp-contract=off so that its single-precision
arithmetic is the IEEE arithmetic the engine's exact-math kernel performs.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
LIB64 = HERE / "liboracle64.so"  # the same loop in FP64 (precision reference)
SRC = HERE / "mc3d_oracle.c"
DEPS = [SRC, HERE.parent / "ymc3d_b200" / "csrc" / "mc3d_exactmath.h"]


def build() -> Path:
    for lib, extra in ((LIB, []), (LIB64, ["-DORC_F64"])):
        if not lib.exists() or any(d.stat().st_mtime > lib.stat().st_mtime for d in DEPS):
            cmd = ["gcc", "-O2", "-std=gnu11", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
                   "-fPIC", "-shared", "-Wall", "-Wno-unused-function", *extra, "-o", str(lib),
                   str(SRC), "-lm"]
            res = subprocess.run(cmd, capture_output=True, text=True)
            if res.returncode != 0 or "warning" in res.stderr:
                sys.stderr.write(res.stdout + res.stderr)
            if res.returncode != 0:
                raise RuntimeError("oracle build failed")
    return LIB


if __name__ == "__main__":
    print(build())
