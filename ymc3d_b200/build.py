"""Build libmc3d.so and the gpu-mc CLI in-tree for sm_100a.

Each translation unit is compiled with the flags its math needs:
  mc3d_kernel_fast.cu   -use_fast_math (the reference's numerics, CMakeLists.txt:18)
  mc3d_kernel_exact.cu  -fmad=false, IEEE division and square root (bit-reproducible)
  mc3d_seed.cu          -fmad=false
Objects go to ymc3d_b200/_build/, the library and the CLI next to this file.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
INCLUDE = HERE.parent / "include"
LIB = HERE / "libmc3d.so"
CLI = HERE / "gpu-mc"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(CSRC),
               "-I", str(INCLUDE)] + ARCH

UNITS = {
    "mc3d_kernel_fast.cu": ["-use_fast_math", "-Xptxas", "-v"],
    "mc3d_kernel_exact.cu": ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
                             "-Xptxas", "-v"],
    "mc3d_kernel_f64.cu": ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
                           "-Xptxas", "-v"],
    "mc3d_seed.cu": ["-fmad=false"],
    "mc3d_safedist.cu": [],
    "mc3d_api.cu": ["-fmad=false", "-Xcompiler", "-ffp-contract=off"],
    "mc3d_noalloc.cu": ["-use_fast_math", "-Xcompiler", "-ffp-contract=off", "-Xptxas", "-v"],
}
CXX_UNITS = ["mc3d_safeprimes.cpp", "mc3d_io.cpp"]
CXX_FLAGS = ["-O2", "-fPIC", "-std=c++17", "-pthread", "-ffp-contract=off", "-I", str(CSRC),
             "-I", str(INCLUDE)]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _headers() -> list[Path]:
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def _run(cmd: list[str], log: Path) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    log.write_text(" ".join(cmd) + "\n" + res.stdout + res.stderr)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd)}")


def build(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    hdrs = _headers()
    jobs = []
    objs = []
    for src, flags in UNITS.items():
        obj = BUILD / (src + ".o")
        objs.append(obj)
        if _stale(obj, [CSRC / src] + hdrs + [Path(__file__)]):
            jobs.append(([nvcc(), "-c", str(CSRC / src), "-o", str(obj)] + NVCC_COMMON + flags,
                         BUILD / (src + ".log")))
    for src in CXX_UNITS:
        obj = BUILD / (src + ".o")
        objs.append(obj)
        if _stale(obj, [CSRC / src] + hdrs + [Path(__file__)]):
            jobs.append((["g++", "-c", str(CSRC / src), "-o", str(obj)] + CXX_FLAGS,
                         BUILD / (src + ".log")))
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        list(ex.map(lambda j: _run(*j), jobs))
    if jobs or _stale(LIB, objs):
        _run([nvcc(), "-shared", "-o", str(LIB)] + [str(o) for o in objs] + ARCH +
             ["-Xcompiler", "-pthread"], BUILD / "link.log")
    cli_src = CSRC / "gpu_mc.cpp"
    if _stale(CLI, [cli_src, LIB] + hdrs):
        _run(["g++", "-O2", "-std=c++17", str(cli_src), "-o", str(CLI), "-I", str(INCLUDE),
              "-L", str(HERE), "-lmc3d", "-Wl,-rpath,$ORIGIN"], BUILD / "cli.log")
    if verbose:
        for log in sorted(BUILD.glob("mc3d_kernel_*.log")):
            print(log.read_text())
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
