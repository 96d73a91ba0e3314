"""Compile the reference's own code into oracle/_ref/ (test infrastructure).

The sources are compiled where they lie under the reference checkout, never
copied.  Products (all git-ignored, they travel with the working tree):
  _ref/libref_rng.so        init_RNG + a rand_MWC_co test kernel
                            (gpumcml_rng/gpumcml_rng.cu, via ref/rng_harness.cu)
  _ref/libref_io.so         the file readers and save_diff_refl (src/mc3d_io.cu,
                            via ref/io_harness.cu)
  _ref/gpu-mc-ref           run_3dmc_gpu and its kernels (src/mc3d_gpu.cu,
                            src/mc3d_photons.cu, src/mc3d_io.cu) driven by
                            ref/ref_main.cu; mc3d_gpu.cu gets ref/texture_shim.h
                            force-included because CUDA 12 removed texture references
  _ref/gpu-mc-bridge        the reference's own command line (src/mc3d_main.cu,
                            src/mc3d_io.cu) with run_3dmc_gpu forwarded to this
                            repository's libmc3d.so by ref/mc3d_b200_bridge.cu:
                            the drop-in as a maintainer would build it
  _ref/safeprimes_base32.txt  the safe-prime table the reference reads from its
                            working directory (not distributed with the reference)
Flags follow CMakeLists.txt:18 (-use_fast_math, -Xptxas -v) with sm_100a for
sm_30 and OpenMP for the host tally.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
# the reference checkout: $YMC3D_REFERENCE, else a directory named `reference`
# beside this repository
REF = Path(os.environ.get("YMC3D_REFERENCE", HERE.parent.parent / "reference"))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
TABLE_LINES = 1 + 230400  # n_rng = 600 blocks * 384 threads (src/mc3d_gpu.cu:434)


def _nvcc() -> str:
    return os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _run(cmd):
    res = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    (OUT / "build.log").open("a").write(" ".join(map(str, cmd)) + "\n" + res.stdout + res.stderr)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("reference build step failed: " + " ".join(map(str, cmd)))


def write_table(path: Path, table) -> None:
    with open(path, "w") as f:
        for a in table:
            p = (int(a) << 32) - 1
            f.write(f"{int(a)} {p >> 32} {p & 0xffffffff}\n")


def build(table=None) -> bool:
    """Returns False when the reference checkout is absent (prebuilt files are used)."""
    if not (REF / "src" / "mc3d_gpu.cu").exists():
        return False
    OUT.mkdir(exist_ok=True)
    src, rng = REF / "src", REF / "gpumcml_rng"
    inc = ["-I", src, "-I", rng]
    rng_so = OUT / "libref_rng.so"
    if not rng_so.exists() or rng_so.stat().st_mtime < (HERE / "ref" / "rng_harness.cu").stat().st_mtime:
        _run([_nvcc(), "-shared", "-Xcompiler", "-fPIC", "-O2", *ARCH, *inc,
              HERE / "ref" / "rng_harness.cu", "-o", rng_so])
    io_so = OUT / "libref_io.so"
    if not io_so.exists() or io_so.stat().st_mtime < (HERE / "ref" / "io_harness.cu").stat().st_mtime:
        _run([_nvcc(), "-shared", "-Xcompiler", "-fPIC", "-O2", *ARCH, *inc,
              src / "mc3d_io.cu", HERE / "ref" / "io_harness.cu", "-o", io_so])
    exe = OUT / "gpu-mc-ref"
    deps = [HERE / "ref" / "ref_main.cu", HERE / "ref" / "texture_shim.h"]
    if not exe.exists() or any(d.stat().st_mtime > exe.stat().st_mtime for d in deps):
        flags = ["-O3", "-use_fast_math", *ARCH, "-Xcompiler", "-fopenmp", *inc]
        objs = []
        for name, extra in (("mc3d_gpu.cu", ["-include", HERE / "ref" / "texture_shim.h",
                                             "-Dtime=mc3d_ref_seed_clock"]),
                            ("mc3d_photons.cu", []), ("mc3d_io.cu", [])):
            obj = OUT / (name + ".o")
            _run([_nvcc(), "-c", src / name, "-o", obj, *flags, *extra])
            objs.append(obj)
        obj = OUT / "ref_main.o"
        _run([_nvcc(), "-c", HERE / "ref" / "ref_main.cu", "-o", obj, *flags])
        objs.append(obj)
        _run([_nvcc(), *ARCH, "-Xcompiler", "-fopenmp", *objs, "-o", exe, "-lgomp"])
    lib = HERE.parent / "ymc3d_b200" / "libmc3d.so"
    bridge = OUT / "gpu-mc-bridge"
    deps = [HERE / "ref" / "mc3d_b200_bridge.cu", lib, HERE.parent / "include" / "mc3d.h"]
    if lib.exists() and (not bridge.exists() or
                         any(d.stat().st_mtime > bridge.stat().st_mtime for d in deps)):
        flags = ["-O3", *ARCH, *inc, "-I", HERE.parent / "include"]
        objs = []
        for path in (src / "mc3d_main.cu", src / "mc3d_io.cu", HERE / "ref" / "mc3d_b200_bridge.cu"):
            obj = OUT / ("bridge_" + path.name + ".o")
            _run([_nvcc(), "-c", path, "-o", obj, *flags])
            objs.append(obj)
        _run([_nvcc(), *ARCH, *objs, "-o", bridge, "-L", lib.parent, "-lmc3d",
              "-Xlinker", "-rpath=$ORIGIN/../../ymc3d_b200"])
    tab = OUT / "safeprimes_base32.txt"
    if not tab.exists():
        if table is None:
            sys.path.insert(0, str(HERE.parent))
            import ymc3d_b200
            table = ymc3d_b200.default_table()[:TABLE_LINES]
        write_table(tab, table[:TABLE_LINES])
    return True


if __name__ == "__main__":
    print(build())
