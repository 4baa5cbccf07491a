"""Build libqcb.so (sm_100a CUDA kernels + C ABI) and the gauge_hb_ncb / gauge_ecmc_ncb drivers
in-tree.

    python ecmc-qncb_b200/build.py [--force] [-j N]

Objects go to ecmc-qncb_b200/_build/, the library to ecmc-qncb_b200/lib/libqcb.so and the
drivers to ecmc-qncb_b200/bin/.  Every CUDA source is compiled for sm_100a only
(-gencode arch=compute_100a,code=sm_100a).  A target is rebuilt when a source or any
header under csrc/ or include/ is newer than it.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libqcb.so"
BIN = PKG / "bin"
DRIVER = BIN / "gauge_hb_ncb"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -prec-div=false / -prec-sqrt=false: FP32 division and square root by the hardware
# approximations (a few ulp) instead of the IEEE-rounded sequences; FP64 is unaffected.  The
# FP32 heatbath pass is 5% faster with them (the KP draw's divisions and roots); the FP32 flow
# results are unchanged.
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
              "--expt-relaxed-constexpr", "-prec-div=false", "-prec-sqrt=false", "-I", str(INCLUDE)] + ARCH
DRIVER_SOURCES = {"gauge_hb_ncb.cpp", "gauge_ecmc_ncb.cpp"}
# k_ecmc.cu spells out its fused multiply-adds; no automatic contraction, so that every
# instantiation of the event-chain kernel rounds alike.
FILE_FLAGS = {"k_ecmc.cu": ["-fmad=false"]}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libqcb")


def _headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))
                  + list(INCLUDE.glob("*.hpp")))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    """Compile every source under csrc/ and link libqcb.so and the driver; returns LIB."""
    BUILD.mkdir(parents=True, exist_ok=True)
    LIB.parent.mkdir(parents=True, exist_ok=True)
    DRIVER.parent.mkdir(parents=True, exist_ok=True)
    cc = nvcc()
    hdrs = _headers()
    srcs = sorted([p for p in CSRC.iterdir() if p.suffix in (".cu", ".cpp") and p.name not in DRIVER_SOURCES])
    objs, todo = [], []
    for s in srcs:
        o = BUILD / (s.name + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            todo.append((s, o))

    def compile_one(so):
        s, o = so
        cmd = [cc, "-c", str(s), "-o", str(o)] + NVCC_FLAGS + FILE_FLAGS.get(s.name, [])
        if s.suffix == ".cpp":
            cmd = [cc, "-x", "c++", "-c", str(s), "-o", str(o), "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                   "-Xcompiler", "-Wall", "-I", str(INCLUDE)]
        if verbose:
            print(" ".join(cmd), flush=True)
        _run(cmd)
        return o

    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
            list(ex.map(compile_one, todo))
    if force or todo or _stale(LIB, objs):
        _run([cc, "-shared", "-o", str(LIB)] + [str(o) for o in objs] + ARCH + ["-lpthread"])
    for name in sorted(DRIVER_SOURCES):
        drv_src, exe = CSRC / name, BIN / Path(name).stem
        if drv_src.exists() and (force or _stale(exe, [drv_src, LIB] + hdrs)):
            _run([cc, "-x", "c++", str(drv_src), "-o", str(exe), "-O2", "-std=c++17", "-I", str(INCLUDE),
                  "-L", str(LIB.parent), "-lqcb", "-Xlinker", "-rpath=$ORIGIN/../lib"])
    return LIB


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", "--jobs", type=int, default=None)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    lib = build(force=a.force, jobs=a.jobs, verbose=a.verbose)
    print(lib)
    return 0


if __name__ == "__main__":
    sys.exit(main())
