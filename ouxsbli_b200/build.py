"""Build liboux.so (the sm_100a C-ABI library) in-tree with nvcc.

    python -m ouxsbli_b200.build [--force] [--jobs N]

Every translation unit is compiled for ``-gencode arch=compute_100a,code=sm_100a``.
The FP64 units are compiled with ``-fmad=false`` so that no multiply-add is
contracted: the FP64 path then evaluates the reference's arithmetic in the
reference's operation order, which the bit-exact parity tests rely on.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "liboux.so"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
          f"-I{INCLUDE}", f"-I{CSRC}"]

# (source, extra flags)
UNITS = [
    ("oux_api.cu", ["-fmad=false"]),
    ("oux_sweep_fp64_o2.cu", ["-fmad=false"]),
    ("oux_sweep_fp64_o4.cu", ["-fmad=false"]),
    ("oux_sweep_fp64_o6.cu", ["-fmad=false"]),
    ("oux_sweep_mx_o2.cu", []),
    ("oux_sweep_mx_o4.cu", []),
    ("oux_sweep_mx_o6.cu", []),
    ("oux_batch_api.cu", ["-fmad=false"]),
    ("oux_batch_fp64_o2.cu", ["-fmad=false"]),
    ("oux_batch_fp64_o4.cu", ["-fmad=false"]),
    ("oux_batch_fp64_o6.cu", ["-fmad=false"]),
    ("oux_batch_mx_o2.cu", []),
    ("oux_batch_mx_o4.cu", []),
    ("oux_batch_mx_o6.cu", []),
]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not pathlib.Path(exe).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build liboux")
    return exe


def _stale(obj: pathlib.Path, src: pathlib.Path) -> bool:
    if not obj.exists():
        return True
    deps = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h")) + [src]
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: str, flags: list[str], force: bool) -> pathlib.Path:
    s = CSRC / src
    o = BUILD / (s.stem + ".o")
    if force or _stale(o, s):
        cmd = [nvcc(), *ARCH, *COMMON, *flags, "-c", str(s), "-o", str(o)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return o


def build(force: bool = False, jobs: int | None = None) -> pathlib.Path:
    """Compile and link liboux.so; returns its path."""
    BUILD.mkdir(exist_ok=True)
    jobs = jobs or min(len(UNITS), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda u: _compile(u[0], u[1], force), UNITS))
    if force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    a = ap.parse_args(argv)
    print(build(force=a.force, jobs=a.jobs))
    return 0


if __name__ == "__main__":
    sys.exit(main())
