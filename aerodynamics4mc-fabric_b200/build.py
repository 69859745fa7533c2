"""Build the CUDA library libaero_lbm_b200.so in-tree (sm_100a only).

Every .cu/.cpp under csrc/ is compiled by nvcc for sm_100a, objects go to
_build/ beside this file, and the shared library lands next to this file so
that it travels with the source tree. Rebuilds only what changed.

Usage: python build.py [--force] [--jobs N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libaero_lbm_b200.so"
INCLUDE = HERE.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden", f"-I{INCLUDE}"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libaero_lbm_b200.so")


def sources() -> list[Path]:
    return sorted(p for p in CSRC.iterdir() if p.suffix in (".cu", ".cpp"))


def headers() -> list[Path]:
    return sorted(p for p in CSRC.iterdir() if p.suffix in (".cuh", ".h")) + sorted(INCLUDE.glob("*.h"))


def per_file_flags(src: Path) -> list[str]:
    # Reference-order kernels must not contract multiply-adds (bit parity).
    return ["--fmad=false"] if src.stem.endswith("_exact") else []


def compile_one(src: Path, force: bool, extra: list[str]) -> Path:
    obj = BUILD / (src.name + ".o")
    extra = [*extra, *per_file_flags(src)]
    newest_dep = max([src.stat().st_mtime] + [h.stat().st_mtime for h in headers()])
    if not force and obj.exists() and obj.stat().st_mtime >= newest_dep:
        return obj
    cmd = [nvcc(), *ARCH, *COMMON, *extra, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd = [nvcc(), "-x", "cu", *ARCH, *COMMON, *extra, "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stdout}\n{res.stderr}")
    return obj


def build(force: bool = False, jobs: int | None = None, extra: list[str] | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    extra = extra or []
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda s: compile_one(s, force, extra), srcs))
    if force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", *map(str, objs), "-o", str(tmp)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
        os.replace(tmp, LIB)
    return LIB


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--ptxas-verbose", action="store_true", help="print register/spill usage")
    args = ap.parse_args()
    extra = ["-Xptxas", "-v"] if args.ptxas_verbose else []
    lib = build(force=args.force or args.ptxas_verbose, jobs=args.jobs, extra=extra)
    print(lib)
    return 0


if __name__ == "__main__":
    sys.exit(main())
