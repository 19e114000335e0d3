"""Build the in-tree shared libraries.

- ``shaderous_b200/libshaderous_b200.so``: the CUDA kernels (sm_100a) and the C ABI of
  ``include/shaderous_b200.h``, compiled with nvcc.
- ``oracle/liboracle.so``: the float64 CPU oracle (test infrastructure only), compiled with g++.

Run ``python -m shaderous_b200.build`` or call :func:`build_all`.
"""
from __future__ import annotations

import os
import subprocess
from concurrent.futures import ThreadPoolExecutor
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "shaderous_b200"
CSRC = PKG / "csrc"
LIB = PKG / "libshaderous_b200.so"
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "liboracle.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h")))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _newest(paths: list[Path]) -> float:
    return max(p.stat().st_mtime for p in paths)


def _compile(src: Path, obj: Path, verbose: bool, deps: list[Path] = ()) -> None:
    # the object is stamped with the newest input's time as read before compiling, so an input
    # edited while the compiler runs still makes the object stale
    stamp = _newest([src, *deps])
    cmd = [NVCC, "-O3", "-std=c++17", *ARCH, "-lineinfo", "--use_fast_math", "-Xcompiler", "-fPIC,-fopenmp,-O3",
           "-I", str(ROOT / "include"), "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cu":
        cmd[1:1] = ["-Xptxas", "-v"] if verbose else []
    else:
        cmd[1:1] = ["-x", "cu"]
    subprocess.run(cmd, check=True)
    os.utime(obj, (stamp, stamp))


def build_library(force: bool = False, verbose: bool = False) -> Path:
    """Compile the objects that are older than their source or any header (all of them in
    parallel, one nvcc per core) and link the library when any object changed."""
    srcs = _sources()
    deps = _headers() + [Path(__file__)]
    obj_dir = PKG / "_build"
    obj_dir.mkdir(exist_ok=True)
    objs = [obj_dir / (src.stem + ".o") for src in srcs]
    todo = [(s, o) for s, o in zip(srcs, objs) if force or _stale(o, [s] + deps)]
    if todo:
        with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as pool:
            for f in [pool.submit(_compile, s, o, verbose, deps) for s, o in todo]:
                f.result()
    if todo or force or _stale(LIB, objs):
        tmp = LIB.with_suffix(".so.tmp")
        subprocess.run([NVCC, "-shared", *ARCH, "-o", str(tmp), *map(str, objs), "-Xcompiler", "-fopenmp", "-lgomp"],
                       check=True)
        os.replace(tmp, LIB)
    return LIB


def build_oracle(force: bool = False) -> Path:
    srcs = [ORACLE_DIR / "ref_hydro.cpp", ORACLE_DIR / "amr_ref.cpp"]
    if not force and not _stale(ORACLE_LIB, srcs + [ORACLE_DIR / "hydro_ref.h", Path(__file__)]):
        return ORACLE_LIB
    tmp = ORACLE_LIB.with_suffix(".so.tmp")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-o", str(tmp), *map(str, srcs)],
                   check=True)
    os.replace(tmp, ORACLE_LIB)
    return ORACLE_LIB


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_oracle(force)
    build_library(force, verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose="-v" in sys.argv)
