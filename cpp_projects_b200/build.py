"""Build recipe for the native library (sm_100a only).

    python -m cpp_projects_b200.build        # incremental build
    python -m cpp_projects_b200.build --force

Compiles every ``csrc/*.cu`` with nvcc for ``sm_100a`` and every
``csrc/*.cpp`` with g++, and links ``lib/libbfs_b200.so`` in-tree (static
CUDA runtime).  Objects go to ``_build/`` (git-ignored).  Host code is built
with ``-ffp-contract=off``: the FDMT plan must not fuse multiply-adds, or its
row offsets stop matching the reference's.
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
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libbfs_b200.so"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
CXX = shutil.which("g++") or "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON_INC = [f"-I{INCLUDE}", f"-I{CSRC}", f"-I{CUDA_HOME / 'include'}"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
                     "-Xcompiler", "-fPIC,-ffp-contract=off", "-Xptxas", "-warn-spills"]
CXX_FLAGS = ["-O2", "-fPIC", "-std=c++17", "-ffp-contract=off", "-Wall"]
LINK_LIBS = ["-lcufft", "-Xlinker", f"-rpath,{CUDA_HOME / 'lib64'}"]


def _sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _headers():
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _obj(src: Path) -> Path:
    return BUILD / (src.name + ".o")


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, force: bool) -> Path:
    obj = _obj(src)
    if not force and not _stale(obj, [src] + _headers()):
        return obj
    if src.suffix == ".cu":
        cmd = [NVCC] + NVCC_FLAGS + COMMON_INC + ["-c", str(src), "-o", str(obj)]
    else:
        cmd = [CXX] + CXX_FLAGS + COMMON_INC + ["-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip():
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] + \
              [f"-L{CUDA_HOME / 'lib64'}"] + LINK_LIBS
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force))


if __name__ == "__main__":
    main()
