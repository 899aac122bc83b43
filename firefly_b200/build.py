"""Build libfirefly_b200.so in-tree with nvcc for sm_100a.

Usage: python -m firefly_b200.build [--verbose] [--ptxas-info]

Every .cu file under firefly_b200/csrc is compiled and linked into
firefly_b200/lib/libfirefly_b200.so (static CUDA runtime, so the library does
not depend on the toolkit being on the loader path).  Rebuilds only when a
source or header is newer than the library.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libfirefly_b200.so"
OBJDIR = ROOT / "_build" / "obj"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = [
    "-O3", "-std=c++17", "-lineinfo",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-I", str(ROOT / "include"), "-I", str(CSRC),
    "--expt-relaxed-constexpr",
]
# Kernels whose results are compared with the oracle bit for bit or within a
# tight tolerance are compiled without FMA contraction, so every float
# expression rounds once per operation like the reference's host build.  The
# adjoint megakernels follow: their paths then equal the wavefront's path for
# path, so the store-all variant checks the wavefront replay sample by sample.
NO_FMAD = {"ff_wavefront.cu", "ff_envmap.cu", "ff_scene.cu", "ff_adjoint.cu"}


def _sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted((ROOT / "include").glob("*.h"))


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in _sources() + _headers() + [Path(__file__)])


def build(verbose: bool = False, ptxas_info: bool = False, force: bool = False) -> Path:
    if not force and not needs_build():
        return LIB
    OBJDIR.mkdir(parents=True, exist_ok=True)
    LIBDIR.mkdir(parents=True, exist_ok=True)
    cmds, objs = [], []
    for src in _sources():
        obj = OBJDIR / (src.stem + ".o")
        flags = list(COMMON)
        flags += ["-fmad=false"] if src.name in NO_FMAD else ["-fmad=true"]
        if ptxas_info:
            flags += ["-Xptxas", "-v"]
        cmds.append([NVCC, *ARCH, *flags, "-c", str(src), "-o", str(obj)])
        objs.append(str(obj))
    # translation units compile independently: one nvcc per core
    jobs = max(1, min(len(cmds), os.cpu_count() or 1))
    with ThreadPoolExecutor(jobs) as pool:
        results = list(pool.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds))
    for cmd, res in zip(cmds, results):
        if verbose or res.returncode != 0 or ptxas_info:
            print(" ".join(cmd), flush=True)
            sys.stdout.write(res.stdout)
            sys.stderr.write(res.stderr)
    failed = [c for c, r in zip(cmds, results) if r.returncode != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(tmp), *objs, "-lpthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args(argv)
    path = build(verbose=a.verbose, ptxas_info=a.ptxas_info, force=a.force or a.ptxas_info)
    print(path)
    return 0


if __name__ == "__main__":
    sys.exit(main())
