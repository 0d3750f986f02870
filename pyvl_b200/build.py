"""Build libpvl_b200.so (the C-ABI library) in-tree with nvcc for sm_100a.

    python -m pyvl_b200.build [--verbose]

The library is compiled from pyvl_b200/csrc/*.cu and *.cpp with
``-gencode arch=compute_100a,code=sm_100a`` and lands next to this file, where the
Python layer loads it.  nvcc cross-compiles without a GPU.  Beside it, libpvl_probe.so
(pyvl_b200/probe: an FMA-throughput probe and test hooks) is built for benchmarks and tests;
the product never loads it.  Extra nvcc flags (e.g. a tuning define such as
``-DPVL_UPD_WARPS=4``) can be passed in the environment variable PVL_NVCC_FLAGS.
"""

from __future__ import annotations

import argparse
import os
import shlex
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "libpvl_b200.so"
PROBE_SRC = HERE / "probe"
PROBE_LIB = HERE / "libpvl_probe.so"  # measurement and test probes, not part of the product ABI
BUILD_DIR = HERE.parent / "_build"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + [HERE.parent / "include" / "pvl_b200.h"]


def needs_build(lib: Path = LIB, srcs: list[Path] | None = None) -> bool:
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    deps = (sources() if srcs is None else srcs) + _headers() + sorted(PROBE_SRC.glob("*.h"))
    return any(p.stat().st_mtime > t for p in deps)


def build(verbose: bool = False, force: bool = False) -> Path:
    """Build libpvl_b200.so and the probe library beside it; returns the product library."""
    _build_lib(LIB, sources(), "", verbose, force)
    # the probes reach internal launchers of the product library: link it, found beside them
    _build_lib(PROBE_LIB, sorted(PROBE_SRC.glob("*.cu")), "probe_", verbose, force,
               ["-L", str(HERE), "-lpvl_b200", "-Xlinker", "-rpath=$ORIGIN"], after=LIB)
    return LIB


def _build_lib(lib: Path, srcs: list[Path], prefix: str, verbose: bool, force: bool, link: list[str] | None = None,
               after: Path | None = None) -> Path:
    stale = after is not None and lib.exists() and after.stat().st_mtime > lib.stat().st_mtime
    if not force and not stale and not needs_build(lib, srcs):
        return lib
    BUILD_DIR.mkdir(exist_ok=True)
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(HERE.parent / "include"), "-I", str(CSRC),
              "-I", str(PROBE_SRC), *shlex.split(os.environ.get("PVL_NVCC_FLAGS", ""))]

    def compile_one(src: Path) -> str:
        obj = BUILD_DIR / (prefix + src.name + ".o")
        cmd = [nvcc(), *common, *ARCH, "-lineinfo", "-c", str(src), "-o", str(obj)]
        if verbose and src.suffix == ".cu":
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}")
        return str(obj)

    with ThreadPoolExecutor(max_workers=max(1, min(len(srcs), os.cpu_count() or 1))) as pool:
        objs = list(pool.map(compile_one, srcs))
    tmp = lib.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, *(link or []), "-lcudart_static", "-lrt", "-ldl",
           "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(tmp, lib)
    return lib


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(verbose=a.verbose, force=a.force))


if __name__ == "__main__":
    main()
