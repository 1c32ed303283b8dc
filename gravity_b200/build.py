"""Builds the sm_100a P3M library in-tree: gravity_b200/lib/libgravity_p3m.so.

Each .cu file under gravity_b200/csrc is compiled by nvcc for
``-gencode arch=compute_100a,code=sm_100a`` and the objects are linked into
one shared library that exports the C-ABI of include/p3m.h. The library links
the CUDA runtime statically (nvcc's default), so it needs only the driver.

The stage sources under csrc/step/ are compiled as one translation unit
(p3m_step.cu), which also holds the batched form's persistent kernel. The code
there that derives integers or positions from floating point (keys, deposit
weights, drift) uses explicit round-to-nearest intrinsics, so no multiply-add
is contracted and it rounds exactly like the CPU oracle; the aim previews
(p3m_trajectory.cu) are compiled with ``--fmad=false`` for the same reason.

Usage: ``python -m gravity_b200.build [--force] [--verbose]``.
"""

from __future__ import annotations

import argparse
from concurrent.futures import ThreadPoolExecutor
import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
REPO = PACKAGE.parent
CSRC = PACKAGE / "csrc"
INCLUDE = REPO / "include"
OBJ_DIR = PACKAGE / "_build"
LIB_DIR = PACKAGE / "lib"
LIB_PATH = LIB_DIR / "libgravity_p3m.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "--expt-relaxed-constexpr"]
# Sources whose arithmetic must not contract a*b+c into one rounding.
NO_FMA = {"p3m_trajectory.cu"}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build gravity_b200")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def headers() -> list[Path]:
    """Everything a translation unit may include: the internal headers, the
    stage sources under csrc/step/ (compiled through p3m_step.cu) and the
    public header."""
    return (sorted(CSRC.glob("*.cuh")) + sorted((CSRC / "step").glob("*.cu")) +
            sorted((CSRC / "step").glob("*.cuh")) + sorted(INCLUDE.glob("*.h")))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def needs_build() -> bool:
    deps = sources() + headers() + [Path(__file__)]
    return _stale(LIB_PATH, deps)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> Path:
    """Compile every CUDA source for sm_100a and link the shared library."""
    OBJ_DIR.mkdir(parents=True, exist_ok=True)
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    cc = nvcc()
    hdrs = headers() + [Path(__file__)]
    objs, jobs = [], []
    for src in sources():
        obj = OBJ_DIR / (src.stem + ".o")
        objs.append(obj)
        if not force and not _stale(obj, [src] + hdrs):
            continue
        cmd = [cc, *ARCH, *COMMON, "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(src), "-o", str(obj)]
        if src.name in NO_FMA:
            cmd.append("--fmad=false")
        if ptxas_verbose:
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), flush=True)
        jobs.append((src, cmd))
    # Translation units compile independently: run them side by side.
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        results = list(pool.map(
            lambda job: (job[0], subprocess.run(job[1], capture_output=True, text=True)), jobs))
    for src, res in results:
        if verbose or ptxas_verbose:
            sys.stdout.write(res.stdout)
            sys.stderr.write(res.stderr)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stdout}\n{res.stderr}")
    if force or _stale(LIB_PATH, objs):
        tmp = LIB_PATH.with_suffix(".so.tmp")
        cmd = [cc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs)]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc link failed:\n{res.stdout}\n{res.stderr}")
        os.replace(tmp, LIB_PATH)
    return LIB_PATH


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true", help="print registers/spills per kernel")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, ptxas_verbose=a.ptxas_verbose))


if __name__ == "__main__":
    main()
