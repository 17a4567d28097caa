"""Builds libtrex_b200.so (all CUDA sources in trex_b200/csrc) for sm_100a.

    python -m trex_b200.build            # incremental
    python -m trex_b200.build --force    # rebuild everything

Output: <repo>/build/libtrex_b200.so plus symlinks with the reference's
library names (libprefix_compose.so, libmonoid_batch.so, libmonoid_scan.so,
libnfa_tc_evolution.so) so the reference's own ctypes bridges load this
library unchanged.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
OUT_DIR = REPO / "build"
OBJ_DIR = OUT_DIR / "obj"
LIB = OUT_DIR / "libtrex_b200.so"
REFERENCE_NAMES = ("libprefix_compose.so", "libmonoid_batch.so", "libmonoid_scan.so",
                   "libnfa_tc_evolution.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
              "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build trex_b200")
    return cand


def _sources():
    return sorted(CSRC.glob("*.cu"))


def _headers():
    return sorted(CSRC.glob("*.cuh")) + sorted((REPO / "include").glob("*.h"))


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, force: bool) -> Path:
    obj = OBJ_DIR / (src.stem + ".o")
    if force or _stale(obj, [src] + _headers()):
        cmd = [_nvcc(), *ARCH, *NVCC_FLAGS, "-I", str(REPO / "include"), "-c", str(src),
               "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
        warn = [ln for ln in (r.stdout + r.stderr).splitlines() if "spill" in ln.lower()
                and " 0 bytes spill" not in ln]
        if warn:
            print(f"[trex_b200.build] {src.name}: " + " | ".join(warn), file=sys.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJ_DIR.mkdir(parents=True, exist_ok=True)
    srcs = _sources()
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
    if force or _stale(LIB, objs):
        cmd = [_nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcuda"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    for name in REFERENCE_NAMES:
        link = OUT_DIR / name
        if link.is_symlink() or link.exists():
            if link.is_symlink() and os.readlink(link) == LIB.name:
                continue
            link.unlink()
        link.symlink_to(LIB.name)
    if verbose:
        print(f"[trex_b200.build] {LIB}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
