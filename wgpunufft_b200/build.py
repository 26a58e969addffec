"""Builds libb200nufft.so in place with nvcc for sm_100a.

Every source under csrc/ is compiled to an object under _build/ (rebuilt
when it or a header is newer) and linked into wgpunufft_b200/libb200nufft.so
against cuFFT and the CUDA runtime.
"""

from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
CSRC = PACKAGE / "csrc"
BUILD = ROOT / "_build"
LIBRARY = PACKAGE / "libb200nufft.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include")]


def nvcc() -> str:
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(found).exists():
        raise RuntimeError("nvcc not found: the CUDA library cannot be built")
    return found


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted((ROOT / "include").glob("*.h"))


def _compile(source: Path, newest_header: float, verbose: bool) -> Path:
    obj = BUILD / (source.name + ".o")
    if obj.exists() and obj.stat().st_mtime >= max(source.stat().st_mtime, newest_header):
        return obj
    cmd = [nvcc(), *ARCH, *COMMON, "-c", str(source), "-o", str(obj)]
    if source.suffix == ".cu":
        cmd[1:1] = ["-Xptxas", "-v"] if verbose else []
    else:
        cmd += ["-x", "cu"]
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"nvcc failed for {source.name}:\n{result.stdout}\n{result.stderr}")
    if verbose and result.stderr:
        (BUILD / (source.name + ".ptxas.txt")).write_text(result.stderr)
    return obj


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    newest_header = max((h.stat().st_mtime for h in _headers()), default=0.0)
    workers = jobs or min(len(sources), os.cpu_count() or 4)
    with concurrent.futures.ThreadPoolExecutor(max_workers=workers) as pool:
        objects = list(pool.map(lambda s: _compile(s, newest_header, verbose), sources))
    newest_obj = max(o.stat().st_mtime for o in objects)
    if LIBRARY.exists() and LIBRARY.stat().st_mtime >= newest_obj:
        return LIBRARY
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIBRARY), *map(str, objects), "-lcufft", "-lcudart"]
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"link failed:\n{result.stdout}\n{result.stderr}")
    return LIBRARY


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
