"""Build libacoustic_rt.so in-tree with nvcc for sm_100a.

Usage: ``python acoustic-agent_b200/build.py [--force]``.  Every translation
unit targets ``-gencode arch=compute_100a,code=sm_100a``.  The float64 tracer,
the band synthesis, the late reverberation and the direct-path queries are compiled with ``-fmad=false`` so that their
arithmetic rounds operation by operation like the reference's float64 code;
the float32 tracer keeps FMA contraction.
"""
from __future__ import annotations

import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
REPO_DIR = PACKAGE_DIR.parent
CSRC = PACKAGE_DIR / "csrc"
INCLUDE = REPO_DIR / "include"
BUILD_DIR = PACKAGE_DIR / "_build"
LIBRARY = PACKAGE_DIR / "libacoustic_rt.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          f"-I{INCLUDE}", f"-I{CSRC}", "--expt-relaxed-constexpr"]
# Units whose float64 arithmetic must not be contracted into FMAs.
NO_FMA = {"trace_f64.cu", "synth.cu", "late_reverb.cu", "direct.cu", "bvh_device.cu"}
SOURCES = ["abi.cu", "scene.cu", "trace_f32.cu", "trace_f64.cu", "synth.cu", "late_reverb.cu", "direct.cu",
           "bvh_device.cu", "refstream.cu", "service.cu", "bvh_build.cpp", "fast_bvh.cpp"]


def nvcc() -> str:
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(found).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build the backend")
    return found


def _compile(source: str, verbose: bool) -> Path:
    src = CSRC / source
    obj = BUILD_DIR / (source + ".o")
    cmd = [nvcc(), *ARCH, *COMMON, "-c", str(src), "-o", str(obj)]
    if source in NO_FMA:
        cmd.insert(-4, "-fmad=false")
    if verbose:
        cmd.insert(-4, "-Xptxas=-v")
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"nvcc failed for {source}:\n{result.stdout}\n{result.stderr}")
    if verbose and result.stderr:
        sys.stderr.write(result.stderr)
    return obj


def _stale() -> bool:
    if not LIBRARY.exists():
        return True
    built = LIBRARY.stat().st_mtime
    inputs = list(CSRC.glob("*")) + list(INCLUDE.glob("*.h")) + [Path(__file__)]
    return any(p.stat().st_mtime > built for p in inputs if p.is_file())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not _stale():
        return LIBRARY
    BUILD_DIR.mkdir(exist_ok=True)
    workers = min(len(SOURCES), os.cpu_count() or 1)
    with concurrent.futures.ThreadPoolExecutor(max_workers=workers) as pool:
        objects = list(pool.map(lambda s: _compile(s, verbose), SOURCES))
    tmp = LIBRARY.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objects), "-cudart", "static", "-lpthread"]
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"link failed:\n{result.stdout}\n{result.stderr}")
    os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("--force", action="store_true")
    parser.add_argument("--verbose", action="store_true", help="print ptxas register/spill reports")
    args = parser.parse_args()
    print(build(force=args.force, verbose=args.verbose))
