"""Build recipe for the product library (libcep_b200.so, sm_100a only).

    python -m 2ddrugsimulation_b200.build      (or import and call build())

Compiles every CUDA source under csrc/ with nvcc for sm_100a into
2ddrugsimulation_b200/lib/libcep_b200.so (in-tree, so it ships with the
repository snapshot). The FP32 half of the mixed-precision kernels uses
approximate division/sqrt and flush-to-zero; FP64 arithmetic is unaffected
by those flags.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "lib"
LIB = LIB_DIR / "libcep_b200.so"
BUILD_DIR = PKG / "_build"
PROBE_LIB = LIB_DIR / "libcep_probe.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--prec-div=false",
              "--prec-sqrt=false", "--ftz=true", "-Xptxas", "-v", "-I", str(PKG.parent / "include")]


# Per-file additions: the grid assembly is compiled without FMA contraction
# so every matrix entry is the same IEEE expression as a scalar assembly.
FILE_FLAGS = {"fem_assembly.cu": ["-fmad=false"]}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    deps = [src] + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list((PKG.parent / "include").glob("*.h"))
    return any(d.stat().st_mtime > obj.stat().st_mtime for d in deps)


def build(verbose: bool = False, force: bool = False) -> Path:
    BUILD_DIR.mkdir(exist_ok=True)
    LIB_DIR.mkdir(exist_ok=True)
    objs = []
    logs = []
    for src in sources():
        obj = BUILD_DIR / (src.stem + ".o")
        objs.append(obj)
        if not force and not _stale(obj, src):
            continue
        if src.suffix == ".cu":
            cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *FILE_FLAGS.get(src.name, []), "-c", str(src), "-o", str(obj)]
        else:
            cmd = [nvcc(), "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(PKG.parent / "include"),
                   "-c", str(src), "-o", str(obj)]
        out = subprocess.run(cmd, capture_output=True, text=True)
        logs.append(out.stdout + out.stderr)
        if out.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src.name}:\n{out.stdout}\n{out.stderr}")
        (BUILD_DIR / (src.stem + ".ptxas.txt")).write_text(out.stderr)
    if not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs) or force:
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        out = subprocess.run(cmd, capture_output=True, text=True)
        if out.returncode != 0:
            raise RuntimeError(f"link failed:\n{out.stdout}\n{out.stderr}")
    # measurement probes (bench.py roofline denominators), a separate library
    probe_src = PKG / "probes" / "peaks.cu"
    if probe_src.exists() and (force or not PROBE_LIB.exists() or probe_src.stat().st_mtime > PROBE_LIB.stat().st_mtime):
        cmd = [nvcc(), *ARCH, "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", str(probe_src), "-o",
               str(PROBE_LIB)]
        out = subprocess.run(cmd, capture_output=True, text=True)
        if out.returncode != 0:
            raise RuntimeError(f"probe build failed:\n{out.stdout}\n{out.stderr}")
    if verbose:
        for l in logs:
            sys.stderr.write(l)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
