"""Builds the sm_100a shared library fvhoe_b200/_lib/libfvh.so with nvcc.

Usage: python -m fvhoe_b200.build [--force] [-j N]

Objects go to fvhoe_b200/_build/ and the library to fvhoe_b200/_lib/, both in
the source tree, so a copied checkout carries the built library with it.
The FP64 stage runner is compiled with -fmad=false: every product and sum
rounds on its own, in the same order as the NumPy reference.
"""

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libfvh.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-I", os.path.join(ROOT, "include"), "-I", CSRC]

# translation unit -> extra flags
UNITS = {
    "fvh_api.cu": [],
    "fvh_stage_f64.cu": ["-fmad=false"],
    # the FP32 path is never compared bit for bit: fast division, square root and FTZ
    "fvh_stage_f32.cu": ["-fmad=true", "--use_fast_math"],
    "fvh_noalloc.cu": ["-fmad=false"],
    # learned troubled-cell predictor (tensor cores, FP32 epilogues)
    "fvh_mlp.cu": [],
    # batched ensemble: host API and one launch unit per precision
    "fvh_ensemble.cu": [],
    "fvh_ens_f64.cu": ["-fmad=false"],
    "fvh_ens_f32.cu": ["-fmad=true", "--use_fast_math"],
}


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; set NVCC or put the CUDA toolkit on PATH")


def _sources_mtime():
    newest = 0.0
    for root in (CSRC, os.path.join(ROOT, "include")):
        for name in os.listdir(root):
            newest = max(newest, os.path.getmtime(os.path.join(root, name)))
    return max(newest, os.path.getmtime(__file__))


def _compile(unit, flags, verbose):
    src = os.path.join(CSRC, unit)
    obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
    cmd = [nvcc(), *ARCH, *COMMON, *flags, "-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {unit}:\n{res.stderr}")
    return obj, res.stderr


def build(force: bool = False, jobs: int = 0, verbose: bool = False) -> str:
    """Compiles every unit for sm_100a and links libfvh.so; returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _sources_mtime():
        return LIB
    if jobs <= 0:
        jobs = min(len(UNITS), os.cpu_count() or 1)
    with ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        results = list(ex.map(lambda kv: _compile(kv[0], kv[1], verbose), UNITS.items()))
    if verbose:
        for _, log in results:
            sys.stderr.write(log)
    objs = [o for o, _ in results]
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", *objs, "-o", tmp]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stderr}")
    os.replace(tmp, LIB)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=0, help="parallel nvcc jobs (0: one per unit, at most the CPU count)")
    ap.add_argument("-v", action="store_true", help="print ptxas resource usage")
    args = ap.parse_args()
    print(build(force=args.force, jobs=args.j, verbose=args.v))


if __name__ == "__main__":
    main()
