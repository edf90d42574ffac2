"""Build libwmles_cuda.so in-tree for sm_100a.

    python -m wmles_jax_b200.build [--force] [--jobs N]

Each .cu file in csrc/ is compiled separately (surface.cu and geom.cu with -fmad=false so
that the ghost-cell maps and the block geometry round exactly like the reference's NumPy
arithmetic; stage.cu with fast
single-precision division and square root for the mixed form), then linked into
wmles_jax_b200/libwmles_cuda.so against the shared CUDA runtime.
"""
import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libwmles_cuda.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-I", os.path.join(HERE, "..", "include")]
# stage.cu: single-precision division and square root without IEEE rounding and with
# denormals flushed.  These options act on FP32 operations only: the FP64 stage kernels are
# unchanged, and the mixed form's FP32 fluxes, gradients and SGS are compared with FP64
# at a tolerance far above the last-place error of these instructions.
PER_FILE = {"surface.cu": ["-fmad=false"], "geom.cu": ["-fmad=false"],
            "stage.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"]}


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found")
    return exe


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, jobs=None, verbose=False, extra=()):
    os.makedirs(OBJ, exist_ok=True)
    sources = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    headers.append(os.path.join(HERE, "..", "include", "wmles_cuda.h"))
    exe = nvcc()

    def compile_one(src):
        obj = os.path.join(OBJ, src[:-3] + ".o")
        path = os.path.join(CSRC, src)
        if not force and not _stale(obj, [path] + headers):
            return obj
        cmd = [exe, *ARCH, *COMMON, *PER_FILE.get(src, []), *extra, "-c", path, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{res.stdout}\n{res.stderr}")
        if verbose and res.stderr.strip():
            print(res.stderr, flush=True)
        return obj

    with ThreadPoolExecutor(max_workers=jobs or min(8, len(sources))) as ex:
        objs = list(ex.map(compile_one, sources))
    if force or _stale(LIB, objs):
        cmd = [exe, *ARCH, "-shared", "-cudart", "shared", "-o", LIB, *objs]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args()
    extra = ("-Xptxas", "-v") if a.ptxas_verbose else ()
    print(build(force=a.force, jobs=a.jobs, verbose=a.verbose or a.ptxas_verbose, extra=extra))
    sys.exit(0)
