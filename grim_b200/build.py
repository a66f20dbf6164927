"""Builds libgrim_b200.so in place (nvcc, sm_100a).

kernels_exact.cu, faces_exact.cu and geometry.cu are compiled with
--fmad=false so the FP64 parity path keeps the reference's operation order
without FMA contraction; kernels_fast.cu and faces_fast.cu (tangent /
mixed-precision Newton) keep contraction on.
Objects are rebuilt only when a source or header is newer.
"""
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgrim_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
EXACT = ["--fmad=false"]
UNITS = {
    "kernels_exact.cu": EXACT,
    "kernels_fast.cu": [],
    "faces_exact.cu": EXACT,
    "faces_fast.cu": [],
    "geometry.cu": EXACT,
    "runtime.cu": [],
    "peaks.cu": [],
    "noalloc.cu": EXACT,
    "adjoint.cu": [],
    "io.cu": [],
}


def _newest_header():
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    hs.append(os.path.join(HERE, "..", "include", "grim_b200.h"))
    return max(os.path.getmtime(h) for h in hs if os.path.exists(h))


def _compile(src, flags, verbose):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _newest_header()):
        return obj
    cmd = [NVCC] + COMMON + flags + ["-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, r.stdout, r.stderr))
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def build(verbose=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    srcs = [(os.path.join(CSRC, n), f) for n, f in UNITS.items() if os.path.exists(os.path.join(CSRC, n))]
    with cf.ThreadPoolExecutor(max_workers=jobs or len(srcs)) as ex:
        objs = list(ex.map(lambda a: _compile(a[0], a[1], verbose), srcs))
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB
    cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
