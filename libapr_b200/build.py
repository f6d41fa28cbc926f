"""Builds libaprb200.so (the CUDA kernels and the C ABI of include/aprb200.h)
in-tree for sm_100a with nvcc, so the library travels with the source tree.

Device code is compiled with -fmad=false and IEEE division/square root (no
--use_fast_math): the get_apr path is bit-exact with the reference's strict
IEEE CPU build only without contraction.  Host code is compiled with
-ffp-contract=off for the same reason.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libaprb200.so")
BUILD = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
                "--expt-relaxed-constexpr"]


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _compile(src, verbose):
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    cmd = ["nvcc"] + FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s%s" % (src, r.stdout, r.stderr))
    return obj, r.stderr


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "aprb200.h")]
    if not force and os.path.exists(OUT):
        newest = max(os.path.getmtime(d) for d in deps)
        if os.path.getmtime(OUT) >= newest:
            return OUT
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        res = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if verbose:
        for (_, log), s in zip(res, srcs):
            if log:
                sys.stderr.write("== %s\n%s" % (s, log))
    cmd = ["nvcc"] + ARCH + ["-shared", "-o", OUT] + [o for o, _ in res]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
