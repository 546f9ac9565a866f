"""Build libdvc_b200.so in-tree for sm_100a.

    python -m dvc_b200.build            # compile every csrc/*.cu, *.cpp and link,
                                        # then the dvcdec executable (cli/dvcdec.cpp)

Every CUDA translation unit is compiled with -fmad=false (no contraction of
a*b+c into fused multiply-adds, matching the reference's x86 SSE2 arithmetic)
and IEEE division/square root (no fast-math); host code with
-ffp-contract=off for the same reason.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(LIBDIR, "libdvc_b200.so")
CLI_SRC = os.path.join(HERE, "cli", "dvcdec.cpp")
CLI = os.path.join(LIBDIR, "dvcdec")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
              "-Xcompiler", "-fPIC,-O2,-ffp-contract=off", "-Xptxas", "-O3", "-I", CSRC,
              "-I", os.path.join(ROOT, "include")]


def nvcc():
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _compile(src, verbose=False, extra=()):
    obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
    deps = [src] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    deps.append(os.path.join(ROOT, "include", "dvc_b200.h"))
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps if os.path.exists(d)):
        return obj
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + list(extra) + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [nvcc(), "-x", "cu"] + ARCH + NVCC_FLAGS + list(extra) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    if verbose and r.stderr.strip():
        print(r.stderr)
    return obj


def build(verbose=False, ptxas_info=False):
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose or ptxas_info, extra), sources()))
    if not (os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs)):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    build_cli()
    return LIB


def build_cli():
    """The DvcDec-compatible executable, linked against the library beside it."""
    hdr = os.path.join(ROOT, "include", "dvc_b200.h")
    if os.path.exists(CLI) and os.path.getmtime(CLI) >= max(os.path.getmtime(p) for p in (CLI_SRC, hdr, LIB)):
        return CLI
    cmd = [shutil.which("g++") or "g++", "-O2", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"), CLI_SRC,
           "-L", LIBDIR, "-ldvc_b200", "-Wl,-rpath,$ORIGIN", "-o", CLI]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("dvcdec build failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return CLI


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv))
