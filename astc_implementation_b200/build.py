"""Builds astc_implementation_b200/libastcb200.so (the C-ABI library) with nvcc
for sm_100a.  The encoder kernels are compiled with -fmad=false and IEEE
division / square root: the search's float semantics forbid fused multiply-add
contraction, so every product and sum rounds exactly as the CPU oracle's.

    python -m astc_implementation_b200.build [--verbose-ptxas]
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libastcb200.so")

SOURCES = ["tables.cpp", "decoder.cpp", "kernels_search.cu", "kernels_refine.cu", "capi.cu", "noalloc.cu", "decoder_gpu.cu", "batch.cu", "mlp.cu", "mlp_train.cu", "pipeline.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-I", CSRC, "-I", os.path.join(REPO, "include")]
CU_FLAGS = ARCH + ["-lineinfo", "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
                   "-Xcompiler", "-fPIC,-ffp-contract=off", "--expt-relaxed-constexpr"]
CPP_FLAGS = ["-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall"]


def _compile(src, verbose_ptxas):
    out = os.path.join(BUILD, src + ".o")
    path = os.path.join(CSRC, src)
    if src.endswith(".cu"):
        cmd = [NVCC] + COMMON + CU_FLAGS + (["-Xptxas", "-v"] if verbose_ptxas else []) + ["-c", path, "-o", out]
    else:
        cmd = ["g++"] + COMMON + CPP_FLAGS + ["-I", "/usr/local/cuda/include", "-c", path, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return src, out, r


def build(verbose_ptxas=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(REPO, "include", "astcb200.h")]
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(d) for d in deps):
        return LIB
    with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose_ptxas), SOURCES))
    objs = []
    for src, out, r in results:
        if verbose_ptxas or r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError("compiling %s failed" % src)
        objs.append(out)
    tmp = LIB + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("linking libastcb200.so failed")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose_ptxas="--verbose-ptxas" in sys.argv, force="--force" in sys.argv))
