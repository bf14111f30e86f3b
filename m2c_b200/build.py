"""Build the sm_100a CUDA library m2c_b200/libm2c_gpu.so in-tree with nvcc.

Translation units and their floating-point contract:
  kernels_fp64.cu, context.cu, multiphase.cu, riemann.cu, levelset.cu, batch.cu
      -fmad=false : FP64 path, no FMA contraction (rounds like the reference's
                    x86-64 build)
  kernels_mixed.cu, mlp.cu
      -fmad=true  : mixed path / learned warm start (kernels_mixed.cu also
                    --use_fast_math: FP32 division/sqrt approximate, FTZ)
The library exports the C ABI of include/m2c_gpu.h (plain pointers and sizes).
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libm2c_gpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
                 "-I" + os.path.join(HERE, "..", "include")]
# --use_fast_math changes only single-precision arithmetic (approximate
# division/sqrt, flush to zero): the FP32 flux half of the mixed path.
FAST_FP32 = {"kernels_mixed.cu"}
NO_FMA = {"kernels_fp64.cu", "context.cu", "viscous.cu", "walls.cu", "multiphase.cu", "riemann.cu", "levelset.cu", "batch.cu",
          "noalloc.cu"}


def nvcc():
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def build(verbose=False, jobs=8):
    os.makedirs(OUT, exist_ok=True)
    cc = nvcc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "m2c_gpu.h"))
    hdr_mtime = max(os.path.getmtime(h) for h in headers)
    procs, objs = [], []
    for f in sources():
        src = os.path.join(CSRC, f)
        obj = os.path.join(OUT, f[:-3] + ".o")
        objs.append(obj)
        if os.path.exists(obj) and os.path.getmtime(obj) > max(os.path.getmtime(src), hdr_mtime):
            continue
        flags = COMMON + (["-fmad=false"] if f in NO_FMA else ["-fmad=true"])
        if f in FAST_FP32:
            flags = flags + ["--use_fast_math"]
        cmd = [cc] + flags + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((f, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        while len([p for _, p in procs if p.poll() is None]) >= jobs:
            procs[0][1].wait()
    failed = []
    for f, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((f, out.decode()))
    if failed:
        for f, log in failed:
            sys.stderr.write(f"---- {f}\n{log}\n")
        raise RuntimeError("nvcc failed: " + ", ".join(f for f, _ in failed))
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [cc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
