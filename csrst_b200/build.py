"""Builds libcsrst_gpu.so in this directory from csrc/*.cu for sm_100a.

The FP64 kernels are compiled with --fmad=false: every multiply and add is
rounded separately, as in the reference's x86-64 build, which is what makes
the positions and fields bit-identical to the CPU restatement.  The FP32-mode
particle kernels (particles32.cu) are checked against the FP64 path to a
tolerance and are compiled with FMA contraction on.
"""
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = ["api.cu", "geometry.cu", "particles.cu", "particles32.cu", "fields.cu", "diag.cu", "poisson.cu",
       "gemm.cu", "nn.cu", "noalloc.cu"]
FMA_ON = {"particles32.cu", "gemm.cu", "nn.cu"}
OUT = HERE / "libcsrst_gpu.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "--fmad=false", "-lineinfo", "-Xcompiler", "-fPIC",
         "-Xptxas", "-O3"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (Path(c).exists() or c == "nvcc"):
            return c
    raise RuntimeError("nvcc not found")


def build(force=False, verbose=False):
    srcs = [HERE / "csrc" / s for s in SRC]
    deps = (srcs + list((HERE / "csrc").glob("*.cuh")) + list((HERE / "csrc").glob("*.h")) +
            [HERE.parent / "include" / "csrst.h"])
    if not force and OUT.exists() and all(OUT.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return OUT
    objdir = HERE / "_build"
    objdir.mkdir(exist_ok=True)
    objs = []
    procs = []
    for s in srcs:
        o = objdir / (s.stem + ".o")
        flags = [f for f in FLAGS if f != "--fmad=false"] if s.name in FMA_ON else FLAGS
        cmd = [nvcc(), *ARCH, *flags, "-c", str(s), "-o", str(o)]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        procs.append((subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT), s))
        objs.append(o)
    for p, s in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stdout.write(out.decode())
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed on {s.name}")
    tmp = OUT.with_suffix(".so.tmp")
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs)], check=True)
    tmp.replace(OUT)
    return OUT


if __name__ == "__main__":
    build(force="-f" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
