"""Build librigw.so (the C-ABI CUDA library) in-tree for sm_100a with nvcc."""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "librigw.so"
SOURCES = ["capi.cu", "engine.cu", "ops.cu", "gemm_f64.cu", "kernels_gw.cu", "kernels_aomo.cu",
           "syrk_bf16x3.cu", "syrk_ozaki.cu", "syrk_f64_tma.cu", "qp_noalloc.cu", "scheduler.cu", "serve.cu", "sox.cu",
           "contour.cu", "eigh_jacobi.cu", "dm.cu",
           "ri_ints.cu"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (Path(cand).exists() or cand == "nvcc"):
            return cand
    raise RuntimeError("nvcc not found")


def build(verbose: bool = False, force: bool = False) -> Path:
    srcs = [CSRC / s for s in SOURCES if (CSRC / s).exists()]
    deps = srcs + list(CSRC.glob("*.cuh")) + [HERE.parent / "include" / "rigw.h"]
    if LIB.exists() and not force:
        newest = max(p.stat().st_mtime for p in deps)
        if LIB.stat().st_mtime >= newest:
            return LIB
    objdir = HERE / "_build"
    objdir.mkdir(exist_ok=True)
    objs = []
    procs = []
    for s in srcs:
        o = objdir / (s.stem + ".o")
        objs.append(o)
        cmd = [nvcc(), *NVCC_FLAGS, "-rdc=false", "-c", str(s), "-o", str(o)]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            sys.stderr.write(out.decode())
            raise RuntimeError(f"nvcc failed: {' '.join(cmd)}")
        elif verbose and out:
            sys.stdout.write(out.decode())
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *map(str, objs), "-o", str(tmp),
           "-lcudart"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
