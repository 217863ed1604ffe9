"""Builds the CUDA library ziran2019_b200/lib/libzmpm.so for sm_100a with nvcc.

    python -m ziran2019_b200.build [--force]

The library is built in-tree so that it ships with the repository snapshot.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "lib")
OUT = os.path.join(OUT_DIR, "libzmpm.so")
SOURCES = ["adjoint.cu", "admm.cu", "api.cu", "bin.cu", "io.cu", "noalloc.cu", "phase.cu", "prims.cu", "solver.cu", "transfer.cu"]
HEADERS = ["admm.cuh", "common.cuh", "eig3.cuh", "fused.cuh", "hvp.cuh", "internal.cuh", "mat3.cuh", "models.cuh", "node.cuh", "svd3.cuh",
           "xfer.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--expt-relaxed-constexpr",
    "-ccbin", "/usr/bin/g++",
]


def _stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "zmpm.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    if not force and not _stale():
        return OUT
    os.makedirs(OUT_DIR, exist_ok=True)
    objs = []
    obj_dir = os.path.join(HERE, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    procs = []
    for src in SOURCES:
        obj = os.path.join(obj_dir, src.replace(".cu", ".o"))
        objs.append(obj)
        cmd = [NVCC, *FLAGS, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = False
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed = True
            sys.stderr.write(f"--- nvcc failed on {src}\n{out.decode()}\n")
        elif verbose and out:
            sys.stderr.write(out.decode())
    if failed:
        raise RuntimeError("nvcc build failed")
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", OUT, *objs, "-ccbin", "/usr/bin/g++"]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    args = sys.argv[1:]
    extra = []
    if "--ptxas-v" in args:
        extra = ["-Xptxas", "-v"]
    print(build(force="--force" in args or bool(extra), verbose="-v" in args or bool(extra), extra=extra))
