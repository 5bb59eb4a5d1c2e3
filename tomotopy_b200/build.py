"""Builds libtomotopy_b200.so in-tree for sm_100a (nvcc cross-compiles
without a GPU).  `python -m tomotopy_b200.build` or tomotopy_b200.build.build().
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libtomotopy_b200.so")

SOURCES = ["engine.cu", "server.cu", "ingest.cu", "model.cpp", "synth.cpp", "prepare.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(ROOT, "include", "tomotopy_b200.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    if not force and not _stale():
        return LIB
    objs = []
    tmp = os.path.join(HERE, "_build")
    os.makedirs(tmp, exist_ok=True)
    for src in SOURCES:
        obj = os.path.join(tmp, src + ".o")
        cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
               "-I", os.path.join(ROOT, "include"), "-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cu"):
            cmd[1:1] = ["-Xptxas", "-v"] if verbose else []
        subprocess.run(cmd, check=True)
        objs.append(obj)
    out = LIB + ".tmp"
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", out, *objs, "-lpthread"], check=True)
    os.replace(out, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
