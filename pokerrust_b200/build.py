"""Builds the CUDA library in-tree: pokerrust_b200/_lib/libpokerrust_b200.so (and a static
libpoker.a with the same objects, the archive name the reference's build.rs links)."""
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "_lib")
SO_PATH = os.path.join(LIB_DIR, "libpokerrust_b200.so")
A_PATH = os.path.join(LIB_DIR, "libpoker.a")
SOURCES = ["abi.cu", "river_cfr.cu", "pack_boards.cu", "gen_tables.cu", "game.cu", "upper_tree.cu",
           "batch_solver.cu", "batch_api.cu"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
]


def nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build pokerrust_b200")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    os.makedirs(LIB_DIR, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "pokerrust_b200.h"))
    if not force and not _stale(SO_PATH, deps) and not _stale(A_PATH, deps):
        return SO_PATH
    objs = []
    for src in SOURCES:
        obj = os.path.join(LIB_DIR, src.replace(".cu", ".o"))
        cmd = [nvcc(), *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [nvcc(), *NVCC_FLAGS, "--shared", "-o", SO_PATH, *objs, "-lcudart"]
    subprocess.run(cmd, check=True)
    if os.path.exists(A_PATH):
        os.remove(A_PATH)
    subprocess.run(["ar", "rcs", A_PATH, *objs], check=True)
    return SO_PATH


if __name__ == "__main__":
    print(build(force=True, verbose=True))
