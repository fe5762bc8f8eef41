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
           "batch_solver.cu", "batch_api.cu", "mlp_gemm.cu", "mlp.cu", "full_game.cu"]
# sources built on CuTe's sm100 atoms (tcgen05 MMA, TMA, TMEM): they need the CUTLASS headers
CUTE_SOURCES = {"mlp_gemm.cu", "mlp.cu"}
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
]


def nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build pokerrust_b200")


def cutlass_include():
    """The CUTLASS / CuTe header tree shipped inside the installed flashinfer package."""
    import importlib.util
    for name in ("flashinfer", "tilelang"):
        spec = importlib.util.find_spec(name)
        if spec is None or not spec.submodule_search_locations:
            continue
        for root in spec.submodule_search_locations:
            for rel in ("data/cutlass/include", "3rdparty/cutlass/include"):
                cand = os.path.join(root, rel)
                if os.path.exists(os.path.join(cand, "cute", "tensor.hpp")):
                    return cand
    raise RuntimeError("CUTLASS headers not found (flashinfer/data/cutlass/include)")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, verbose):
    obj = os.path.join(LIB_DIR, src.replace(".cu", ".o"))
    flags = list(NVCC_FLAGS)
    if src in CUTE_SOURCES:
        flags += ["-I", cutlass_include(), "--expt-relaxed-constexpr"]
    cmd = [nvcc(), *flags, "-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return obj


def build(force=False, verbose=False):
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(LIB_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "pokerrust_b200.h"))
    todo = []
    for src in SOURCES:
        obj = os.path.join(LIB_DIR, src.replace(".cu", ".o"))
        if force or _stale(obj, [os.path.join(CSRC, src), *headers]):
            todo.append(src)
    objs = [os.path.join(LIB_DIR, s.replace(".cu", ".o")) for s in SOURCES]
    if not todo and not _stale(SO_PATH, objs) and not _stale(A_PATH, objs):
        return SO_PATH
    with ThreadPoolExecutor(max(1, min(len(todo), os.cpu_count() or 1))) as ex:
        list(ex.map(lambda s: _compile(s, verbose), todo))
    cmd = [nvcc(), *NVCC_FLAGS, "--shared", "-o", SO_PATH, *objs, "-lcudart"]
    subprocess.run(cmd, check=True)
    if os.path.exists(A_PATH):
        os.remove(A_PATH)
    subprocess.run(["ar", "rcs", A_PATH, *objs], check=True)
    return SO_PATH


if __name__ == "__main__":
    print(build(force=True, verbose=True))
