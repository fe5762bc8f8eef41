"""Runs the reference's own CUDA library (oracle/_ref/libpoker_ref.so, built from
src/cuda/interface.cu) through its C ABI on the fixed-flop game's 27,783 river roots and
records, for a sample of roots, the regret state before and after every pass together
with the pass's ranges and returned values. Test infrastructure: tests/test_reference_kernel.py starts it in a
fresh process, because the reference never zeroes its `updates` arrays
(src/cuda/interface.cu:75-81) and relies on freshly mapped device memory being zero.

usage: python ref_kernel_runner.py OUT.npz ITERS SEED
"""
import ctypes
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402


def ranges_for(order, boards, rng):
    r = rng.random((len(boards), 1326), dtype=np.float32)
    r[(order[None, :] & boards[:, None]) != 0] = 0.0
    return r


def main():
    out_path, iters, seed = sys.argv[1], int(sys.argv[2]), int(sys.argv[3])
    L = ctypes.CDLL(O.REF_SO)
    vp = ctypes.c_void_p
    L.init_builder.restype = vp
    L.build_river_cuda.restype = ctypes.c_int
    L.build_river_cuda.argtypes = [ctypes.c_long, ctypes.c_float, vp]
    L.upload_c.argtypes = [vp, ctypes.c_int, vp]
    L.download_c.argtypes = [vp, ctypes.c_int, vp]
    L.transfer_flop_eval_cuda.restype = vp
    L.transfer_flop_eval_cuda.argtypes = [ctypes.c_long, vp, vp, vp, vp, vp]
    L.free_eval_cuda.argtypes = [vp]
    L.evaluate_cuda.argtypes = [vp, vp, ctypes.c_short, ctypes.c_bool]
    cudart = ctypes.CDLL("libcudart.so.12") if os.path.exists("/usr/local/cuda/lib64/libcudart.so.12") \
        else ctypes.CDLL("/usr/local/cuda/lib64/libcudart.so")
    cudart.cudaMemcpy.argtypes = [vp, vp, ctypes.c_size_t, ctypes.c_int]

    g = O.Game(O.REFERENCE_FLOP)
    boards, bets = g.river_roots()
    n = len(boards)
    assert n == 63 * 49 * 9
    order = O.card_order()
    e, c, a = O.pack_flop_tables(O.REFERENCE_FLOP)
    co, ci = order.astype(np.int64), O.card_indexes().astype(np.int16)
    p = lambda x: x.ctypes.data_as(vp)
    b = L.init_builder()
    for i in range(n):
        assert L.build_river_cuda(int(boards[i]), float(bets[i]), b) == i
    ev = L.transfer_flop_eval_cuda(O.REFERENCE_FLOP, p(co), p(ci), p(e.view(np.int16)),
                                   p(c.view(np.int16)), p(a.view(np.int16)))
    # Builder { int current_index; State *states; AbstractVector *abstract_vectors; ... }
    # (src/cuda/structs.h:59-67): the regrets are read straight from the device.
    fields = (ctypes.c_void_p * 7).from_address(b)
    abstract_vectors = fields[2]
    reg = np.zeros((n, 26, 256), np.float32)

    def regrets():
        assert cudart.cudaMemcpy(p(reg), abstract_vectors, reg.nbytes, 2) == 0
        return reg[sample].copy()

    # every pass is recorded for a sample of river roots: the state before it, its input
    # ranges, and what it returned and left behind
    srng = np.random.default_rng(seed + 1)
    sample = np.unique(np.concatenate([[0, 27, 45, 324], srng.choice(n, 252, replace=False)]))
    rng = np.random.default_rng(seed)
    res = np.zeros((n, 1326), np.float32)
    rec = {"before": [], "after": [], "ranges": [], "values": [], "player": [], "exploit": []}
    times = []
    passes = [(player, False) for _ in range(iters) for player in (0, 1)] + [(0, True), (1, True)]
    for player, exploit in passes:
        r = ranges_for(order, boards, rng)
        rec["before"].append(regrets())
        for i in range(n):
            L.upload_c(b, i, p(r[i]))
        t0 = time.perf_counter()
        L.evaluate_cuda(b, ev, player, exploit)
        times.append(time.perf_counter() - t0)
        for i in range(n):
            L.download_c(b, i, p(res[i]))
        rec["after"].append(regrets())
        rec["ranges"].append(r[sample])
        rec["values"].append(res[sample].copy())
        rec["player"].append(player)
        rec["exploit"].append(exploit)
    L.free_eval_cuda(ev)
    np.savez(out_path, sample=sample, seconds=np.array(times),
             **{k: np.array(v) for k, v in rec.items()})


if __name__ == "__main__":
    main()
