"""Generates tests/golden/batch500_golden.npz with the oracle (oracle/batch.cpp, the per-hand
restatement of the batch solver's rules): 64 seeded subgames of the 4096-subgame batch of
general river subgames (pokerrust_b200.random_subgames(4096, seed=4321)), each solved for 500
CFR iterations from zero regrets with uniformly weighted average sums, then
  - the double-precision best-response sums of both players and the exploitability of the
    average strategies, and of the current strategies.
Runs the subgames on worker processes (spawned). Run from the repository root:
    python tests/golden/make_batch500_golden.py [workers]
"""
import multiprocessing as mp
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

BATCH, SEED, SAMPLE, ITERATIONS = 4096, 4321, 64, 500


def solve(args):
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    sp, r = args
    o = O.Subgame(int(sp["board"]), float(sp["pot"]), float(sp["stack"]), int(sp["sizes"]), int(sp["max_raises"]),
                  r[0], r[1])
    o.iterate(ITERATIONS, accumulate=True)
    a0, _ = o.best_response(0, use_average=True)
    a1, _ = o.best_response(1, use_average=True)
    c0, _ = o.best_response(0, use_average=False)
    c1, _ = o.best_response(1, use_average=False)
    j = o.joint()
    return a0, a1, (a0 + a1) / 2 / j, (c0 + c1) / 2 / j


def main():
    import pokerrust_b200 as P
    workers = int(sys.argv[1]) if len(sys.argv) > 1 else os.cpu_count()
    t0 = time.time()
    specs, ranges = P.random_subgames(BATCH, seed=SEED)
    sample = np.sort(np.random.default_rng(500).choice(BATCH, SAMPLE, replace=False))
    with mp.get_context("spawn").Pool(workers) as pool:
        res = pool.map(solve, [(specs[s], ranges[s]) for s in sample], chunksize=1)
    res = np.array(res)
    out = dict(sample=sample, iterations=np.array(ITERATIONS), br0_avg=res[:, 0], br1_avg=res[:, 1],
               expl_avg=res[:, 2], expl_cur=res[:, 3])
    print(f"{time.time() - t0:.0f}s; mean exploitability of the average strategies {res[:, 2].mean():.5f} chips",
          flush=True)
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "batch500_golden.npz"), **out)


if __name__ == "__main__":
    main()
