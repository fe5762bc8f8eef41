"""Generates tests/golden/game_reference_flop_100.npz with the oracle (the CPU restatement
of src/game.rs, src/state.rs and the river path), the stated comparison of the fixed-flop
game: 100 CFR iterations (game.rs:68-119) from zero regrets with average-strategy sums on,
then
  - exploitability in double and single precision (game.rs:120-178, formula at :175);
  - the root's values of the 100th iteration's SB and BB passes (per hand);
  - sums of all upper-tree and river regrets and average sums;
  - average sums of 64 seeded river roots.
About three hours on 8 cores. Run from the repository root:
    python tests/golden/make_game100_golden.py [nthreads]
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

ITERATIONS = 100


def main():
    nthreads = int(sys.argv[1]) if len(sys.argv) > 1 else 0
    t0 = time.time()
    g = O.Game(O.REFERENCE_FLOP, nthreads)
    g.enable_average()
    for it in range(ITERATIONS):
        g.iterate()
        print(f"iteration {it + 1}: {time.time() - t0:.0f}s", flush=True)
    out = {"iterations": np.array(ITERATIONS)}
    out["root_values"] = g.root_values()
    out["totals"] = g.totals()
    sample = np.random.default_rng(100).choice(g.num_rivers, 64, replace=False)
    out["river_sample"] = sample
    out["river_average"] = g.river_average()[sample]
    out["expl_f64"] = np.array(g.exploitability(True))
    print("f64", out["expl_f64"], f"{time.time() - t0:.0f}s", flush=True)
    out["expl_f32"] = np.array(g.exploitability(False))
    print("f32", out["expl_f32"], f"{time.time() - t0:.0f}s", flush=True)
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "game_reference_flop_100.npz"), **out)


if __name__ == "__main__":
    main()
