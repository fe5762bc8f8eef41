"""Generates tests/golden/game_reference_flop_checkpoints.npz with the oracle (the CPU
restatement of src/game.rs, src/state.rs and the river path): the fixed-flop game from zero
regrets with average-strategy sums on, after 10 CFR iterations (game.rs:68-119):
  - exploitability in double precision (game.rs:120-178, formula at :175);
  - the root's values of the last iteration's SB and BB passes (per hand);
  - sums of all upper-tree and river regrets and average sums.
About 25 minutes on 8 cores. Run from the repository root:
    python tests/golden/make_game_checkpoints_golden.py [nthreads]
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

CHECKPOINTS = (10,)


def main():
    nthreads = int(sys.argv[1]) if len(sys.argv) > 1 else 0
    t0 = time.time()
    g = O.Game(O.REFERENCE_FLOP, nthreads)
    g.enable_average()
    out = {"checkpoints": np.array(CHECKPOINTS)}
    for it in range(1, max(CHECKPOINTS) + 1):
        g.iterate()
        print(f"iteration {it}: {time.time() - t0:.0f}s", flush=True)
        if it in CHECKPOINTS:
            out[f"it{it}_totals"] = g.totals()
            out[f"it{it}_root_values"] = g.root_values()
            out[f"it{it}_expl_f64"] = np.array(g.exploitability(True))
            print(it, out[f"it{it}_expl_f64"], f"{time.time() - t0:.0f}s", flush=True)
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "game_reference_flop_checkpoints.npz"), **out)


if __name__ == "__main__":
    main()
