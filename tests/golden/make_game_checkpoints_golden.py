"""Generates tests/golden/game_reference_flop_checkpoints.npz with the oracle (the CPU
restatement of src/game.rs, src/state.rs and the river path): the fixed-flop game from zero
regrets with average-strategy sums on, after 1, 5 and 10 CFR iterations (game.rs:68-119):
  - exploitability in double precision (game.rs:120-178, formula at :175);
  - the root's values of the last iteration's SB and BB passes (per hand);
  - sums of all upper-tree and river regrets and average sums.
With --descending the river passes visit the river cards in descending order (the same sums
in another f32 rounding) and the file is game_reference_flop_checkpoints_descending.npz.
About 30 minutes on 8 cores. Run from the repository root:
    python tests/golden/make_game_checkpoints_golden.py [--descending] [nthreads]
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

CHECKPOINTS = (1, 5, 10)


def main():
    args = sys.argv[1:]
    descending = "--descending" in args
    args = [a for a in args if a != "--descending"]
    nthreads = int(args[0]) if args else 0
    O.set_river_order(descending)
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
    name = "game_reference_flop_checkpoints_descending.npz" if descending else "game_reference_flop_checkpoints.npz"
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", name), **out)


if __name__ == "__main__":
    main()
