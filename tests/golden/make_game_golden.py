"""Generates tests/golden/game_reference_flop.npz with the oracle (the CPU restatement of
src/game.rs, src/state.rs and the river path): exploitability of the fixed-flop game in
single and double precision before any update and after two CFR iterations, and the river
regrets of 64 sampled roots after the two iterations. Run from the repository root:
    python tests/golden/make_game_golden.py
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402


def main():
    t0 = time.time()
    g = O.Game(O.REFERENCE_FLOP)
    out = {}
    for tag in ("it0", "it2"):
        if tag == "it2":
            g.iterate()
            g.iterate()
        a, b, m = g.exploitability(False)
        out[f"{tag}_f32"] = np.array([a, b, m])
        a, b, m = g.exploitability(True)
        out[f"{tag}_f64"] = np.array([a, b, m])
        print(tag, out[f"{tag}_f32"], out[f"{tag}_f64"], f"{time.time() - t0:.0f}s", flush=True)
    sample = np.random.default_rng(77).choice(g.num_rivers, 64, replace=False)
    out["river_sample"] = sample
    out["river_regrets_it2"] = g.river_regrets()[sample]
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "game_reference_flop.npz"), **out)


if __name__ == "__main__":
    main()
