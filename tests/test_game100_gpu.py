"""The fixed-flop game after the stated 100 CFR iterations on the device (pr_game_*), against
the oracle's own 100-iteration run of the same game (tests/golden/game_reference_flop_100.npz,
made by tests/golden/make_game100_golden.py): FP64 exploitability (game.rs:120-178), the
root's counterfactual values of the 100th iteration, and the sums of the regrets and average
sums above and inside the river subgames.

Tolerance 1 % for every aggregate. Single regrets are not compared after 100 iterations: two
f32 implementations that sum in different orders drift apart through the clipping at zero
(a one-ulp change of the oracle's own inputs moves single bucket regrets by up to 1.9e-3
relative after 100 iterations), while exploitability, root values and sums over the whole
game average that drift out. The tests of single passes hold 1e-4 (test_river_gpu.py).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "game_reference_flop_100.npz")
TOL = 1e-2


@pytest.fixture(scope="module")
def golden():
    if not os.path.exists(GOLDEN):
        pytest.skip("100-iteration golden game fixture missing")
    return dict(np.load(GOLDEN))


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-30)


def test_hundred_iterations_match_the_oracle(golden):
    import pokerrust_b200 as P
    g = P.Game(O.REFERENCE_FLOP)
    g.enable_average()
    g.iterate(int(golden["iterations"]))

    d1, d2, dm = g.exploitability(fp64=True)
    w1, w2, wm = golden["expl_f64"]
    print(f"\nFP64 exploitability after 100 iterations: {dm:.4f} mb/h (oracle {wm:.4f}); "
          f"relative {rel(dm, wm):.2e}")
    assert rel(dm, wm) < TOL and rel(d1, w1) < TOL and rel(d2, w2) < TOL, (d1, d2, dm, golden["expl_f64"])

    root = g.root_values()
    want = golden["root_values"]
    for p in range(2):
        err = np.abs(root[p] - want[p]).max() / np.abs(want[p]).max()
        print(f"root values, player {p}: max error {err:.2e} of the largest value")
        assert err < TOL, (p, err)

    up, river = g.regrets()
    aup, ariver = g.average_sums()
    got = np.array([up.astype(np.float64).sum(), aup.astype(np.float64).sum(),
                    river.astype(np.float64).sum(), ariver.astype(np.float64).sum()])
    for name, a, b in zip(("upper regrets", "upper average sums", "river regrets", "river average sums"),
                          got, golden["totals"]):
        print(f"{name}: {a:.6e} (oracle {b:.6e})")
        assert rel(a, b) < TOL, (name, a, b)

    # average sums of the sampled river roots, each an aggregate over 48 rivers and 26 edges
    s = golden["river_sample"]
    ga, wa = ariver[s].astype(np.float64), golden["river_average"].astype(np.float64)
    per_root = np.abs(ga - wa).sum(axis=(1, 2)) / np.abs(wa).sum(axis=(1, 2))
    assert np.median(per_root) < TOL, np.sort(per_root)
    g.close()
