"""Host-side helpers of the full-game comparison and the value-network data (no GPU): the
time-to-level reading of a trajectory, training-set merging and the seeded turn states."""
import numpy as np

import pokerrust_b200 as P
from pokerrust_b200 import full_solve as FS
from pokerrust_b200 import value_data as D


def test_time_to_levels_takes_the_first_checkpoint_at_or_below_each_level():
    points = [{"solver_s": 1.0, "pct": 5.0}, {"solver_s": 2.0, "pct": 2.5}, {"solver_s": 3.0, "pct": 2.7},
              {"solver_s": 4.0, "pct": 1.2}]
    got = FS.time_to_levels(points, "pct", (6.0, 2.5, 2.0, 1.0))
    assert got == {"6.0": 1.0, "2.5": 2.0, "2.0": 4.0, "1.0": None}
    assert FS.time_to_levels([], "pct", (1.0,)) == {"1.0": None}


def test_merge_concatenates_every_array_and_adds_the_solve_time():
    def part(n, s):
        return {"boards": np.arange(n, dtype=np.uint64), "ranges": np.zeros((n, 2, 1326), np.float32),
                "scalars": np.zeros((n, 2), np.float32), "values": np.ones((n, 2652), np.float32) * s,
                "pots": np.full(n, 10.0, np.float32), "stacks": np.full(n, 50.0, np.float32), "solve_s": s}
    m = FS.merge(part(3, 1.5), part(2, 2.0))
    assert len(m["boards"]) == 5 and m["ranges"].shape == (5, 2, 1326) and m["values"].shape == (5, 2652)
    assert np.array_equal(m["values"][:, 0], [1.5, 1.5, 1.5, 2.0, 2.0])
    assert m["solve_s"] == 3.5


def test_turn_states_are_seeded_normalised_and_respect_the_board():
    boards, ranges, pots, stacks = D.turn_states(16, seed=3)
    b2, r2, p2, s2 = D.turn_states(16, seed=3)
    assert np.array_equal(boards, b2) and np.array_equal(ranges, r2)
    assert np.array_equal(pots, p2) and np.array_equal(stacks, s2)
    order = P.card_order()
    for i in range(16):
        assert bin(int(boards[i])).count("1") == 4
        assert pots[i] >= 2 and pots[i] <= 200 and pots[i] <= stacks[i] <= 10 * pots[i]
        blocked = (order & boards[i]) != 0
        for p in range(2):
            assert not ranges[i, p, blocked].any()
            assert abs(float(ranges[i, p].sum()) - 1.0) < 1e-5
            assert (ranges[i, p] >= 0).all()


def test_full_solve_configurations_are_well_formed():
    for name, c in FS.CONFIGS.items():
        assert c["pot"] > 0 and c["stack"] >= c["pot"], name
        assert all(0 < f for f in c["fracs"]) and c["raises"] >= 1, name
