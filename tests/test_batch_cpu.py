"""Batched general river subgames, host side: the library's bet-tree builder against the
oracle's independent restatement of the rules, the workload generator, and the oracle's
own invariants (zero sum, best response dominates, exploitability of a fixed point)."""
import numpy as np
import pytest

from oracle import oracle as O

import pokerrust_b200 as P


def _specs(seed, n):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        pot = float(rng.integers(2, 201))
        stack = float(rng.integers(int(pot), 10 * int(pot) + 1))
        out.append((pot, stack, int(rng.integers(1, 8)), int(rng.integers(1, 4))))
    # edge cases: a short stack (bets capped at all-in), coinciding sizes, all-in only, no
    # chips behind (checks to the showdown, as after an all-in on an earlier street)
    out += [(100.0, 30.0, 7, 3), (100.0, 100.0, 7, 3), (10.0, 10.0, 3, 2), (50.0, 500.0, 4, 3),
            (2.0, 20.0, 1, 1), (200.0, 2000.0, 7, 3), (40.0, 0.0, 3, 2)]
    return out


@pytest.mark.parametrize("seed", [0, 1])
def test_tree_matches_oracle(seed):
    checked = 0
    for pot, stack, sizes, raises in _specs(seed, 150):
        want = O.bet_tree(pot, stack, sizes, raises)
        try:
            nodes, edges, leaves = P.bet_tree(pot, stack, sizes, raises)
        except P.PokerLibError:
            # the library's limits: at most 128 nodes and 64 leaves, depth <= 5
            assert len(want["kind"]) > 128 or want["num_leaves"] > 64 or want["depth"].max() > 5
            continue
        assert len(nodes) == len(want["kind"])
        assert edges == want["num_edges"] and leaves == want["num_leaves"]
        assert np.array_equal(nodes["kind"], want["kind"])
        assert np.array_equal(nodes["depth"], want["depth"])
        assert np.array_equal(nodes["stake"], want["stake"])
        par = np.where(nodes["parent"] == 0xFFFF, -1, nodes["parent"].astype(np.int64))
        assert np.array_equal(par, want["parent"])
        ie = np.where(nodes["in_edge"] == 0xFFFF, -1, nodes["in_edge"].astype(np.int64))
        assert np.array_equal(ie, want["in_edge"])
        dec = nodes["kind"] == 0
        assert np.array_equal(nodes["nchild"][dec], want["nchild"][dec])
        assert np.array_equal(nodes["actor"][dec], want["actor"][dec])
        fold = nodes["kind"] == 1
        assert np.array_equal(nodes["actor"][fold], want["actor"][fold])
        checked += 1
    assert checked > 100


def test_bad_subgame_specs_are_refused():
    # pot positive and finite, stack non-negative and finite, a bet size among bits 0-2,
    # 1..3 bets and raises
    for pot, stack, sizes, raises in [(0.0, 10.0, 3, 2), (float("nan"), 10.0, 3, 2), (float("inf"), 10.0, 3, 2),
                                      (10.0, -1.0, 3, 2), (10.0, float("inf"), 3, 2), (10.0, 100.0, 0, 2),
                                      (10.0, 100.0, 8, 2), (10.0, 100.0, 11, 2), (10.0, 100.0, 3, 0),
                                      (10.0, 100.0, 3, 4)]:
        with pytest.raises(P.PokerLibError):
            P.bet_tree(pot, stack, sizes, raises)
    P.bet_tree(10.0, 0.0, 1, 1)  # no chips behind: checks to the showdown


def test_generator_shapes():
    specs, ranges = P.random_subgames(64, seed=3)
    assert ranges.shape == (64, 2, 1326)
    np.testing.assert_allclose(ranges.sum(axis=2), 1.0, rtol=1e-5)
    order = P.card_order()
    for s, r in zip(specs, ranges):
        assert bin(int(s["board"])).count("1") == 5
        assert 2 <= s["pot"] <= 200 and s["pot"] <= s["stack"] <= 10 * s["pot"]
        blocked = (order & np.uint64(s["board"])) != 0
        assert np.all(r[:, blocked] == 0)
        n, _, _ = P.bet_tree(s["pot"], s["stack"], s["sizes"], s["max_raises"])
        assert 5 <= len(n) <= 60


@pytest.fixture(scope="module")
def small():
    specs, ranges = P.random_subgames(2, seed=11)
    s = specs[0]
    return O.Subgame(int(s["board"]), float(s["pot"]), float(s["stack"]), int(s["sizes"]),
                     int(s["max_raises"]), ranges[0, 0], ranges[0, 1])


def test_oracle_zero_sum_and_best_response(small):
    rng = np.random.default_rng(5)
    small.regrets = rng.random((small.edges, 1326), dtype=np.float32)
    v0, _ = small.value(0)
    v1, _ = small.value(1)
    assert abs(v0 + v1) < 1e-9 * max(1.0, abs(v0))
    b0, _ = small.best_response(0)
    b1, _ = small.best_response(1)
    assert b0 >= v0 - 1e-12 and b1 >= v1 - 1e-12
    assert (b0 + b1) / 2 / small.joint() > 0


def test_oracle_cfr_converges(small):
    small.regrets = np.zeros((small.edges, 1326), np.float32)
    small.average = np.zeros((small.edges, 1326), np.float32)
    _, _, e0 = small.exploitability()
    small.iterate(30, accumulate=True)
    _, _, e1 = small.exploitability(use_average=True)
    assert e1 < 0.3 * e0
