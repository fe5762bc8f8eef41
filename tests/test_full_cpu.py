"""Full fixed-flop game, host side: the library's flop and turn tree builder against the
oracle's independent restatement of the rules (oracle/full_game.py), and the oracle's own
invariants (zero sum of the sweeps, best response dominates the strategy's value)."""
import numpy as np
import pytest

from oracle import full_game as F

import pokerrust_b200 as P

FLOP = (1 << 0) | (1 << 17) | (1 << 42)

SPECS = [
    # (pot, stack, flop (fracs, allin, raises), turn (fracs, allin, raises))
    (10.0, 100.0, ((0.75,), True, 1), ((0.75,), True, 1)),
    (10.0, 500.0, ((0.33, 0.75, 1.5), True, 2), ((0.5,), False, 1)),
    (20.0, 30.0, ((0.5, 1.0), True, 3), ((1.0,), True, 2)),   # short stacks: bets capped at all-in
    (10.0, 0.0, ((0.75,), True, 1), ((0.75,), True, 1)),      # no chips behind: checks only
    (4.0, 400.0, ((), True, 1), ((0.25,), False, 0)),         # all-in only on the flop, no turn bets
]


def _spec(pot, stack, fl, tu):
    return P.full_spec(FLOP, pot, stack, flop_fracs=fl[0], flop_allin=fl[1], flop_raises=fl[2],
                       turn_fracs=tu[0], turn_allin=tu[1], turn_raises=tu[2])


@pytest.mark.parametrize("pot,stack,fl,tu", SPECS)
def test_tree_matches_oracle(pot, stack, fl, tu):
    nodes, kids, edges, leaves = P.full_tree(_spec(pot, stack, fl, tu))
    want = F.Tree(FLOP, pot, stack, [fl, tu])
    assert len(nodes) == len(want)
    assert edges == want.edges and leaves == len(want.leaves)
    assert np.array_equal(nodes["kind"], want.kind)
    assert np.array_equal(nodes["parent"], want.parent)
    assert np.array_equal(nodes["in_edge"], want.in_edge)
    assert np.array_equal(nodes["level"], want.level)
    assert np.array_equal(nodes["street"], want.street)
    assert np.array_equal(nodes["board"], np.array(want.board, np.uint64))
    act = (nodes["kind"] == F.DECISION) | (nodes["kind"] == F.FOLD)
    assert np.array_equal(nodes["actor"][act], np.array(want.actor)[act])
    dec = nodes["kind"] == F.DECISION
    assert np.array_equal(nodes["edge"][dec], np.array(want.first_edge)[dec])
    lf = nodes["kind"] == F.LEAF
    assert np.array_equal(nodes["edge"][lf], np.array(want.leaf_index)[lf])
    pay = nodes["kind"] == F.FOLD
    assert np.array_equal(nodes["stake"][pay | lf], np.array(want.stake, np.float32)[pay | lf])
    assert np.array_equal(nodes["stack"][lf], np.array(want.stack, np.float32)[lf])
    for i in np.flatnonzero((nodes["kind"] == F.DECISION) | (nodes["kind"] == F.DEAL)):
        got = kids[nodes["kids"][i]:nodes["kids"][i] + nodes["nchild"][i]]
        assert list(got) == want.children[i]
    # every deal node deals the 49 cards off the flop
    assert np.all(nodes["nchild"][nodes["kind"] == F.DEAL] == 49)
    if stack == 0:
        assert np.all(nodes["stack"][lf] == 0) and not np.any(pay)


def test_bad_specs_are_rejected():
    with pytest.raises(P.PokerLibError):
        P.full_tree(P.full_spec(0b11, 10.0, 100.0))   # two cards
    with pytest.raises(P.PokerLibError):
        P.full_tree(P.full_spec(FLOP, 0.0, 100.0))    # no pot
    with pytest.raises(P.PokerLibError):
        P.full_tree(P.full_spec(FLOP, 10.0, -1.0))    # negative stack
    bad = [P.full_spec(FLOP, float("nan"), 100.0), P.full_spec(FLOP, float("inf"), 100.0),
           P.full_spec(FLOP, 10.0, float("inf")),                      # non-finite pot or stack
           P.full_spec(FLOP, 10.0, 100.0, flop_fracs=(0.0,)), P.full_spec(FLOP, 10.0, 100.0, turn_fracs=(float("inf"),)),
           P.full_spec(FLOP, 10.0, 100.0, flop_raises=5),              # street raises 0..4
           P.full_spec(FLOP, 10.0, 100.0, river_sizes=0), P.full_spec(FLOP, 10.0, 100.0, river_sizes=0b1001),
           P.full_spec(FLOP, 10.0, 100.0, river_raises=0), P.full_spec(FLOP, 10.0, 100.0, river_raises=4)]
    for spec in bad:
        with pytest.raises(P.PokerLibError):
            P.full_tree(spec)
    # the limits themselves are accepted
    for spec in (P.full_spec(FLOP, 10.0, 0.0), P.full_spec(FLOP, 10.0, 100.0, flop_raises=4, turn_raises=0),
                 P.full_spec(FLOP, 10.0, 100.0, river_sizes=0b111, river_raises=3),
                 P.full_spec(FLOP, 10.0, 100.0, river_sizes=0b100, river_raises=1)):
        P.full_tree(spec)


def test_oracle_sweeps_zero_sum_and_best_response():
    """With zero-sum leaf values (player 0 wins h0^T M h1 from player 1 at each leaf), the
    sweeps give r0.V0 + r1.V1 = 0 at the root; the best response is at least the strategy's
    value."""
    tree = F.Tree(FLOP, 10.0, 100.0, [((0.75,), True, 1), ((0.75,), False, 0)])
    rng = np.random.default_rng(1)
    init = rng.random((2, F.HANDS))
    init[:, F.blocked(FLOP)] = 0
    init /= init.sum(axis=1, keepdims=True)
    reg = rng.random((tree.edges, F.HANDS)).astype(np.float32)
    R = F.reach(tree, init, reg, False)
    # leaf values: a random antisymmetric payoff matrix per leaf
    L = len(tree.leaves)
    vals = []
    mats = [rng.standard_normal((F.HANDS, F.HANDS)) * 0.01 for _ in range(3)]
    for upd in (0, 1):
        lv = np.zeros((L, F.HANDS))
        for j, node in enumerate(tree.leaves):
            M = mats[j % 3] - mats[j % 3].T
            M = M * F._COMPAT
            # player 0 wins h0^T M h1 from player 1
            lv[j] = M @ R[node, 1] if upd == 0 else -(M.T @ R[node, 0])
        V, _, _ = F.sweep_up(tree, R, lv, upd, reg, False, "eval")
        vals.append(init[upd] @ V[0])
        Vb, _, _ = F.sweep_up(tree, R, lv, upd, reg, False, "br")
        assert init[upd] @ Vb[0] >= vals[-1] - 1e-12
    assert abs(vals[0] + vals[1]) < 1e-9 * max(1.0, abs(vals[0]))


def test_river_specs_of_leaf_states():
    """The 48 river subgames of a turn-leaf state: one per card off the 4-card board, in card
    order, with the leaf's pot and stack and the river card's hands removed from the ranges."""
    from pokerrust_b200 import full_solve as FS
    rng = np.random.default_rng(4)
    boards = np.array([sum(1 << int(c) for c in rng.choice(52, 4, replace=False)) for _ in range(3)], np.uint64)
    ranges = rng.random((3, 2, F.HANDS)).astype(np.float32)
    pots = np.array([10.0, 25.0, 62.5], np.float32)
    stacks = np.array([100.0, 92.5, 0.0], np.float32)
    specs, rr = FS.river_specs(boards, ranges, pots, stacks)
    assert len(specs) == 3 * 48 and rr.shape == (3 * 48, 2, F.HANDS)
    k = 0
    for i in range(3):
        for c in range(52):
            if (int(boards[i]) >> c) & 1:
                continue
            assert int(specs["board"][k]) == int(boards[i]) | (1 << c)
            assert specs["pot"][k] == pots[i] and specs["stack"][k] == stacks[i]
            want = ranges[i].copy()
            want[:, F.blocked(1 << c)] = 0.0
            assert np.array_equal(rr[k], want)
            k += 1
