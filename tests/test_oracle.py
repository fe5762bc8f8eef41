"""Oracle self-checks: known answers for the hand ranking, the reference's structural
assertions, and invariants of the river traversal (no GPU)."""
import itertools

import numpy as np
import pytest

from oracle import oracle as O


def test_seven_card_category_counts_and_classes():
    # Published counts of the 133,784,560 seven-card hands per category (high card .. straight
    # flush) and the 4,824 distinct seven-card hand values.
    counts, distinct = O.count_7card()
    assert list(counts) == [23294460, 58627800, 31433400, 6461620, 6180020, 4047644, 3473184,
                            224848, 41584]
    assert distinct == 4824


def test_hand_ranking_examples():
    # card = 13 * suit + rank; rank 0 = deuce, suit order clubs, hearts, spades, diamonds
    def c(r, s):
        return 1 << (13 * s + r)
    royal = c(12, 0) | c(11, 0) | c(10, 0) | c(9, 0) | c(8, 0)
    wheel_sf = c(12, 1) | c(0, 1) | c(1, 1) | c(2, 1) | c(3, 1)
    quads = c(5, 0) | c(5, 1) | c(5, 2) | c(5, 3) | c(0, 0)
    boat = c(4, 0) | c(4, 1) | c(4, 2) | c(9, 0) | c(9, 1)
    flush = c(0, 2) | c(3, 2) | c(5, 2) | c(7, 2) | c(11, 2)
    wheel = c(12, 0) | c(0, 1) | c(1, 2) | c(2, 3) | c(3, 0)
    six_high = c(4, 0) | c(0, 1) | c(1, 2) | c(2, 3) | c(3, 0)
    v = O.hand_value
    assert v(royal) > v(wheel_sf) > v(quads) > v(boat) > v(flush) > v(six_high) > v(wheel)
    # best five of seven: the extra cards do not matter below the kickers
    assert v(quads | c(1, 0) | c(2, 0)) == v(c(5, 0) | c(5, 1) | c(5, 2) | c(5, 3) | c(2, 0))
    # two pair with a third pair: the kicker is the best remaining rank
    tp = c(10, 0) | c(10, 1) | c(8, 0) | c(8, 1) | c(6, 0) | c(6, 1) | c(1, 2)
    assert v(tp) == v(c(10, 0) | c(10, 1) | c(8, 0) | c(8, 1) | c(6, 2))


def test_colex_and_card_tables():
    order = O.card_order()
    assert np.all(np.diff(order.astype(np.float64)) > 0)        # evaluator.rs:39 sorted
    for i in [0, 1, 2, 100, 1325]:
        assert O.load().or_colex_index(int(order[i])) == i     # combination_map.rs:33-42
        assert O.load().or_pair_from_index(i) == order[i]
    ci = O.card_indexes().reshape(52, 51)                        # evaluator.rs:159-172
    for c in range(52):
        assert all((int(order[h]) >> c) & 1 for h in ci[c])
        assert np.all(np.diff(ci[c].astype(int)) > 0)


def test_board_tables_invariants(flop_tables):
    e, coll, a = flop_tables
    e = e.reshape(1326, 1838)
    coll = coll.reshape(1326, 52 * 51)
    a = a.reshape(1326, 1326)
    order = O.card_order()
    flop = O.REFERENCE_FLOP
    valid = [j for j in range(1326) if not (int(order[j]) & flop)]
    assert len(valid) == 1176                                   # C(49, 2) boards
    for j in valid[::97]:
        board = flop | int(order[j])
        pos = e[j, :1326] & 2047
        assert sorted(pos.tolist()) == list(range(1326))        # a permutation
        blocked = np.array([(int(o) & board) != 0 for o in order])
        assert blocked.sum() == 245
        assert np.all(pos[blocked] < 245)                       # Eval::WORST sorts first
        assert a[j].max() <= 255 and np.all(a[j][blocked] == 0)  # strategy.rs:114 bound
        # a card list holds the 51 hands with that card (evaluator.rs:108-130)
        for card in [0, 17, 51]:
            hands = coll[j, card * 51:(card + 1) * 51] & 2047
            assert all((int(order[h]) >> card) & 1 for h in hands)
            assert np.all(np.diff(pos[hands].astype(int)) > 0)   # rank order


def test_tables_match_direct_construction():
    # or_board_tables (evaluator.rs:55-135) against a direct numpy restatement of the sort
    order = O.card_order()
    board = O.REFERENCE_FLOP | (1 << 20) | (1 << 45)
    e, _, a = O.board_tables(board)
    vals = np.array([0 if int(o) & board else O.hand_value(int(o) | board) for o in order])
    perm = np.lexsort((np.arange(1326), vals))
    assert np.array_equal(e[:1326] & 2047, perm)
    starts = np.r_[True, vals[perm][1:] > vals[perm][:-1]]
    assert np.array_equal((e[:1326] & 2048) > 0, starts)
    # phs: (2 * worse + 2 * tied - 1) * 256 / 1980 over opponent hands sharing no card
    live = [h for h in range(1326) if not int(order[h]) & board]
    for h in live[::53]:
        w = t = 0
        for o in live:
            if int(order[o]) & int(order[h]):
                continue
            w += vals[o] < vals[h]
            t += vals[o] == vals[h]
        assert a[h] == ((2 * w + 2 * t - 1) * 256) // 1980


def test_river_tree_structure():
    t = O.river_tree()
    assert (t["terminal"] == 3).sum() == 9                   # showdowns
    assert np.isin(t["terminal"], [1, 2]).sum() == 8         # folds
    assert (t["terminal"] == 0).sum() == 10                  # decision states
    assert (t["edge"] >= 0).sum() == 26                      # interface.cu:76
    assert sorted(t["edge"][t["edge"] >= 0].tolist()) == list(range(26))


def _river_case(rng, n, tables):
    order = O.card_order()
    flop = O.REFERENCE_FLOP
    turns = rng.choice([c for c in range(52) if not (flop >> c) & 1], n)
    board4 = np.array([flop | (1 << int(t)) for t in turns], np.uint64)
    bet = rng.choice([1.0, 2.0, 3.0, 5.0, 9.0], n).astype(np.float32)
    opp = rng.random((n, 1326)).astype(np.float32)
    for i in range(n):
        opp[i][(order & board4[i]) != 0] = 0
    return board4, bet, opp


def _brute_river_values(tables, board4, bet, opp, player):
    """Per-hand values under uniform strategies from a pairwise O(n^2) evaluation."""
    e, _, a = tables
    order = O.card_order()
    tree = O.river_tree()
    flop = O.REFERENCE_FLOP
    total = np.zeros(1326)
    for rc in range(52):
        if (int(board4) >> rc) & 1:
            continue
        board = int(board4) | (1 << rc)
        vals = np.array([0 if int(o) & board else O.hand_value(int(o) | board) for o in order], np.int64)
        live = np.array([not (int(o) & board) for o in order])
        x = np.where(live, opp, 0.0)
        share = (order[:, None] & order[None, :]) != 0
        sgn = np.sign(vals[:, None] - vals[None, :]) * ~share
        sd = sgn @ x
        fold = (~share).astype(np.float64) @ x

        def value(s, reach_opp):
            term = tree["terminal"][s]
            if term == 3:
                return (bet + tree["sb_off"][s]) * sd * reach_opp
            if term in (1, 2):
                folder = 1 if term == 1 else 0
                b = bet + (tree["bb_off"][s] if folder == 1 else tree["sb_off"][s])
                return (-b if folder == player else b) * fold * reach_opp
            nk = tree["nchild"][s]
            out = 0.0
            for k in range(nk):
                c = tree["child"][s][k]
                if tree["actor"][s] == player:
                    out = out + value(c, reach_opp) / nk
                else:
                    out = out + value(c, reach_opp / nk)
            return out

        total += np.where(live, value(1, 1.0), 0.0)
    return total / 48


def test_river_values_match_pairwise_brute_force(flop_tables):
    # evaluate_showdown / evaluate_fold (state.rs:456-569) against the O(n^2) definition
    rng = np.random.default_rng(1)
    board4, bet, opp = _river_case(rng, 2, flop_tables)
    e, _, a = flop_tables
    for player in (0, 1):
        reg = np.zeros((2, 26, 256), np.float32)
        got = O.river_batch(O.REFERENCE_FLOP, e, a, board4, bet, opp, reg, player, False)
        for i in range(2):
            want = _brute_river_values(flop_tables, board4[i], float(bet[i]), opp[i].astype(np.float64), player)
            np.testing.assert_allclose(got[i], want, rtol=1e-4, atol=1e-4 * np.abs(want).max())


def test_river_zero_sum(flop_tables):
    # sum_h r_sb(h) v_sb(h) + sum_h r_bb(h) v_bb(h) = 0 for the same strategies
    rng = np.random.default_rng(2)
    e, _, a = flop_tables
    board4, bet, r_bb = _river_case(rng, 3, flop_tables)
    _, _, r_sb = _river_case(rng, 3, flop_tables)
    reg = rng.random((3, 26, 256)).astype(np.float32) * 5
    v_sb = O.river_batch(O.REFERENCE_FLOP, e, a, board4, bet, r_bb, reg.copy(), 0, True)
    # best response values dominate the strategy's values; use exploit=False for zero-sum
    v_sb = O.river_batch(O.REFERENCE_FLOP, e, a, board4, bet, r_bb, reg.copy(), 0, False)
    v_bb = O.river_batch(O.REFERENCE_FLOP, e, a, board4, bet, r_sb, reg.copy(), 1, False)
    # cfvs weight the opponent range; own reach enters through the own range at the root
    for i in range(3):
        s = np.dot(r_sb[i].astype(np.float64), v_sb[i]) + np.dot(r_bb[i].astype(np.float64), v_bb[i])
        scale = np.abs(r_sb[i] * v_sb[i]).sum()
        assert abs(s) <= 1e-4 * scale


def test_best_response_dominates(flop_tables):
    rng = np.random.default_rng(3)
    e, _, a = flop_tables
    board4, bet, opp = _river_case(rng, 2, flop_tables)
    reg = rng.random((2, 26, 256)).astype(np.float32)
    for player in (0, 1):
        cfv = O.river_batch(O.REFERENCE_FLOP, e, a, board4, bet, opp, reg.copy(), player, False)
        br = O.river_batch(O.REFERENCE_FLOP, e, a, board4, bet, opp, reg.copy(), player, True)
        assert np.all(br >= cfv - 1e-3 * np.abs(cfv).max())
        br64 = O.river_br_f64(O.REFERENCE_FLOP, e, a, board4, bet, opp, reg, player)
        np.testing.assert_allclose(br, br64, rtol=1e-4, atol=1e-4 * np.abs(br64).max())


def test_game_structure():
    g = O.Game(O.REFERENCE_FLOP)
    assert g.num_rivers == 63 * 49 * 9                       # interface.cu:17
    boards, bets = g.river_roots()
    assert all(bin(int(b)).count("1") == 4 for b in boards[:100])
    # preflop raises +1 (bb 1 .. 4), flop +1, turn +2 (state.rs:128-132)
    assert set(np.unique(bets).tolist()) == set(float(x) for x in range(1, 17))


def test_river_order_changes_only_the_rounding(flop_tables):
    # the descending river order (or_set_river_order) sums the same 48 river values: the
    # results agree to f32 rounding, and differ from the reference's order in some bits
    rng = np.random.default_rng(4)
    e, _, a = flop_tables
    board4, bet, opp = _river_case(rng, 3, flop_tables)
    reg0 = rng.random((3, 26, 256)).astype(np.float32) * 5
    try:
        out = {}
        for descending in (False, True):
            O.set_river_order(descending)
            reg = reg0.copy()
            v = O.river_batch(O.REFERENCE_FLOP, e, a, board4, bet, opp, reg, 0, False)
            out[descending] = (v, reg)
    finally:
        O.set_river_order(False)
    (va, ra), (vd, rd) = out[False], out[True]
    assert np.abs(va - vd).max() <= 1e-5 * np.abs(va).max()
    assert np.abs(ra - rd).max() <= 1e-5 * np.abs(ra).max()
    assert not np.array_equal(va, vd)


def test_game_trajectory_depends_on_summation_order():
    """The oracle's fixed-flop game in the reference's river order and in the descending one
    (tests/golden/make_game_checkpoints_golden.py [--descending]): the same sums in another f32
    rounding. After one iteration the runs agree to rounding; by the fifth the root values have
    moved by 2 % (regret matching turns tie residues into pure strategies), and after ten the
    aggregates are back within the bounds tests/test_game100_gpu.py holds the device to."""
    import os
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    asc = dict(np.load(os.path.join(here, "game_reference_flop_checkpoints.npz")))
    desc = dict(np.load(os.path.join(here, "game_reference_flop_checkpoints_descending.npz")))

    def root_err(it):
        a, d = asc[f"it{it}_root_values"], desc[f"it{it}_root_values"]
        return max(np.abs(d[p] - a[p]).max() / np.abs(a[p]).max() for p in range(2))

    def rel(key):
        return np.abs(desc[key] - asc[key]) / np.abs(asc[key])

    assert root_err(1) < 1e-5 and rel("it1_totals").max() < 1e-5 and rel("it1_expl_f64").max() < 1e-5
    assert root_err(5) > 5e-3                      # measured 2.1e-2
    assert root_err(10) < 1e-2 and rel("it10_totals").max() < 1e-2 and rel("it10_expl_f64")[2] < 5e-2
