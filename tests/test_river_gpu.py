"""Parity of the CUDA river solver with the oracle (CPU restatement of state.rs:377-433),
through the C ABI.

Tolerance: results and regrets are f32 sums of up to ~10^5 terms computed in a different
order from the reference; per subgame we require
    max |gpu - oracle| <= 1e-4 * max |oracle|
(1e-4 relative, the parity bound of this path), measured against the largest value of that
subgame's vector so that entries that cancel to ~0 do not turn rounding into a false
failure.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-4


@pytest.fixture(scope="module")
def P():
    import pokerrust_b200 as P
    P.lib()
    return P


@pytest.fixture(scope="module")
def gpu_tables(P, flop_tables):
    e, c, a = flop_tables
    h = P.transfer_flop_eval(O.REFERENCE_FLOP, O.card_order(), O.card_indexes(), e, c, a)
    yield h
    P.free_eval(h)


def subgames(rng, n, turns=None):
    order = O.card_order()
    flop = O.REFERENCE_FLOP
    free = [c for c in range(52) if not (flop >> c) & 1]
    if turns is None:
        turns = rng.choice(free, n)
    board4 = np.array([flop | (1 << int(t)) for t in turns], np.uint64)
    bet = rng.choice(np.arange(1, 17), len(board4)).astype(np.float32)
    opp = rng.random((len(board4), 1326)).astype(np.float32)
    opp[rng.random(opp.shape) < 0.2] = 0.0
    for i in range(len(board4)):
        opp[i][(order & board4[i]) != 0] = 0
    return board4, bet, opp


def random_regrets(rng, n):
    reg = (rng.random((n, 26, 256)) * 50).astype(np.float32)
    reg[rng.random(reg.shape) < 0.3] = 0.0
    reg[:, :, :8] = 0.0                         # all-zero buckets: the 1e-4 cutoff path
    return reg


def assert_close(got, want, what):
    for i in range(len(want)):
        scale = float(np.abs(want[i]).max())
        err = float(np.abs(got[i] - want[i]).max())
        assert err <= TOL * max(scale, 1e-30), f"{what}[{i}]: max err {err:.3e} vs scale {scale:.3e}"


def run_both(P, gpu_tables, flop_tables, board4, bet, opp, reg, player, exploit):
    e, _, a = flop_tables
    b = P.Builder()
    for cards, bt in zip(board4, bet):
        b.add(int(cards), float(bt))
    b.set_regrets(reg)
    b.upload_all(opp)
    P.evaluate_gpu(b.ptr, gpu_tables, player, exploit)
    got = b.download_all()
    got_reg = b.regrets()
    ref_reg = reg.copy()
    want = O.river_batch(O.REFERENCE_FLOP, e, a, board4, bet, opp, ref_reg, player, exploit)
    b.close()
    return got, want, got_reg, ref_reg


@pytest.mark.parametrize("player", [0, 1])
@pytest.mark.parametrize("exploit", [False, True])
def test_one_pass_random_regrets(P, gpu_tables, flop_tables, player, exploit):
    rng = np.random.default_rng(10 + player + 2 * exploit)
    board4, bet, opp = subgames(rng, 12)
    reg = random_regrets(rng, 12)
    got, want, got_reg, ref_reg = run_both(P, gpu_tables, flop_tables, board4, bet, opp, reg, player, exploit)
    assert_close(got, want, "values")
    if exploit:
        assert np.array_equal(got_reg, reg)
    else:
        assert_close(got_reg.reshape(12, -1), ref_reg.reshape(12, -1), "regrets")


def test_one_pass_from_zero_regrets(P, gpu_tables, flop_tables):
    # the reference's starting point: all regrets zero, uniform strategies everywhere
    rng = np.random.default_rng(7)
    board4, bet, opp = subgames(rng, 8)
    reg = np.zeros((8, 26, 256), np.float32)
    got, want, got_reg, ref_reg = run_both(P, gpu_tables, flop_tables, board4, bet, opp, reg, 0, False)
    assert_close(got, want, "values")
    assert_close(got_reg.reshape(8, -1), ref_reg.reshape(8, -1), "regrets")


def test_blocked_and_masked_hands(P, gpu_tables, flop_tables):
    # hands sharing a card with the turn board get exactly zero, whatever range they carry
    rng = np.random.default_rng(8)
    order = O.card_order()
    board4, bet, opp = subgames(rng, 4)
    opp_dirty = opp.copy()
    opp_dirty[:, :] += 1.0                       # nonzero range on blocked hands too
    got, want, _, _ = run_both(P, gpu_tables, flop_tables, board4, bet, opp_dirty,
                               random_regrets(rng, 4), 1, False)
    for i in range(4):
        blocked = (order & board4[i]) != 0
        assert np.all(got[i][blocked] == 0.0)
    assert_close(got, want, "values")


def _trajectory_case(rng, n):
    board4, bet, opp_bb = subgames(rng, n)
    turns = [(int(b) ^ O.REFERENCE_FLOP).bit_length() - 1 for b in board4]
    _, _, opp_sb = subgames(rng, n, turns=turns)
    return board4, bet, opp_bb, opp_sb


def test_iterations_teacher_forced(P, gpu_tables, flop_tables):
    # CFR amplifies f32 rounding: the oracle against itself with a 1-ulp input perturbation
    # differs by ~1e-3 after 100 iterations. So the GPU's update map is checked at states
    # the oracle's own 100-iteration trajectory (SB update then BB update, game.rs:68-119)
    # passes through: from each checkpoint state, one pass per player must agree to 1e-4.
    rng = np.random.default_rng(11)
    n = 6
    board4, bet, opp_bb, opp_sb = _trajectory_case(rng, n)
    e, _, a = flop_tables
    b = P.Builder()
    for cards, bt in zip(board4, bet):
        b.add(int(cards), float(bt))
    ref_reg = np.zeros((n, 26, 256), np.float32)
    checkpoints = {0, 1, 9, 49, 99}
    for it in range(100):
        for player, opp in ((0, opp_bb), (1, opp_sb)):
            if it in checkpoints:
                b.set_regrets(ref_reg)
                b.upload_all(opp)
                P.evaluate_gpu(b.ptr, gpu_tables, player, False)
                got, got_reg = b.download_all(), b.regrets()
            want = O.river_batch(O.REFERENCE_FLOP, e, a, board4, bet, opp, ref_reg, player, False)
            if it in checkpoints:
                assert_close(got, want, f"values, iteration {it + 1}, player {player}")
                assert_close(got_reg.reshape(n, -1), ref_reg.reshape(n, -1),
                             f"regrets, iteration {it + 1}, player {player}")
    b.close()


def test_iterations_free_running(P, gpu_tables, flop_tables):
    # ten iterations on the GPU alone against ten on the oracle alone (drift still small)
    rng = np.random.default_rng(21)
    n = 6
    board4, bet, opp_bb, opp_sb = _trajectory_case(rng, n)
    e, _, a = flop_tables
    b = P.Builder()
    for cards, bt in zip(board4, bet):
        b.add(int(cards), float(bt))
    ref_reg = np.zeros((n, 26, 256), np.float32)
    for it in range(10):
        for player, opp in ((0, opp_bb), (1, opp_sb)):
            b.upload_all(opp)
            P.evaluate_gpu(b.ptr, gpu_tables, player, False)
            got = b.download_all()
            want = O.river_batch(O.REFERENCE_FLOP, e, a, board4, bet, opp, ref_reg, player, False)
    assert_close(got, want, "values after 10 iterations")
    assert_close(b.regrets().reshape(n, -1), ref_reg.reshape(n, -1), "regrets after 10 iterations")
    b.close()


def test_deterministic(P, gpu_tables, flop_tables):
    # no atomics: two runs from the same state give bit-identical values and regrets
    rng = np.random.default_rng(31)
    board4, bet, opp = subgames(rng, 16)
    reg = random_regrets(rng, 16)
    outs = []
    for _ in range(2):
        b = P.Builder()
        for cards, bt in zip(board4, bet):
            b.add(int(cards), float(bt))
        b.set_regrets(reg)
        b.upload_all(opp)
        P.evaluate_gpu(b.ptr, gpu_tables, 0, False)
        outs.append((b.download_all(), b.regrets()))
        b.close()
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])


def test_one_turn_card_all_river_roots(P, gpu_tables, flop_tables):
    # the reduced case: every river root of one turn card (63 * 9 = 567 subgames)
    g = O.Game(O.REFERENCE_FLOP)
    boards, bets = g.river_roots()
    turn = boards[0]
    sel = np.nonzero(boards == turn)[0]
    assert len(sel) == 567
    rng = np.random.default_rng(12)
    _, _, opp = subgames(rng, len(sel), turns=[(int(turn) ^ O.REFERENCE_FLOP).bit_length() - 1] * len(sel))
    reg = random_regrets(rng, len(sel))
    got, want, got_reg, ref_reg = run_both(P, gpu_tables, flop_tables, boards[sel], bets[sel], opp, reg, 0, False)
    assert_close(got, want, "values")
    assert_close(got_reg.reshape(len(sel), -1), ref_reg.reshape(len(sel), -1), "regrets")


def test_full_fixed_flop_pass_sampled(P, gpu_tables, flop_tables):
    # all 27,783 river roots of the fixed-flop game in one launch; 48 of them re-checked
    g = O.Game(O.REFERENCE_FLOP)
    boards, bets = g.river_roots()
    n = len(boards)
    rng = np.random.default_rng(13)
    order = O.card_order()
    opp = rng.random((n, 1326)).astype(np.float32)
    opp[(order[None, :] & boards[:, None]) != 0] = 0
    reg = random_regrets(rng, n)
    e, _, a = flop_tables
    b = P.Builder()
    for cards, bt in zip(boards, bets):
        b.add(int(cards), float(bt))
    b.set_regrets(reg)
    b.upload_all(opp)
    P.evaluate_gpu(b.ptr, gpu_tables, 1, False)
    got = b.download_all()
    got_reg = b.regrets()
    b.close()
    sample = rng.choice(n, 48, replace=False)
    ref_reg = reg[sample].copy()
    want = O.river_batch(O.REFERENCE_FLOP, e, a, boards[sample], bets[sample], opp[sample], ref_reg, 1, False)
    assert_close(got[sample], want, "values")
    assert_close(got_reg[sample].reshape(48, -1), ref_reg.reshape(48, -1), "regrets")
    # size-independent properties on all roots: finite, blocked hands zero, regrets >= 0
    assert np.all(np.isfinite(got))
    assert np.all(got[(order[None, :] & boards[:, None]) != 0] == 0)
    assert np.all(got_reg >= 0)


@pytest.mark.parametrize("player", [0, 1])
def test_best_response_double_precision(P, gpu_tables, flop_tables, player):
    # the double-precision best response against the oracle's double traversal; the only
    # differences are summation orders, so the bound is far tighter than in single precision
    rng = np.random.default_rng(40 + player)
    board4, bet, opp = subgames(rng, 10)
    reg = random_regrets(rng, 10)
    e, _, a = flop_tables
    b = P.Builder()
    for cards, bt in zip(board4, bet):
        b.add(int(cards), float(bt))
    b.set_regrets(reg)
    got = b.best_response_f64(gpu_tables, player, opp.astype(np.float64))
    assert np.array_equal(b.regrets(), reg)
    b.close()
    want = O.river_br_f64(O.REFERENCE_FLOP, e, a, board4, bet.astype(np.float64), opp.astype(np.float64),
                          reg, player)
    for i in range(10):
        scale = np.abs(want[i]).max()
        assert np.abs(got[i] - want[i]).max() <= 1e-9 * scale


def test_shared_memory_sized_by_flop(P, gpu_tables):
    # group arrays are sized by the flop's largest tie-group counts and fit one CTA per SM
    for exploit, fp64 in ((0, 0), (1, 0), (1, 1)):
        smem = P.lib().pr_river_smem_bytes(gpu_tables, exploit, fp64)
        assert 0 < smem <= 227 * 1024


@pytest.mark.parametrize("player", [0, 1])
def test_average_strategy_sums(P, gpu_tables, flop_tables, player):
    # average-strategy sums of one CFR pass and of a second pass on top (the reference keeps
    # none; checked against the oracle's restatement, oracle/river.cpp)
    rng = np.random.default_rng(50 + player)
    n = 8
    board4, bet, opp = subgames(rng, n)
    _, _, own = subgames(rng, n, turns=[(int(x) ^ O.REFERENCE_FLOP).bit_length() - 1 for x in board4])
    reg = random_regrets(rng, n)
    e, _, a = flop_tables
    b = P.Builder()
    for cards, bt in zip(board4, bet):
        b.add(int(cards), float(bt))
    b.enable_average()
    b.set_regrets(reg)
    ref_reg = reg.copy()
    ref_avg = np.zeros((n, 26, 256), np.float32)
    for _ in range(2):
        b.upload_all(opp)
        b.upload_own_all(own)
        P.evaluate_gpu(b.ptr, gpu_tables, player, False)
        got = b.download_all()
        want = O.river_batch_avg(O.REFERENCE_FLOP, e, a, board4, bet, opp, own, ref_reg, ref_avg, player)
        assert_close(got, want, "values")
    avg = b.average_sums()
    b.close()
    assert_close(avg.reshape(n, -1), ref_avg.reshape(n, -1), "average-strategy sums")
    # only the updater's edges accumulate
    t = O.river_tree()
    other = [int(t["edge"][s][k]) for s in range(28) if t["terminal"][s] == 0 and t["actor"][s] != player
             for k in range(t["nchild"][s])]
    assert np.all(avg[:, other, :] == 0)
