"""Failure handling through the C ABI, with every failure made on the host (no kernel is made
to fault): inconsistent table uploads are refused by pr_eval_status and by evaluate; river
roots whose board does not extend the tables' flop are refused before any launch; ranges
holding NaNs, infinities or negative weights are refused by upload_c, pr_upload_batch and
pr_batch_new, and NaNs and infinities by pr_batch_set_ranges (whose finite negative weights
serve gradient checks). After each refusal the sticky status is cleared and the
same objects still solve correctly."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

ERR_ARG, ERR_TABLES = 2, 3


@pytest.fixture(scope="module")
def packed():
    return O.pack_flop_tables(O.REFERENCE_FLOP)


def _builder(P, boards):
    b = P.Builder()
    for cards in boards:
        b.add(int(cards), 1.0)
    return b


def _boards():
    return [O.REFERENCE_FLOP | (1 << t) for t in (5, 20, 33)]


def test_inconsistent_tables_are_refused(packed):
    import pokerrust_b200 as P
    L = P.lib()
    e, c, a = packed
    slot = 33 * 32 // 2 + 5  # colex index of the {turn, river} pair {5, 33}
    bad_cases = []
    # two hands at the same sorted position: not a permutation
    e1 = e.copy().reshape(1326, 1838)
    e1[slot, 1] = (e1[slot, 1] & 2048) | (e1[slot, 0] & 2047)
    bad_cases.append((e1.reshape(-1), c, a))
    # a bucket outside 0..255
    a1 = a.copy().reshape(1326, 1326)
    a1[slot, 7] = 300
    bad_cases.append((e, c, a1.reshape(-1)))
    for ee, cc, aa in bad_cases:
        L.pr_clear_error()
        with pytest.raises(P.PokerLibError):
            P.transfer_flop_eval(O.REFERENCE_FLOP, O.card_order(), O.card_indexes(), ee, cc, aa)
        assert L.pr_last_error() == ERR_TABLES
    # a refused handle kept by a caller is refused again by evaluate, with no launch
    order = np.ascontiguousarray(O.card_order(), np.uint64)
    idx = np.ascontiguousarray(O.card_indexes(), np.uint16)
    ee, cc, aa = (np.ascontiguousarray(x, np.uint16) for x in bad_cases[1])
    h = L.transfer_flop_eval_cuda(O.REFERENCE_FLOP, order.ctypes.data, idx.ctypes.data, ee.ctypes.data,
                                  cc.ctypes.data, aa.ctypes.data)
    assert L.pr_eval_status(h) != 0
    b = _builder(P, _boards())
    rng = np.random.default_rng(1)
    ranges = rng.random((3, 1326), dtype=np.float32)
    ranges[(O.card_order()[None, :] & np.array(_boards(), np.uint64)[:, None]) != 0] = 0
    b.upload_all(ranges)
    L.pr_clear_error()
    assert L.pr_evaluate(b.ptr, h, 0, 0) == ERR_TABLES
    assert np.array_equal(b.download_all(), ranges)  # the staging was left as it was
    L.free_eval_cuda(h)
    # the good tables still work on the same builder
    L.pr_clear_error()
    good = P.transfer_flop_eval(O.REFERENCE_FLOP, O.card_order(), O.card_indexes(), e, c, a)
    b.evaluate(good, 0)
    assert np.all(np.isfinite(b.download_all()))
    assert L.pr_last_error() == 0
    P.free_eval(good)
    b.close()


def test_boards_without_the_flop_are_refused(packed):
    import pokerrust_b200 as P
    L = P.lib()
    e, c, a = packed
    tables = P.transfer_flop_eval(O.REFERENCE_FLOP, O.card_order(), O.card_indexes(), e, c, a)
    other = (1 << 10) | (1 << 20) | (1 << 30) | (1 << 40)  # shares no card with 2c 3c 4c
    b = _builder(P, _boards() + [other])
    ranges = np.ones((4, 1326), np.float32)
    b.upload_all(ranges)
    L.pr_clear_error()
    assert L.pr_evaluate(b.ptr, tables, 0, 0) == ERR_ARG
    assert np.array_equal(b.download_all(), ranges)
    with pytest.raises(P.PokerLibError):
        P.evaluate_gpu(b.ptr, tables, 1, False)
    L.pr_clear_error()
    b.close()
    # the same tables with valid roots
    b = _builder(P, _boards())
    b.upload_all(np.ones((3, 1326), np.float32))
    b.evaluate(tables, 0)
    assert L.pr_last_error() == 0
    b.close()
    P.free_eval(tables)


@pytest.mark.parametrize("bad", [np.nan, np.inf, -1.0])
def test_bad_ranges_are_refused(bad):
    import pokerrust_b200 as P
    L = P.lib()
    b = _builder(P, _boards())
    ok = np.full((3, 1326), 0.5, np.float32)
    b.upload_all(ok)
    row = ok[1].copy()
    row[17] = bad
    L.pr_clear_error()
    L.upload_c(b.ptr, 1, row.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    assert L.pr_last_error() == ERR_ARG
    assert np.array_equal(b.download_all(), ok)  # the slot kept its range
    rows = np.full((3, 1326), 0.25, np.float32)
    rows[2, 5] = bad
    L.pr_clear_error()
    with pytest.raises(P.PokerLibError):
        b.upload_all(rows)
    got = b.download_all()
    assert np.array_equal(got[:2], rows[:2]) and np.array_equal(got[2], ok[2])  # good rows copied
    L.pr_clear_error()
    b.close()

    specs, ranges = P.random_subgames(3, seed=2)
    r = ranges.copy()
    r[1, 0, 100] = bad
    with pytest.raises(P.PokerLibError):
        P.Batch(specs, r)
    bt = P.Batch(specs, ranges)
    if np.isfinite(bad):
        bt.set_ranges(1, r[1])  # finite negative weights: allowed for gradient checks
        bt.set_ranges(1, ranges[1])
    else:
        with pytest.raises(P.PokerLibError):
            bt.set_ranges(1, r[1])
    bt.iterate(2)  # the batch still solves with its valid ranges
    bt.close()
