"""Device-generated hand-rank tables (pr_tables_build) against the oracle's restatement of
src/evaluator.rs:55-135,243-308 and src/cuda_interface.rs:444-475: bit-exact, for the
reference flop and seeded flops."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def P():
    import pokerrust_b200 as P
    P.lib()
    return P


def seeded_flops():
    rng = np.random.default_rng(2024)
    flops = [O.REFERENCE_FLOP]
    for _ in range(3):
        cards = rng.choice(52, 3, replace=False)
        flops.append(int(sum(1 << int(c) for c in cards)))
    return flops


@pytest.mark.parametrize("flop", seeded_flops())
def test_tables_bit_exact(P, flop):
    h = P.build_flop_tables(flop)
    try:
        e, c, a = P.export_tables(h)
    finally:
        P.free_eval(h)
    oe, oc, oa = O.pack_flop_tables(flop)
    assert np.array_equal(e, oe), "eval (sorted order, group flags, chunk bounds)"
    assert np.array_equal(c, oc), "per-card collision lists"
    assert np.array_equal(a, oa), "phs buckets"


def test_generated_tables_drive_the_solver(P, flop_tables):
    # a pass on device-generated tables equals a pass on uploaded oracle tables
    e, c, a = flop_tables
    up = P.transfer_flop_eval(O.REFERENCE_FLOP, O.card_order(), O.card_indexes(), e, c, a)
    gen = P.build_flop_tables(O.REFERENCE_FLOP)
    rng = np.random.default_rng(5)
    order = O.card_order()
    boards = np.array([O.REFERENCE_FLOP | (1 << t) for t in (7, 19, 40)], np.uint64)
    opp = rng.random((3, 1326)).astype(np.float32)
    opp[(order[None, :] & boards[:, None]) != 0] = 0
    outs = []
    for tables in (up, gen):
        b = P.Builder()
        for cards in boards:
            b.add(int(cards), 3.0)
        b.upload_all(opp)
        P.evaluate_gpu(b.ptr, tables, 1, False)
        outs.append((b.download_all(), b.regrets()))
        b.close()
    P.free_eval(up)
    P.free_eval(gen)
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])


def test_table_file_round_trip(tmp_path):
    import pokerrust_b200 as P
    from pokerrust_b200 import interface as I
    t = P.build_flop_tables(0b111)
    path = str(tmp_path / "flop7.prbt")
    I.save_tables(t, path)
    u = I.load_tables(path)
    for a, b in zip(P.export_tables(t), P.export_tables(u)):
        assert np.array_equal(a, b)
    data = bytearray(open(path, "rb").read())
    data[5000] ^= 0x10
    open(path, "wb").write(bytes(data))
    with pytest.raises(P.PokerLibError):
        I.load_tables(path)
    P.free_eval(t)
    P.free_eval(u)
