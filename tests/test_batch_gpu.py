"""Batched general river subgames on the GPU (pr_batch_*) against the oracle's per-hand
restatement (oracle/batch.cpp).

Tolerances: one CFR iteration from the same regrets differs from the oracle only by the
rounding of the leaf values (f32 prefix sums on the device, f64 pairwise sums rounded to
f32 in the oracle), so regrets and average sums agree to 1e-4 of their largest entry.
Best responses and strategy evaluations run in double precision on both sides: 1e-9.
Free-running iterations amplify f32 rounding through the clipping at zero, so after many
iterations only exploitability is compared, at 2 %.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _oracle(specs, ranges, s):
    sp = specs[s]
    return O.Subgame(int(sp["board"]), float(sp["pot"]), float(sp["stack"]), int(sp["sizes"]),
                     int(sp["max_raises"]), ranges[s, 0], ranges[s, 1])


def _big_tree_specs(P, n, seed):
    """Specs with many leaves, so that leaves are processed in several groups."""
    specs, ranges = P.random_subgames(n, seed=seed)
    for i in range(n):
        specs[i]["sizes"] = 7
        specs[i]["max_raises"] = 3
        specs[i]["stack"] = specs[i]["pot"] * 4
    return specs, ranges


def _rel(got, want):
    return np.abs(got - want).max() / max(np.abs(want).max(), 1e-30)


@pytest.fixture(scope="module")
def mixed():
    import pokerrust_b200 as P
    specs, ranges = P.random_subgames(5, seed=21)
    bs, br = _big_tree_specs(P, 2, seed=22)
    return np.concatenate([specs, bs]), np.concatenate([ranges, br])


def test_one_iteration_matches_oracle(mixed):
    import pokerrust_b200 as P
    specs, ranges = mixed
    b = P.Batch(specs, ranges)
    b.enable_average()
    rng = np.random.default_rng(3)
    assert max(b.shape(s)[2] for s in range(b.count)) > 16  # several leaf groups
    oracles = []
    for s in range(b.count):
        o = _oracle(specs, ranges, s)
        reg = rng.random((o.edges, 1326), dtype=np.float32) * 0.05
        reg[rng.random(reg.shape) < 0.3] = 0.0
        o.regrets = reg
        b.set_regrets(s, reg)
        oracles.append(o)
    b.iterate(1)
    for s, o in enumerate(oracles):
        o.iterate(1, accumulate=True)
        order = P.card_order()
        live = (order & np.uint64(specs[s]["board"])) == 0
        got, want = b.regrets(s)[:, live], o.regrets[:, live]
        assert _rel(got, want) < 1e-4, (s, _rel(got, want))
        ga, wa = b.average(s)[:, live], o.average[:, live]
        assert _rel(ga, wa) < 1e-5, (s, _rel(ga, wa))
    b.close()


def test_best_response_and_values_fp64(mixed):
    import pokerrust_b200 as P
    specs, ranges = mixed
    b = P.Batch(specs, ranges)
    rng = np.random.default_rng(4)
    oracles = []
    for s in range(b.count):
        o = _oracle(specs, ranges, s)
        reg = rng.random((o.edges, 1326), dtype=np.float32)
        o.regrets = reg
        b.set_regrets(s, reg)
        oracles.append(o)
    b0, b1, ex = b.exploitability(use_average=False, fp64=True)
    v0, s0 = b.root_values(0)
    v1, s1 = b.root_values(1)
    for s, o in enumerate(oracles):
        w0, _ = o.best_response(0)
        w1, _ = o.best_response(1)
        assert abs(b0[s] - w0) <= 1e-9 * abs(w0) and abs(b1[s] - w1) <= 1e-9 * abs(w1)
        assert abs(ex[s] - (w0 + w1) / 2 / o.joint()) <= 1e-9 * abs(ex[s])
        e0, r0 = o.value(0)
        e1, r1 = o.value(1)
        assert _rel(v0[s], r0) < 1e-9 and _rel(v1[s], r1) < 1e-9
        assert abs(s0[s] - e0) <= 1e-9 * max(abs(e0), 1e-12)
        # zero sum: the two players' values cancel
        assert abs(s0[s] + s1[s]) <= 1e-9 * max(abs(s0[s]), 1e-12)
        assert b0[s] >= s0[s] - 1e-9 and b1[s] >= s1[s] - 1e-9
    # single precision best response agrees to f32 rounding
    f0, f1, fex = b.exploitability(use_average=False, fp64=False)
    assert np.all(np.abs(f0 - b0) <= 1e-4 * np.abs(b0) + 1e-6)
    b.close()


def test_launch_configurations_are_bit_identical():
    import pokerrust_b200 as P
    specs, ranges = P.random_subgames(300, seed=5)
    bs, br = _big_tree_specs(P, 40, seed=6)
    specs, ranges = np.concatenate([specs, bs]), np.concatenate([ranges, br])
    results = []
    # the last configuration is the dense one: registers capped for 3 CTAs per SM, 10-leaf groups
    for K, per_sm, order in [(2, 1, 0), (3, 1, 1), (4, 1, 0), (2, 1, 1), (4, 3, 0)]:
        b = P.Batch(specs, ranges)
        b.enable_average()
        for c in range(2):
            b.set_config(c, K, per_sm, order)
        b.iterate(3)
        results.append([b.regrets(s) for s in (0, 17, 299, 320, 339)] +
                       [b.average(s) for s in (5, 330)])
        b.close()
    for r in results[1:]:
        for a, w in zip(r, results[0]):
            assert np.array_equal(a, w)


def test_many_subgames_through_the_queue():
    """More subgames than resident CTAs: every one is solved, and sampled ones match the
    oracle after one iteration from zero regrets."""
    import pokerrust_b200 as P
    specs, ranges = P.random_subgames(700, seed=7)
    b = P.Batch(specs, ranges)
    b.iterate(1)
    for s in (0, 350, 699):
        o = _oracle(specs, ranges, s)
        o.iterate(1)
        order = P.card_order()
        live = (order & np.uint64(specs[s]["board"])) == 0
        assert _rel(b.regrets(s)[:, live], o.regrets[:, live]) < 1e-4
    b.close()


def test_tuner_keeps_state_and_results():
    import pokerrust_b200 as P
    specs, ranges = P.random_subgames(400, seed=8)
    a = P.Batch(specs, ranges)
    b = P.Batch(specs, ranges)
    a.iterate(2)
    b.iterate(2)
    before = [b.regrets(s) for s in (0, 399)]
    ms = b.tune()
    assert np.all(ms >= 0) and ms[0] > 0
    for s, r in zip((0, 399), before):
        assert np.array_equal(b.regrets(s), r)
    a.iterate(2)
    b.iterate(2)
    for s in (0, 123, 399):
        assert np.array_equal(a.regrets(s), b.regrets(s))
    a.close()
    b.close()


def test_convergence_matches_oracle():
    import pokerrust_b200 as P
    specs, ranges = P.random_subgames(3, seed=9)
    b = P.Batch(specs, ranges)
    b.enable_average()
    _, _, e_start = b.exploitability(use_average=False)
    b.iterate(40)
    _, _, e_avg = b.exploitability(use_average=True)
    for s in range(2):
        o = _oracle(specs, ranges, s)
        o.iterate(40, accumulate=True)
        _, _, want = o.exploitability(use_average=True)
        assert abs(e_avg[s] - want) <= 0.02 * abs(want), (s, e_avg[s], want)
    assert np.all(e_avg < 0.2 * e_start)
    b.close()


def test_linear_average():
    """Linear averaging: the first iteration's sums equal the uniform ones (weight 1); the
    second adds twice its terms; and the weighted average converges faster."""
    import pokerrust_b200 as P
    specs, ranges = P.random_subgames(6, seed=13)
    u = P.Batch(specs, ranges)
    u.enable_average()
    w = P.Batch(specs, ranges)
    w.enable_average()
    w.set_linear_average(True)
    u.iterate(1)
    w.iterate(1)
    for s in range(6):
        assert np.array_equal(u.average(s), w.average(s))
    a1 = [u.average(s) for s in range(6)]
    u.iterate(1)
    w.iterate(1)
    for s in range(6):
        # both ran the same regrets; the second iteration's terms are doubled
        assert np.array_equal(u.regrets(s), w.regrets(s))
        du = u.average(s) - a1[s]
        dw = w.average(s) - a1[s]
        assert np.allclose(dw, 2 * du, rtol=1e-5, atol=1e-7)
    u.iterate(58)
    w.iterate(58)
    _, _, eu = u.exploitability(use_average=True)
    _, _, ew = w.exploitability(use_average=True)
    assert np.mean(ew) < np.mean(eu), (np.mean(ew), np.mean(eu))
    u.close()
    w.close()


def test_bulk_rows_match_per_subgame_rows():
    """pr_batch_get_all returns every subgame's rows in batch order, as the per-subgame calls do."""
    import pokerrust_b200 as P
    specs, ranges = P.random_subgames(40, seed=14)
    b = P.Batch(specs, ranges)
    b.enable_average()
    b.iterate(3)
    reg, avg = b.all_rows(0), b.all_rows(1)
    off = 0
    for s in range(b.count):
        e = b.shape(s)[1]
        assert np.array_equal(reg[off:off + e], b.regrets(s))
        assert np.array_equal(avg[off:off + e], b.average(s))
        off += e
    assert off == reg.shape[0]
    b.close()
