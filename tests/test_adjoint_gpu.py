"""Adjoint of the subgame value (pr_batch_value / pr_batch_value_grad) at average
strategies after CFR: dV/dr0 and dV/dr1 are the players' counterfactual values (checked
against the oracle's double-precision evaluation and against FP64 central finite
differences, h = 1e-3, on 64 seeded coordinates per subgame), and dV/dsigma at the root is
checked through the average sums by the chain rule, also by central differences.

V is bilinear in (r0, r1), so central differences in the ranges are exact up to rounding:
1e-6 relative. The strategy is a ratio of average sums, so its differences carry an O(h^2)
term: 1e-4.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

H = 1e-3


@pytest.fixture(scope="module")
def solved():
    import pokerrust_b200 as P
    specs, ranges = P.random_subgames(16, seed=31)
    b = P.Batch(specs, ranges)
    b.enable_average()
    b.iterate(60)
    yield b, specs, ranges.copy()
    b.close()


def test_gradient_is_the_counterfactual_values(solved):
    import pokerrust_b200 as P
    b, specs, ranges = solved
    V = b.value(use_average=True)
    g0, g1, gs = b.value_grad(use_average=True)
    v0, s0 = b.root_values(0, use_average=True)
    v1, s1 = b.root_values(1, use_average=True)
    for s in range(b.count):
        # bilinear: V = r0 . dV/dr0 = r1 . dV/dr1
        assert abs(V[s] - ranges[s, 0] @ g0[s]) <= 1e-9 * abs(V[s]) + 1e-12
        assert abs(V[s] - ranges[s, 1] @ g1[s]) <= 1e-9 * abs(V[s]) + 1e-12
        assert np.array_equal(g0[s], v0[s]) and np.array_equal(g1[s], -v1[s])
    # against the oracle, from the same average sums
    for s in (0, 7):
        sp = specs[s]
        o = O.Subgame(int(sp["board"]), float(sp["pot"]), float(sp["stack"]), int(sp["sizes"]),
                      int(sp["max_raises"]), ranges[s, 0], ranges[s, 1])
        o.average = b.average(s)
        e0, r0 = o.value(0, use_average=True)
        e1, r1 = o.value(1, use_average=True)
        assert abs(e0 - V[s]) <= 1e-9 * abs(V[s])
        scale = np.abs(r0).max()
        assert np.abs(g0[s] - r0).max() <= 1e-9 * scale
        assert np.abs(g1[s] + r1).max() <= 1e-9 * np.abs(r1).max()
        # the root action values: sum_a sigma_a * child_a = root value at the root's hands
        nch = P.bet_tree(sp["pot"], sp["stack"], sp["sizes"], sp["max_raises"])[0][0]["nchild"]
        assert np.all(gs[s, nch:] == 0)


def test_central_differences_in_the_ranges(solved):
    b, specs, ranges = solved
    rng = np.random.default_rng(64)
    g0, g1, _ = b.value_grad(use_average=True)
    order = None
    import pokerrust_b200 as P
    order = P.card_order()
    coords = []
    for s in range(b.count):
        live = np.flatnonzero((order & np.uint64(specs[s]["board"])) == 0)
        coords.append(rng.choice(live, 64, replace=False))
    coords = np.array(coords)
    for player, g in ((0, g0), (1, g1)):
        for j in range(64):
            vals = []
            for sign in (1.0, -1.0):
                for s in range(b.count):
                    r = ranges[s].copy()
                    r[player, coords[s, j]] += sign * H
                    b.set_ranges(s, r)
                vals.append(b.value(use_average=True))
            fd = (vals[0] - vals[1]) / (2 * H)
            # the perturbed coordinate holds r + h rounded to f32: use the stored steps
            for s in range(b.count):
                h_hi = np.float32(ranges[s, player, coords[s, j]] + np.float32(H)) - ranges[s, player, coords[s, j]]
                h_lo = ranges[s, player, coords[s, j]] - np.float32(ranges[s, player, coords[s, j]] - np.float32(H))
                want = g[s, coords[s, j]]
                got = (vals[0][s] - vals[1][s]) / (float(h_hi) + float(h_lo))
                assert abs(got - want) <= 1e-6 * max(np.abs(g[s]).max(), 1e-12), (player, s, j, got, want)
            del fd
    for s in range(b.count):
        b.set_ranges(s, ranges[s])


def test_root_strategy_gradient_by_chain_rule(solved):
    import pokerrust_b200 as P
    b, specs, ranges = solved
    rng = np.random.default_rng(65)
    _, _, gs = b.value_grad(use_average=True)
    order = P.card_order()
    for s in (0, 3, 9):
        sp = specs[s]
        root = P.bet_tree(sp["pot"], sp["stack"], sp["sizes"], sp["max_raises"])[0][0]
        n = int(root["nchild"])
        e0 = int(root["edge"])
        A = b.average(s)
        live = np.flatnonzero((order & np.uint64(sp["board"])) == 0)
        for h in rng.choice(live, 6, replace=False):
            tot = A[e0:e0 + n, h].astype(np.float64).sum()
            sigma = A[e0:e0 + n, h] / tot
            for a in range(n):
                # dV/dA_a = (dV/dsigma_a - sum_b sigma_b dV/dsigma_b) / sum A
                want = (gs[s, a, h] - (sigma * gs[s, :n, h]).sum()) / tot
                step = np.float32(1e-3 * tot)
                vals = []
                for sign in (1, -1):
                    B = A.copy()
                    B[e0 + a, h] = A[e0 + a, h] + sign * step
                    b.set_average(s, B)
                    vals.append(b.value(use_average=True)[s])
                b.set_average(s, A)
                hi = np.float32(A[e0 + a, h] + step) - A[e0 + a, h]
                lo = A[e0 + a, h] - np.float32(A[e0 + a, h] - step)
                got = (vals[0] - vals[1]) / (float(hi) + float(lo))
                scale = np.abs(gs[s, :n, h]).max() / tot
                assert abs(got - want) <= 1e-4 * max(scale, 1e-30), (s, h, a, got, want)


def test_device_outputs_match_host_outputs(solved):
    """pr_batch_value_grad_device writes the same gradients into device buffers."""
    import torch
    b, specs, ranges = solved
    g0, g1, gs = b.value_grad(use_average=True)
    d0 = torch.zeros((b.count, 1326), dtype=torch.float64, device="cuda")
    d1 = torch.zeros_like(d0)
    ds = torch.zeros((b.count, 8, 1326), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    b.value_grad_device(d0, d1, ds, use_average=True)
    assert np.array_equal(d0.cpu().numpy(), g0)
    assert np.array_equal(d1.cpu().numpy(), g1)
    assert np.array_equal(ds.cpu().numpy(), gs)


def test_adjoint_on_a_sample_of_the_1024_subgame_batch():
    """The adjoint at its stated size: the 1024-subgame batch at its average strategies after
    100 CFR iterations (the batch the bench times), checked on a seeded sample of 64
    subgames: dV/dr against FP64 central differences on 64 seeded coordinates per subgame
    and player (1e-6 of the largest gradient entry), and against the oracle's
    double-precision counterfactual values from the same average sums (1e-9)."""
    import pokerrust_b200 as P
    specs, ranges = P.random_subgames(1024, seed=777)
    b = P.Batch(specs, ranges)
    b.enable_average()
    b.iterate(100)
    rng = np.random.default_rng(1024)
    sample = np.sort(rng.choice(1024, 64, replace=False))
    g0, g1, _ = b.value_grad(use_average=True)
    order = P.card_order()
    coords = np.array([rng.choice(np.flatnonzero((order & np.uint64(specs[s]["board"])) == 0), 64, replace=False)
                       for s in sample])
    for player, g in ((0, g0), (1, g1)):
        for j in range(64):
            vals = []
            for sign in (1.0, -1.0):
                for i, s in enumerate(sample):
                    r = ranges[s].copy()
                    r[player, coords[i, j]] += sign * H
                    b.set_ranges(int(s), r)
                vals.append(b.value(use_average=True))
            for i, s in enumerate(sample):
                x = ranges[s, player, coords[i, j]]
                step = float(np.float32(x + np.float32(H)) - x) + float(x - np.float32(x - np.float32(H)))
                got = (vals[0][s] - vals[1][s]) / step
                want = g[s, coords[i, j]]
                assert abs(got - want) <= 1e-6 * max(np.abs(g[s]).max(), 1e-12), (player, s, j, got, want)
        for s in sample:
            b.set_ranges(int(s), ranges[s])
    for s in sample:
        sp = specs[s]
        o = O.Subgame(int(sp["board"]), float(sp["pot"]), float(sp["stack"]), int(sp["sizes"]),
                      int(sp["max_raises"]), ranges[s, 0], ranges[s, 1])
        o.average = b.average(int(s))
        _, r0 = o.value(0, use_average=True)
        _, r1 = o.value(1, use_average=True)
        assert np.abs(g0[s] - r0).max() <= 1e-9 * np.abs(r0).max()
        assert np.abs(g1[s] + r1).max() <= 1e-9 * np.abs(r1).max()
    b.close()
