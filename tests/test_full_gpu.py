"""Full fixed-flop game with general bets on the device (pr_full_*), against the oracle.

Layered parity: the flop and turn sweeps are checked against the numpy restatement
(oracle/full_game.py) fed with the same leaf values the device used, and sampled leaves'
values are checked against the river oracle (oracle/batch.cpp) on each of their 48 river
subgames with the device's reach as ranges.

Tolerances: reach and values of a CFR pass are f32 on the device and f64 in the oracle:
1e-5 of the largest entry for reach, 1e-4 for values, regrets and average sums (the
reference's 1e-4 bar). Best-response sweeps are f64 on both sides: 1e-10. River leaf values
against the oracle: 1e-4 (CFR pass, f32 leaf arithmetic on the device) and 1e-6 (best
response; the oracle takes the reach rounded to f32 as its ranges). Net leaves: the
kernel's normalised inputs and masses against f64 ones, 1e-6; its leaf values against the
network run on those same inputs, 1e-6 (f32 scaling).
"""
import numpy as np
import pytest

from oracle import full_game as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FLOP = (1 << 3) | (1 << 20) | (1 << 45)
STREETS = [((0.75,), True, 1), ((0.5,), True, 1)]
POT, STACK = 10.0, 100.0
RIVER_SIZES, RIVER_RAISES = 0b011, 2


def _rel(got, want):
    return np.abs(np.asarray(got, np.float64) - want).max() / max(np.abs(want).max(), 1e-30)


def _init(seed):
    rng = np.random.default_rng(seed)
    r = rng.random((2, F.HANDS)).astype(np.float32)
    r[rng.random(r.shape) < 0.3] = 0.0
    r[:, F.blocked(FLOP)] = 0.0
    return (r / r.sum(axis=1, keepdims=True)).astype(np.float32)


@pytest.fixture(scope="module")
def game():
    import pokerrust_b200 as P
    (ff, fa, fr), (tf, ta, tr) = STREETS
    spec = P.full_spec(FLOP, POT, STACK, flop_fracs=ff, flop_allin=fa, flop_raises=fr, turn_fracs=tf,
                       turn_allin=ta, turn_raises=tr, river_sizes=RIVER_SIZES, river_raises=RIVER_RAISES)
    init = _init(5)
    g = P.FullGame(spec, init)
    tree = F.Tree(FLOP, POT, STACK, STREETS)
    yield g, tree, init
    g.close()


def _leaf_oracle(tree, node, R, make):
    """Mean over the 48 river subgames of a leaf of the oracle's root values; make(sub, k)
    sets the subgame's strategy sums and returns its root values."""
    board = tree.board[node]
    acc = np.zeros(F.HANDS)
    k = 0
    for c in range(52):
        if (board >> c) & 1:
            continue
        o = O.Subgame(board | (1 << c), tree.stake[node], tree.stack[node], RIVER_SIZES, RIVER_RAISES,
                      R[node, 0].astype(np.float32), R[node, 1].astype(np.float32))
        acc += make(o, k)
        k += 1
    assert k == 48
    return acc / 48


def test_one_cfr_pass_matches_oracle(game):
    g, tree, init = game
    assert g.nodes == len(tree) and g.edges == tree.edges and g.leaves == len(tree.leaves)
    assert abs(g.joint - F.joint(init, FLOP)) <= 1e-12 * g.joint
    rng = np.random.default_rng(11)
    reg = (rng.random((g.edges, F.HANDS)) * 0.05).astype(np.float32)
    reg[rng.random(reg.shape) < 0.3] = 0.0
    av = (rng.random((g.edges, F.HANDS)) * 0.01).astype(np.float32)
    g.set_regrets(reg)
    g.set_average(av)
    for b in (0, 1):
        bt = g.batch(b)
        assert bt is not None and bt.count == 48 * len(g.batch_leaves(b))
    g.half_iteration(0)
    R = g.reach()
    LV = g.leaf_values()
    V = g.node_values()
    Rw = F.reach(tree, init, reg, False)
    assert _rel(R, Rw) < 1e-5
    Vw, regw, avw = F.sweep_up(tree, Rw, LV.astype(np.float64), 0, reg, False, "cfr", reg, av)
    assert _rel(V, Vw) < 1e-4
    assert _rel(g.regrets(), regw) < 1e-4
    assert _rel(g.average(), avw) < 1e-4
    # river leaves: one with chips behind, one all-in; fresh subgames have zero regrets
    for b in (0, 1):
        node = int(g.batch_leaves(b)[len(g.batch_leaves(b)) // 2])
        want = _leaf_oracle(tree, node, R, lambda o, k: o.value(0, use_average=False)[1])
        assert _rel(LV[tree.leaf_index[node]], want) < 1e-4, b


def test_best_response_matches_oracle(game):
    g, tree, init = game
    g.reset()
    g.iterate(3)
    br0, br1, ex = g.exploitability()
    assert ex > 0 and br0 + br1 > 0
    assert abs(ex - (br0 + br1) / 2 / g.joint) <= 1e-12 * abs(ex)
    # the last sweep was player 1's best response
    av = g.average()
    R = g.reach(fp64=True)
    Rw = F.reach(tree, init.astype(np.float64), av, True)
    assert _rel(R, Rw) < 1e-10
    LV = g.leaf_values(fp64=True)
    Vw, _, _ = F.sweep_up(tree, R, LV, 1, av, True, "br")
    assert _rel(g.node_values(fp64=True), Vw) < 1e-10
    assert abs(br1 - init[1].astype(np.float64) @ Vw[0]) <= 1e-10 * abs(br1)
    # sampled river leaves: best responses to the subgames' average strategies
    for b in (0, 1):
        bt = g.batch(b)
        leaves = g.batch_leaves(b)
        j = len(leaves) // 3
        node = int(leaves[j])

        def br(o, k):
            o.average = bt.average(j * 48 + k)
            return o.best_response(1, use_average=True)[1]

        want = _leaf_oracle(tree, node, R, br)
        assert _rel(LV[tree.leaf_index[node]], want) < 1e-6, b


def test_cfr_converges(game):
    g, tree, init = game
    g.reset()
    _, _, e0 = g.exploitability()
    g.iterate(1)
    _, _, e1 = g.exploitability()
    g.iterate(24)
    _, _, e25 = g.exploitability()
    assert e25 < 0.5 * e1 and e25 < e0, (e0, e1, e25)


def test_net_leaves(game):
    """Net-leaf mode: leaves with chips behind take the network's outputs x pot x the
    opponent's reach mass; all-in leaves keep their river subgames."""
    import torch
    import pokerrust_b200 as P
    g, tree, init = game
    net = P.ValueNet(rows=256, seed=3)
    g.set_net(net)
    try:
        g.half_iteration(1)
        R = g.reach()
        LV = g.leaf_values()
        nodes = g.batch_leaves(0)
        n = len(nodes)
        assert n > 256  # several forward calls
        mass = R[nodes].astype(np.float64).sum(axis=2)
        want_in = R[nodes] / np.where(mass > 0, mass, 1.0)[:, :, None]
        rin, gmass = g.net_inputs()
        assert _rel(gmass, mass) < 1e-6
        assert _rel(rin, want_in) < 1e-6
        boards = np.array([tree.board[v] for v in nodes], np.int64)
        scal = np.array([[tree.stake[v] / 200.0, tree.stack[v] / (10.0 * tree.stake[v])] for v in nodes], np.float32)
        out = np.zeros((n, 2 * F.HANDS), np.float32)
        for j0 in range(0, n, 256):
            j1 = min(n, j0 + 256)
            o = torch.zeros((j1 - j0, 2 * F.HANDS), device="cuda")
            net.forward(torch.from_numpy(rin[j0:j1]).cuda(), torch.from_numpy(boards[j0:j1]).cuda(),
                        torch.from_numpy(scal[j0:j1]).cuda(), o)
            out[j0:j1] = o.cpu().numpy()
        pots = np.array([tree.stake[v] for v in nodes])
        # the network run on the kernel's own inputs: the outputs scaled by pot x mass
        want = out[:, F.HANDS:] * (pots * gmass[:, 0].astype(np.float64))[:, None]
        got = LV[[tree.leaf_index[v] for v in nodes]]
        assert _rel(got, want) < 1e-6
        # the re-solve evaluation runs the river subgames under the average strategies
        b0, b1, ex = g.exploitability(resolve_iterations=2)
        assert np.isfinite(ex) and b0 + b1 >= 0
    finally:
        g.set_net(None)
        net.close()
