"""Training data for the turn-leaf value network, made by the batched river solver.

A sample is a turn state: a 4-card board, both players' ranges over the 1326 hands (U(0,1)
with 25 % of the hands zeroed, hands on the board zeroed, each range normalised to sum 1),
a pot and a stack. Its 48 river subgames (one per river card, ranges with the river card's
hands zeroed, the same river bet tree) are solved together for `iterations` CFR iterations;
the target is each player's counterfactual value per hand under the average strategies,
taken from the adjoint (dV/dr0 = cfv0, dV/dr1 = -cfv1), averaged over the 48 rivers and
divided by the pot.
"""
import numpy as np

from . import interface as P

RIVER_SIZES = 0b011    # river bets of half pot and pot
RIVER_RAISES = 2


def turn_states(n, seed):
    """Seeded turn states: boards (4-card masks), ranges [n][2][1326], pots, stacks."""
    rng = np.random.default_rng(seed)
    order = P.card_order()
    boards = np.zeros(n, np.uint64)
    ranges = np.zeros((n, 2, 1326), np.float32)
    pots = rng.integers(2, 201, n).astype(np.float32)
    stacks = np.array([rng.integers(int(p), 10 * int(p) + 1) for p in pots], np.float32)
    for i in range(n):
        b = 0
        for c in rng.choice(52, 4, replace=False):
            b |= 1 << int(c)
        boards[i] = b
        live = (order & np.uint64(b)) == 0
        for p in range(2):
            r = rng.random(1326, dtype=np.float32)
            r[rng.random(1326) < 0.25] = 0.0
            r[~live] = 0.0
            ranges[i, p] = r / r.sum()
    return boards, ranges, pots, stacks


def river_values(boards, ranges, pots, stacks, iterations=200, tune=True):
    """Turn-leaf values [n][2][1326] (pot-normalised, averaged over the 48 rivers) and the
    seconds spent in the river solves."""
    import time
    order = P.card_order()
    n = len(boards)
    specs = np.zeros(n * 48, P.SPEC_DTYPE)
    rr = np.zeros((n * 48, 2, 1326), np.float32)
    k = 0
    for i in range(n):
        for c in range(52):
            if (int(boards[i]) >> c) & 1:
                continue
            board5 = int(boards[i]) | (1 << c)
            specs[k] = (board5, pots[i], stacks[i], RIVER_SIZES, RIVER_RAISES)
            hit = (order & np.uint64(1 << c)) != 0
            rr[k] = ranges[i]
            rr[k][:, hit] = 0.0
            k += 1
    t0 = time.perf_counter()
    b = P.Batch(specs, rr)
    b.enable_average()
    if tune:
        b.iterate(1)
        b.tune()
        b.iterate(iterations - 1)
    else:
        b.iterate(iterations)
    g0, g1, _ = b.value_grad(use_average=True)
    dt = time.perf_counter() - t0
    b.close()
    v = np.stack([g0, -g1], axis=1).reshape(n, 48, 2, 1326).mean(axis=1)
    return (v / pots[:, None, None]).astype(np.float32), dt


def make_dataset(n, seed, iterations=200, chunk=256):
    """n samples in chunks of `chunk` turn states (48 river subgames each)."""
    boards, ranges, pots, stacks = turn_states(n, seed)
    values = np.zeros((n, 2, 1326), np.float32)
    solve_s = 0.0
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        values[s:e], dt = river_values(boards[s:e], ranges[s:e], pots[s:e], stacks[s:e], iterations)
        solve_s += dt
    scalars = np.stack([pots / 200.0, stacks / (10.0 * pots)], axis=1).astype(np.float32)
    return dict(boards=boards, ranges=ranges, scalars=scalars, values=values, pots=pots, stacks=stacks,
                solve_s=solve_s)
