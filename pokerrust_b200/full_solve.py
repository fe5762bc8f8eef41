"""Full fixed-flop solve with general bets: the plain river traversal against value-network
leaves, on one GPU.

    python -m pokerrust_b200.full_solve --config small --iterations 400 --check 50

Both forms run CFR on the same game: flop and turn streets on the device, and at the end of
the turn either the 48 river subgames of each leaf (plain, the batched river solver) or the
turn-leaf value network (net-leaf; all-in leaves keep their betting-free river subgames).
Every `check` iterations the FP64 exploitability of the average strategies is measured: for
the net-leaf form after re-solving the river subgames under its flop and turn strategies
(`--resolve` iterations), since its strategy stops at the turn. The network is trained first
on turn-leaf states of this game (the leaves' boards, pots and stacks; ranges from random
strategy profiles of the game and random ranges), valued by the batched river solver and
the adjoint. Prints one JSON line: the game's size,
both trajectories (iterations, solver seconds, exploitability in % of the starting pot),
when each first reached the target, and the network's data and training cost.
"""
import argparse
import json
import sys
import time

import numpy as np

from . import interface as P
from . import train_value_net as T
from . import value_data as D

CONFIGS = {
    # 0.75-pot bets and all-in, one bet or raise per street, stacks 10x the pot
    "small": dict(pot=10.0, stack=100.0, fracs=(0.75,), allin=True, raises=1),
    # the large game's sizes (0.33, 0.75, 1.5 pot, all-in) and 50x stacks, one bet or raise per street
    "large": dict(pot=10.0, stack=500.0, fracs=(0.33, 0.75, 1.5), allin=True, raises=1),
    # the same sizes with two bets or raises on the flop and one on the turn: 548,016 river
    # subgames, about 150 GB of solver state, the largest of these games that fits one B200
    # (two raises on both streets: 1.87 M subgames, about 490 GB; three: 8.9 M, 1.6 TB)
    "large2": dict(pot=10.0, stack=500.0, fracs=(0.33, 0.75, 1.5), allin=True, raises=2, turn_raises=1),
}


def seeded_game(config, seed):
    """(spec, ranges): a seeded flop and both ranges U(0,1) with 30 % of the hands zeroed
    (hands on the flop zeroed), each normalised to sum 1."""
    c = CONFIGS[config]
    rng = np.random.default_rng(seed)
    flop = 0
    for card in rng.choice(52, 3, replace=False):
        flop |= 1 << int(card)
    order = P.card_order()
    ranges = rng.random((2, P.HANDS)).astype(np.float32)
    ranges[rng.random(ranges.shape) < 0.3] = 0.0
    ranges[:, (order & np.uint64(flop)) != 0] = 0.0
    ranges /= ranges.sum(axis=1, keepdims=True)
    spec = P.full_spec(flop, c["pot"], c["stack"], flop_fracs=c["fracs"], flop_allin=c["allin"],
                       flop_raises=c["raises"], turn_fracs=c["fracs"], turn_allin=c["allin"],
                       turn_raises=c.get("turn_raises", c["raises"]), river_sizes=D.RIVER_SIZES, river_raises=D.RIVER_RAISES)
    return spec, ranges


def trajectory(game, iterations, check, pot, target_pct, resolve=0, resolve_too=0):
    """CFR in steps of `check` iterations; after each step the FP64 exploitability (solver
    seconds exclude the measurement), and with resolve_too > 0 also the same strategies
    measured with their river subgames re-solved for that many iterations (the measure the
    net-leaf form needs)."""
    points, reached = [], None
    done, solver_s = 0, 0.0
    while done < iterations:
        n = min(check, iterations - done)
        t0 = time.perf_counter()
        game.iterate(n)
        solver_s += time.perf_counter() - t0
        done += n
        t0 = time.perf_counter()
        _, _, ex = game.exploitability(resolve_iterations=resolve)
        pct = 100.0 * ex / pot
        points.append({"iterations": done, "solver_s": solver_s, "pct_pot": pct,
                       "measure_s": time.perf_counter() - t0})
        if resolve_too:
            _, _, ex2 = game.exploitability(resolve_iterations=resolve_too)
            points[-1]["pct_pot_resolved"] = 100.0 * ex2 / pot
        if reached is None and pct <= target_pct:
            reached = {"iterations": done, "solver_s": solver_s}
    return points, reached


def time_to_levels(points, key, levels):
    """Solver seconds at which a trajectory first reaches each exploitability level."""
    out = {}
    for lv in levels:
        hit = next((p for p in points if p[key] <= lv), None)
        out[str(lv)] = None if hit is None else round(hit["solver_s"], 4)
    return out


def leaf_ranges(game, n, rng, per_draw=64):
    """Ranges at the game's leaves with chips behind under random flop and turn strategies:
    each draw sets random regrets (uniform values raised to a random power, 30 % zeroed), runs
    one pass and takes the reach of `per_draw` random leaves, normalised. Returns the leaf
    node ids and ranges [n][2][1326]."""
    nodes = game.batch_leaves(0)
    saved = game.regrets()
    ids, out = [], []
    while len(ids) < n:
        reg = rng.random((game.edges, P.HANDS), dtype=np.float32) ** rng.uniform(1.0, 8.0)
        reg[rng.random(reg.shape) < 0.3] = 0.0
        game.set_regrets(reg.astype(np.float32))
        game.half_iteration(0)
        R = game.reach()
        for v in rng.choice(nodes, min(per_draw, len(nodes)), replace=False):
            m = R[v].astype(np.float64).sum(axis=1)
            if np.all(m > 1e-12) and len(ids) < n:
                ids.append(int(v))
                out.append((R[v] / m[:, None]).astype(np.float32))
    game.reset()
    game.set_regrets(saved)
    return np.array(ids), np.stack(out)


def hybrid_trajectory(game, net, net_iterations, iterations, check, pot, target_pct, zero_sum):
    """Net leaves first, then the plain river traversal as the fallback: `net_iterations`
    CFR iterations with network leaves, then plain iterations (the river subgames start from
    zero regrets; flop and turn regrets and the average sums carry over), up to `iterations`
    in all. Exploitability is the plain game's own FP64 measure of the average strategies,
    whose river part comes from the river subgames; solver seconds include the net phase."""
    game.reset()
    game.set_net(net)
    game.set_zero_sum(zero_sum)
    t0 = time.perf_counter()
    game.iterate(net_iterations)
    solver_s = time.perf_counter() - t0
    game.set_net(None)
    points, reached = [], None
    done = net_iterations
    while done < iterations:
        n = min(check, iterations - done)
        t0 = time.perf_counter()
        game.iterate(n)
        solver_s += time.perf_counter() - t0
        done += n
        t0 = time.perf_counter()
        _, _, ex = game.exploitability()
        pct = 100.0 * ex / pot
        points.append({"iterations": done, "solver_s": solver_s, "pct_pot": pct,
                       "measure_s": time.perf_counter() - t0})
        if reached is None and pct <= target_pct:
            reached = {"iterations": done, "solver_s": solver_s}
    return points, reached


def harvest(game, leaf_ids):
    """The current leaf ranges of the game (the reach of its last CFR pass at the leaves with
    chips behind), normalised per player, for the leaves both players reach."""
    R = game.reach()
    ids, out = [], []
    for v in leaf_ids:
        m = R[v].astype(np.float64).sum(axis=1)
        if np.all(m > 1e-9):
            ids.append(int(v))
            out.append((R[v] / m[:, None]).astype(np.float32))
    return np.array(ids, np.int64), np.stack(out)


def label_states(nodes, ids, ranges, iterations):
    """Training states for leaves `ids` with the given ranges, valued by the river solver."""
    pick = nodes[ids]
    boards = pick["board"].astype(np.uint64)
    pots = pick["stake"].astype(np.float32)
    stacks = pick["stack"].astype(np.float32)
    values, solve_s = river_values(boards, ranges, pots, stacks, iterations)
    scalars = np.stack([pots / 200.0, stacks / (10.0 * pots)], axis=1).astype(np.float32)
    return dict(boards=boards, ranges=np.asarray(ranges, np.float32), scalars=scalars, values=values, pots=pots,
                stacks=stacks, solve_s=solve_s)


def merge(a, b):
    out = {k: np.concatenate([a[k], b[k]]) for k in ("boards", "ranges", "scalars", "values", "pots", "stacks")}
    out["solve_s"] = a["solve_s"] + b["solve_s"]
    return out


def refine(g, net, spec, data, rounds, iterations, check, river_iterations, epochs, seed, zero_sum, held):
    """On-policy refinement: `rounds` times, run the net-leaf solve for `iterations`
    iterations, take the leaf ranges it visits every `check` iterations, value them with the
    river solver, add them to the training data and train on. The network is then trained on
    the ranges that CFR with its own leaf values reaches, not only on random profiles.
    Returns the data, the training-set mask and the per-round counts and seconds."""
    import torch
    nodes, _, _, _ = P.full_tree(spec)
    leaf_ids = g.batch_leaves(0)
    log = []
    for r in range(rounds):
        t0 = time.perf_counter()
        g.reset()
        g.set_net(net)
        g.set_zero_sum(zero_sum)
        ids, rr = [], []
        done = 0
        while done < iterations:
            g.iterate(check)
            done += check
            i, x = harvest(g, leaf_ids)
            ids.append(i)
            rr.append(x)
        g.set_net(None)
        new = label_states(nodes, np.concatenate(ids), np.concatenate(rr), river_iterations)
        data = merge(data, new)
        held = np.concatenate([held, np.zeros(len(new["boards"]), bool)])
        label_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        T.train(net, data, np.flatnonzero(~held), epochs, 256, 1e-3 * 0.5 ** (r + 1), seed + 100 + r)
        torch.cuda.synchronize()
        log.append({"round": r + 1, "states": int(len(new["boards"])), "total": int(len(data["boards"])),
                    "harvest_label_s": label_s, "train_s": time.perf_counter() - t0})
    return data, held, log


def river_specs(boards, ranges, pots, stacks):
    """The 48 river subgames of each turn-leaf state, in card order: specs [n * 48] and
    ranges [n * 48][2][1326] (the state's ranges with the river card's hands zeroed)."""
    m = len(boards)
    order = P.card_order()
    holds = ((order[None, :] >> np.arange(52, dtype=np.uint64)[:, None]) & np.uint64(1)) != 0  # [card][hand]
    b4 = np.asarray(boards, np.uint64)
    off = ((b4[:, None] >> np.arange(52, dtype=np.uint64)[None, :]) & np.uint64(1)) == 0
    river = np.nonzero(off)[1].reshape(m, 48)
    specs = np.zeros(m * 48, P.SPEC_DTYPE)
    specs["board"] = (b4[:, None] | (np.uint64(1) << river.astype(np.uint64))).ravel()
    specs["pot"] = np.repeat(np.asarray(pots, np.float32), 48)
    specs["stack"] = np.repeat(np.asarray(stacks, np.float32), 48)
    specs["sizes"] = D.RIVER_SIZES
    specs["max_raises"] = D.RIVER_RAISES
    rr = np.repeat(np.asarray(ranges, np.float32), 48, axis=0)
    rr *= ~holds[river.ravel()][:, None, :]
    return specs, rr


def river_values(boards, ranges, pots, stacks, iterations, chunk=1024):
    """Leaf values [n][2][1326] (pot-normalised, mean over the 48 rivers) of the states, by
    the batched solver in batches of `chunk` states (48 subgames each), the launch
    configuration tuned on the first batch and reused; and the seconds spent."""
    n = len(boards)
    values = np.zeros((n, 2, P.HANDS), np.float32)
    cfg = None
    t0 = time.perf_counter()
    for s0 in range(0, n, chunk):
        s1 = min(n, s0 + chunk)
        m = s1 - s0
        specs, rr = river_specs(boards[s0:s1], ranges[s0:s1], pots[s0:s1], stacks[s0:s1])
        b = P.Batch(specs, rr)
        b.enable_average()
        b.set_linear_average(True)
        b.iterate(1)
        if cfg is None:
            b.tune()
            cfg = [b.config(c) for c in range(2)]
        else:
            for c in range(2):
                if cfg[c]["count"]:
                    b.set_config(c, cfg[c]["K"], cfg[c]["per_sm"], cfg[c]["order"])
        b.iterate(iterations - 1)
        # each player's counterfactual values at the root: the adjoint's dV/dr0 and -dV/dr1
        c0, _ = b.root_values(0, use_average=True)
        c1, _ = b.root_values(1, use_average=True)
        b.close()
        v = np.stack([c0, c1], axis=1).reshape(m, 48, 2, P.HANDS).mean(axis=1)
        values[s0:s1] = v / pots[s0:s1, None, None]
    return values, time.perf_counter() - t0


def leaf_dataset(spec, n, seed, iterations, game=None):
    """n turn-leaf states of the game, valued over the 48 rivers by the batched solver
    (pot-normalised counterfactual values). Each state is a leaf with chips behind (its 4-card
    board, pot and stack). Its ranges are either the reach of random strategy profiles
    (half the states, when `game` is given; see leaf_ranges) or random (U(0,1), 25 % zeroed,
    board hands zeroed, normalised)."""
    nodes, _, _, _ = P.full_tree(spec)
    rng = np.random.default_rng(seed)
    order = P.card_order()
    n_game = n // 2 if game is not None else 0
    if n_game:
        ids, game_ranges = leaf_ranges(game, n_game, rng)
        pick_game = nodes[ids]
    leaves = nodes[(nodes["kind"] == 3) & (nodes["stack"] > 0)]
    pick = leaves[rng.integers(0, len(leaves), n - n_game)]
    if n_game:
        pick = np.concatenate([pick_game, pick])
    boards = pick["board"].astype(np.uint64)
    pots = pick["stake"].astype(np.float32)
    stacks = pick["stack"].astype(np.float32)
    ranges = np.zeros((n, 2, P.HANDS), np.float32)
    if n_game:
        ranges[:n_game] = game_ranges
    for i in range(n_game, n):
        live = (order & boards[i]) == 0
        for p in range(2):
            r = rng.random(P.HANDS, dtype=np.float32)
            r[rng.random(P.HANDS) < 0.25] = 0.0
            r[~live] = 0.0
            ranges[i, p] = r / r.sum()
    values, solve_s = river_values(boards, ranges, pots, stacks, iterations)
    scalars = np.stack([pots / 200.0, stacks / (10.0 * pots)], axis=1).astype(np.float32)
    return dict(boards=boards, ranges=ranges, scalars=scalars, values=values, pots=pots, stacks=stacks,
                solve_s=solve_s)


def run(config, seed, iterations, check, target_pct, samples, river_iterations, epochs, resolve, net_iterations,
        plain_only=False, refine_rounds=0, refine_iterations=200, zero_sum=False, hybrid=()):
    import torch
    spec, ranges = seeded_game(config, seed)
    pot = CONFIGS[config]["pot"]
    out = {"config": config, "seed": seed, "target_pct_pot": target_pct}
    t0 = time.perf_counter()
    g = P.FullGame(spec, ranges)
    setup_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    g.tune()
    out["game"] = {"nodes": g.nodes, "edges": g.edges, "leaves": g.leaves, "river_subgames": g.bet_subgames,
                   "allin_subgames": g.allin_subgames, "setup_s": setup_s, "tune_s": time.perf_counter() - t0}
    pts, reached = trajectory(g, iterations, check, pot, target_pct, resolve_too=0 if plain_only else resolve)
    out["plain"] = {"trajectory": pts, "reached": reached}
    if plain_only:
        g.close()
        return out
    # the same strategies measured the net-leaf way (rivers re-solved under the flop and
    # turn strategies), to calibrate that measurement
    _, _, ex = g.exploitability(resolve_iterations=resolve)
    out["plain"]["resolved_pct_pot"] = 100.0 * ex / pot
    # the network: data from this game's leaves, then training
    g.reset()
    t0 = time.perf_counter()
    data = leaf_dataset(spec, samples, seed + 1, river_iterations, game=g)
    gen_s = time.perf_counter() - t0
    net = P.ValueNet(rows=256, seed=seed)
    # every tenth state held out, from both halves (game reach and random ranges)
    held = np.arange(samples) % 10 == 9
    t0 = time.perf_counter()
    curve = T.train(net, data, np.flatnonzero(~held), epochs, 256, 1e-3, seed)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    refine_log = []
    if refine_rounds:
        data, held, refine_log = refine(g, net, spec, data, refine_rounds, refine_iterations, 25, river_iterations,
                                        epochs, seed, zero_sum, held)
    te = np.flatnonzero(held)
    pred = T.predict(net, data, te)
    want = data["values"][te]
    game_half = te < samples // 2
    out["network"] = {"samples": samples, "refine": refine_log, "zero_sum": zero_sum, "river_iterations": river_iterations, "generation_s": gen_s,
                      "epochs": epochs, "train_s": train_s, "final_loss": curve[-1] if curve else None,
                      "held_out_mse": {"network_game_ranges": T.mse(pred[game_half], want[game_half]),
                                       "zero_game_ranges": T.mse(0 * want[game_half], want[game_half]),
                                       "network_random_ranges": T.mse(pred[~game_half], want[~game_half]),
                                       "zero_random_ranges": T.mse(0 * want[~game_half], want[~game_half])}}
    g.reset()
    g.set_net(net)
    g.set_zero_sum(zero_sum)
    pts, reached = trajectory(g, net_iterations, check, pot, target_pct, resolve=resolve)
    out["net_leaf"] = {"trajectory": pts, "reached": reached, "resolve_iterations": resolve}
    # both forms under the same measure (rivers re-solved under the flop and turn strategies)
    levels = (4.0, 3.0, 2.5, 2.0, 1.5, 1.0)
    plain_t = time_to_levels(out["plain"]["trajectory"], "pct_pot_resolved", levels)
    net_t = time_to_levels(pts, "pct_pot", levels)
    out["same_measure_seconds_to_pct_pot"] = {
        "plain": plain_t, "net_leaf": net_t,
        "speedup": {k: (round(plain_t[k] / net_t[k], 2) if plain_t[k] and net_t[k] else None) for k in plain_t}}
    g.set_net(None)
    out["hybrid"] = []
    for h in hybrid:
        hp, hr = hybrid_trajectory(g, net, h, iterations, check // 2, pot, target_pct, zero_sum)
        out["hybrid"].append({"net_iterations": h, "trajectory": hp, "reached": hr})
    g.set_net(None)
    g.close()
    net.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="small", choices=sorted(CONFIGS))
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--iterations", type=int, default=400)
    ap.add_argument("--net-iterations", type=int, default=400)
    ap.add_argument("--check", type=int, default=50)
    ap.add_argument("--target", type=float, default=0.5, help="exploitability target, % of the starting pot")
    ap.add_argument("--samples", type=int, default=32768)
    ap.add_argument("--river-iterations", type=int, default=100)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--resolve", type=int, default=200)
    ap.add_argument("--plain-only", action="store_true", help="skip the network and the net-leaf solve")
    ap.add_argument("--refine", type=int, default=0,
                    help="rounds of on-policy refinement (leaf ranges of the net-leaf solve, valued and added)")
    ap.add_argument("--refine-iterations", type=int, default=200)
    ap.add_argument("--zero-sum", action="store_true", help="shift the network's leaf values to zero sum")
    ap.add_argument("--hybrid", default="", help="comma-separated net-leaf iteration counts after which the solve "
                                                 "continues with plain river subgames (e.g. 50,100)")
    a = ap.parse_args(argv)
    print(json.dumps(run(a.config, a.seed, a.iterations, a.check, a.target, a.samples, a.river_iterations,
                         a.epochs, a.resolve, a.net_iterations, a.plain_only, a.refine, a.refine_iterations,
                         a.zero_sum, tuple(int(x) for x in a.hybrid.split(",") if x))), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
