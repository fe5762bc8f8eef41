"""Solve the fixed-flop limit game with the B200 river solver, like the reference's
`cargo run --release --features GPU` (src/main.rs, src/game.rs): CFR iterations, and every
`--every` iterations the exploitability of the current strategies, here in double
precision. Stops at --target-mbh (default 7.5 mb/h = 0.5% of the 1.5 BB pot at the root)
or after --iterations. Prints one JSON line per checkpoint and a summary line.

    python -m pokerrust_b200.solve --iterations 200 --every 10
"""
import argparse
import json
import sys
import time

from . import interface as P

POT_BB = 1.5  # blinds at the root of the game (src/builder.rs:14)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--flop", type=lambda s: int(s, 0), default=0b111,
                    help="3-card mask, bit i = card i (13*suit + rank); default 2c 3c 4c")
    ap.add_argument("--iterations", type=int, default=100)
    ap.add_argument("--every", type=int, default=10)
    ap.add_argument("--target-mbh", type=float, default=7.5)
    ap.add_argument("--single", action="store_true", help="exploitability in single precision")
    ap.add_argument("--threads", type=int, default=0)
    args = ap.parse_args(argv)

    t_build = time.perf_counter()
    game = P.Game(args.flop, args.threads)
    t0 = time.perf_counter()
    solve_s = 0.0
    reached = None
    it = 0
    while it < args.iterations:
        step = min(args.every, args.iterations - it)
        ts = time.perf_counter()
        game.iterate(step)
        solve_s += time.perf_counter() - ts
        it += step
        te = time.perf_counter()
        _, _, mbh = game.exploitability(fp64=not args.single)
        exp_s = time.perf_counter() - te
        pct = mbh / 1000.0 / POT_BB * 100.0
        print(json.dumps({"iteration": it, "solve_s": round(solve_s, 3), "exploit_s": round(exp_s, 3),
                          "exploitability_mbh": mbh, "pct_of_pot": pct}), flush=True)
        if reached is None and mbh <= args.target_mbh:
            reached = {"iteration": it, "solve_s": solve_s, "wall_s": time.perf_counter() - t0}
            break
    host, dev = game.timings()
    print(json.dumps({"summary": True, "flop": args.flop, "iterations": it, "build_s": t0 - t_build,
                      "target_mbh": args.target_mbh, "reached": reached,
                      "host_traversal_s": host, "device_s": dev}), flush=True)
    game.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
