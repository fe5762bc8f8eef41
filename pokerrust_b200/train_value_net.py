"""Trains the turn-leaf value network on data from the batched river solver and reports what
it gains over the river solves it replaces.

    python -m pokerrust_b200.train_value_net --train 4096 --test 512 --iterations 200 --epochs 40

Prints one JSON line: dataset cost, training curve, held-out error of the network against a
zero predictor, the training-set mean and a short river solve (the same 48 river subgames
solved for only --cheap iterations, which costs more than a network evaluation), and the
time per turn state of the full solve, the short solve and the network.
"""
import argparse
import json
import sys
import time

import numpy as np

from . import interface as P
from . import value_data as D


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def train(net, data, idx, epochs, batch, lr, seed=0, log=None):
    """Minibatch Adam over the samples idx; returns the per-epoch mean losses."""
    import torch
    rng = np.random.default_rng(seed)
    r = _dev(data["ranges"])
    b = _dev(data["boards"].astype(np.int64))
    s = _dev(data["scalars"])
    t = _dev(data["values"].reshape(len(data["boards"]), -1))
    curve = []
    for ep in range(epochs):
        perm = rng.permutation(idx)
        losses = []
        for k in range(0, len(perm) - batch + 1, batch):
            sel = torch.from_numpy(perm[k:k + batch]).cuda()
            losses.append(net.train_step(r[sel].contiguous(), b[sel].contiguous(), s[sel].contiguous(),
                                         t[sel].contiguous(), lr))
        curve.append(float(np.mean(losses)))
        if log:
            log(ep, curve[-1])
    return curve


def predict(net, data, idx):
    import torch
    out = torch.zeros((len(idx), 2 * 1326), device="cuda")
    sel = torch.from_numpy(np.asarray(idx)).cuda()
    for k in range(0, len(idx), net.rows):
        j = sel[k:k + net.rows]
        net.forward(_dev(data["ranges"])[j].contiguous(), _dev(data["boards"].astype(np.int64))[j].contiguous(),
                    _dev(data["scalars"])[j].contiguous(), out[k:k + len(j)])
    return out.cpu().numpy().reshape(len(idx), 2, 1326)


def mse(a, b):
    return float(np.mean((a - b) ** 2))


def run(train_n, test_n, iterations, cheap, epochs, batch, lr, seed):
    import torch
    t0 = time.perf_counter()
    data = D.make_dataset(train_n + test_n, seed, iterations)
    gen_s = time.perf_counter() - t0
    tr = np.arange(train_n)
    te = np.arange(train_n, train_n + test_n)
    net = P.ValueNet(rows=batch, seed=seed)
    t0 = time.perf_counter()
    curve = train(net, data, tr, epochs, batch, lr, seed)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    pred = predict(net, data, te)
    infer_s = time.perf_counter() - t0
    want = data["values"][te]
    mean = data["values"][tr].mean(axis=0, keepdims=True)
    # the method without the network at a small budget: the same rivers, few iterations
    short, short_s = D.river_values(data["boards"][te], data["ranges"][te], data["pots"][te], data["stacks"][te],
                                    cheap, tune=False)
    out = {
        "samples": {"train": train_n, "test": test_n, "river_subgames_per_sample": 48,
                    "solver_iterations": iterations, "generation_s": gen_s, "solve_s": data["solve_s"]},
        "train": {"epochs": epochs, "batch": batch, "lr": lr, "seconds": train_s, "loss_curve": curve},
        "test_mse": {"network": mse(pred, want), "zero": mse(0 * want, want),
                     "train_mean": mse(np.broadcast_to(mean, want.shape), want),
                     f"river_solve_{cheap}_iterations": mse(short, want)},
        "seconds_per_state": {f"river_solve_{iterations}_iterations": data["solve_s"] / (train_n + test_n),
                              f"river_solve_{cheap}_iterations": short_s / test_n,
                              "network": infer_s / test_n},
    }
    net.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=4096)
    ap.add_argument("--test", type=int, default=512)
    ap.add_argument("--iterations", type=int, default=200)
    ap.add_argument("--cheap", type=int, default=4)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=1)
    a = ap.parse_args(argv)
    print(json.dumps(run(a.train, a.test, a.iterations, a.cheap, a.epochs, a.batch, a.lr, a.seed)), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
