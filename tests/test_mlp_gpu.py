"""Turn-leaf value network on the device (pr_mlp_*): forward output and gradients of one
training step against the CPU oracle (oracle/mlp_ref.py, float64 with the device's bfloat16
rounding points), and a short training run that lowers the loss.

Tolerances: both sides round the same values to bfloat16, but a sum that lands on a
rounding boundary can round the other way, so single entries differ by a bfloat16 step
(2^-8 relative); layer gradients are compared by relative Frobenius norm at 2e-2 and the
output at 1e-2 of its scale."""
import numpy as np
import pytest

from oracle import mlp_ref as R

pytestmark = pytest.mark.gpu


def _batch(n, seed):
    rng = np.random.default_rng(seed)
    ranges = rng.random((n, 2, 1326), dtype=np.float32) / 600.0
    boards = np.zeros(n, np.int64)
    for i in range(n):
        for c in rng.choice(52, 4, replace=False):
            boards[i] |= 1 << int(c)
    scalars = rng.random((n, 2), dtype=np.float32)
    targets = (rng.standard_normal((n, 2652)) * 0.1).astype(np.float32)
    return ranges, boards, scalars, targets


def _dev(*arrays):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrays]


def test_gradients_match_oracle():
    import pokerrust_b200 as P
    net = P.ValueNet(rows=256, seed=3)
    ranges, boards, scalars, targets = _batch(16, 5)
    r, b, s, t = _dev(ranges, boards, scalars, targets)
    loss = net.train_step(r, b, s, t, lr=0.0)
    W = [net.layer(l)[0].astype(np.float64) for l in range(5)]
    bias = [net.layer(l)[1].astype(np.float64) for l in range(5)]
    x = R.inputs(ranges.astype(np.float64), boards, scalars.astype(np.float64))
    want_loss, dW, db, y = R.forward_backward(W, bias, x, targets.astype(np.float64))
    assert abs(loss - want_loss) <= 1e-2 * want_loss
    for l in range(5):
        gW, gb = net.grad(l)
        eW = np.linalg.norm(gW - dW[l]) / np.linalg.norm(dW[l])
        eb = np.linalg.norm(gb - db[l]) / max(np.linalg.norm(db[l]), 1e-30)
        assert eW < 2e-2 and eb < 2e-2, (l, eW, eb)
    import torch
    out = torch.zeros((16, 2652), device="cuda")
    net.forward(r, b, s, out)
    got = out.cpu().numpy()
    assert np.abs(got - y).max() <= 1e-2 * np.abs(y).max()
    net.close()


def test_training_lowers_the_loss():
    import pokerrust_b200 as P
    net = P.ValueNet(rows=512, seed=4)
    ranges, boards, scalars, _ = _batch(512, 6)
    # a target that the inputs determine: a fixed random projection of the ranges
    rng = np.random.default_rng(7)
    proj = rng.standard_normal((2652, 64)).astype(np.float32) / 8.0
    mix = rng.standard_normal((64, 2652)).astype(np.float32) / 8.0
    targets = np.tanh(ranges.reshape(512, 2652) * 600.0 @ proj / 40.0) @ mix
    r, b, s, t = _dev(ranges, boards, scalars, targets.astype(np.float32))
    first = net.train_step(r, b, s, t, lr=1e-3)
    for _ in range(60):
        last = net.train_step(r, b, s, t, lr=1e-3)
    assert last < 0.3 * first, (first, last)
    net.close()


def test_persistent_gemms_give_the_same_bits():
    """The network's passes through the persistent GEMM form (128 x 128 tiles, overlapped
    epilogues) give the same loss, gradients and outputs bit for bit: every output element
    is accumulated over K in the same order in both forms."""
    import torch
    import pokerrust_b200 as P
    ranges, boards, scalars, targets = _batch(512, 9)
    r, b, s, t = _dev(ranges, boards, scalars, targets)
    res = []
    for persistent in (False, True):
        net = P.ValueNet(rows=512, seed=5)
        net.set_persistent(persistent)
        losses = [net.train_step(r, b, s, t, lr=1e-3) for _ in range(3)]
        out = torch.zeros((512, 2652), device="cuda")
        net.forward(r, b, s, out)
        res.append((losses, [net.grad(l)[0] for l in range(5)], out.cpu().numpy()))
        net.close()
    assert res[0][0] == res[1][0]
    for a, w in zip(res[0][1], res[1][1]):
        assert np.array_equal(a, w)
    assert np.array_equal(res[0][2], res[1][2])
