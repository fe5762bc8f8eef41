"""Parity with the reference itself: the reference's CUDA library (src/cuda/interface.cu,
compiled from its sources into oracle/_ref by oracle/Makefile) runs ITERS CFR iterations and
two best-response passes on all 27,783 river roots of the fixed-flop game through its C ABI
(tests/ref_kernel_runner.py, in a fresh process). For a sample of roots each pass is then
replayed on this library from the reference's own regret state ("teacher forcing"): same
regrets, same ranges, one pass; values and the regrets it leaves must agree.

Why replay rather than run both freely: many buckets hold regrets that are f32
cancellation residues (~1e-3 against values of 1e3-1e6); clipping at zero and regret
matching turn those residues into O(1) strategy changes, so two correct f32
implementations that sum in different orders drift apart after a few iterations. The
oracle shows the same drift against itself under a one-ulp input change.

Tolerance: the reference compiles with --use_fast_math and sums with atomics; per root
    max |ours - reference| <= 1e-4 * max |reference|
over each 1326-value vector and each 26 x 256 regret block.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

ITERS = 3
SEED = 99
HERE = os.path.dirname(os.path.abspath(__file__))


def ranges_for(order, boards, rng):
    r = rng.random((len(boards), 1326), dtype=np.float32)
    r[(order[None, :] & boards[:, None]) != 0] = 0.0
    return r


def rel_err_per_row(got, want):
    got = got.reshape(len(got), -1).astype(np.float64)
    want = want.reshape(len(want), -1).astype(np.float64)
    scale = np.abs(want).max(axis=1)
    err = np.abs(got - want).max(axis=1)
    return err / np.maximum(scale, 1e-30)


@pytest.fixture(scope="module")
def reference_run(tmp_path_factory):
    if not os.path.exists(O.REF_SO):
        pytest.skip("oracle/_ref/libpoker_ref.so not built (reference sources absent)")
    out = str(tmp_path_factory.mktemp("ref") / "ref.npz")
    r = subprocess.run([sys.executable, os.path.join(HERE, "ref_kernel_runner.py"), out, str(ITERS), str(SEED)],
                       capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return dict(np.load(out))


@pytest.fixture(scope="module")
def replay(reference_run, flop_tables):
    import pokerrust_b200 as P
    g = O.Game(O.REFERENCE_FLOP)
    boards, bets = g.river_roots()
    sample = reference_run["sample"]
    e, c, a = flop_tables
    tables = P.transfer_flop_eval(O.REFERENCE_FLOP, O.card_order(), O.card_indexes(), e, c, a)
    b = P.Builder()
    for i in sample:
        b.add(int(boards[i]), float(bets[i]))
    out = []
    for k in range(len(reference_run["player"])):
        b.set_regrets(reference_run["before"][k])
        b.upload_all(reference_run["ranges"][k])
        P.evaluate_gpu(b.ptr, tables, int(reference_run["player"][k]), bool(reference_run["exploit"][k]))
        out.append((b.download_all(), b.regrets()))
    b.close()
    P.free_eval(tables)
    return out


@pytest.mark.parametrize("k", range(2 * ITERS + 2))
def test_pass_matches_reference_kernel(reference_run, replay, k):
    values, regrets = replay[k]
    err_v = rel_err_per_row(values, reference_run["values"][k])
    assert err_v.max() <= 1e-4, f"pass {k}: values rel err {err_v.max():.3e} (root {int(np.argmax(err_v))})"
    if reference_run["exploit"][k]:
        assert np.array_equal(regrets, reference_run["before"][k])
    else:
        err_r = rel_err_per_row(regrets, reference_run["after"][k])
        assert err_r.max() <= 1e-4, f"pass {k}: regrets rel err {err_r.max():.3e} (root {int(np.argmax(err_r))})"


def test_reference_kernel_timing_recorded(reference_run):
    # wall time of the reference's synchronous evaluate_cuda (malloc + copies + kernel)
    secs = reference_run["seconds"]
    print(f"\nreference evaluate_cuda: median {np.median(secs) * 1e3:.1f} ms over {len(secs)} calls")
    assert np.all(secs > 0)
