"""pr_batch_iterate_noalloc, the entry point for callers that may not allocate while they
solve (their GPU memory belongs to their own allocator, or a cudaMalloc or graph build would
stall a shared GPU), against pr_batch_iterate: two calls in a row on identical batches give
the same regrets and average sums, within the batch tests' tolerance of 1e-4 of the largest
entry (the kernels are the same, so in practice they agree bit for bit). Covered: uniform and
linearly weighted average sums, the autotuner's default configuration and the dense one
(K = 4, three CTAs per SM), and the refusal of batches above the 65,536-subgame limit. This
file is collected last, so a run that stops at the first failure has run every other test
first."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _close(x, y):
    return np.abs(x - y).max() <= 1e-4 * max(np.abs(x).max(), 1e-30)


@pytest.mark.parametrize("linear,dense", [(False, False), (True, False), (True, True)])
def test_noalloc_iterations_match(linear, dense):
    import pokerrust_b200 as P
    specs, ranges = P.random_subgames(300, seed=77)
    a = P.Batch(specs, ranges)
    b = P.Batch(specs, ranges)
    for x in (a, b):
        x.enable_average()
        if linear:
            x.set_linear_average(True)
        if dense:
            for c in range(2):
                if x.config(c)["count"]:
                    x.set_config(c, 4, 3, 0)
    for call in range(2):
        a.iterate(2)
        b.iterate_noalloc(2)
        for s in (0, 150, 299):
            assert _close(a.regrets(s), b.regrets(s)), (call, s)
            assert _close(a.average(s), b.average(s)), (call, s)
    a.close()
    b.close()


def test_noalloc_refuses_batches_over_the_limit():
    import pokerrust_b200 as P
    # 65,537 copies of a few small subgames (one all-in bet: 8 edges), about 5 GB on the device
    specs0, ranges0 = P.random_subgames(4, seed=5)
    specs0["sizes"] = 0b100
    specs0["max_raises"] = 1
    n = 65537
    big = P.Batch(np.resize(specs0, n), np.resize(ranges0, (n, 2, P.HANDS)))
    assert P.lib().pr_batch_iterate_noalloc(big.ptr, 1) == 2
    # the batch is still usable through the allocating entry point
    big.iterate(1)
    big.close()
