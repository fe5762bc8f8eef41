"""pr_batch_iterate_noalloc, the entry point for callers that may not allocate while they
solve (their GPU memory belongs to their own allocator, or a cudaMalloc or graph build would
stall a shared GPU), against pr_batch_iterate: two calls in a row on identical batches give
the same regrets and average sums, within the batch tests' tolerance of 1e-4 of the largest
entry (the kernels are the same, so in practice they agree bit for bit). This file is
collected last, so a run that stops at the first failure has run every other test first."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_iterations_match():
    import pokerrust_b200 as P
    specs, ranges = P.random_subgames(300, seed=77)
    a = P.Batch(specs, ranges)
    b = P.Batch(specs, ranges)
    a.enable_average()
    b.enable_average()
    for call in range(2):
        a.iterate(2)
        b.iterate_noalloc(2)
        for s in (0, 150, 299):
            ra, rb = a.regrets(s), b.regrets(s)
            assert np.abs(ra - rb).max() <= 1e-4 * max(np.abs(ra).max(), 1e-30), (call, s)
            aa, ab = a.average(s), b.average(s)
            assert np.abs(aa - ab).max() <= 1e-4 * max(np.abs(aa).max(), 1e-30), (call, s)
    a.close()
    b.close()
