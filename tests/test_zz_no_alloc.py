"""ps_fit_items_noalloc, the allocation-free entry point, against
ps_gpu_fit_items on the same object and items.

Who needs it: callers that cannot call cudaMalloc -- a host framework whose
caching allocator owns all device memory, or a pipeline that forbids
allocation once it runs (cudaMalloc can synchronise the device).  The entry
point keeps every device byte in one static 64 MiB arena, so it must give
the same fits as the allocating path; both run the same kernel, one fit per
CTA, so the results agree to the last bit whatever the grid size.  Two calls
in a row check that the arena's leftover contents from the first call (queue
counter, status word, scratch) do not leak into the second.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test.
"""
import numpy as np
import pytest

from conftest import prepared

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["mixed", "c2"])
def test_noalloc_matches_allocating_entry_point(kind):
    from ps_claude_opt_b200 import native

    obj = prepared(kind)
    nfq = 3 if kind == "mixed" else 2
    nf = np.repeat(np.arange(1, nfq + 1), 10)
    pl = np.tile(np.arange(10), nfq)
    with native.Engine(obj) as eng:
        eng.configure()
        ref, ref_it, ref_st = eng.fit_items(nf, pl)
    for _ in range(2):
        got, it, st = native.fit_items_noalloc(obj, nf, pl)
        assert np.array_equal(it, ref_it)
        assert np.array_equal(st, ref_st)
        assert np.allclose(got, ref, rtol=1e-12, atol=0.0)


def test_noalloc_rejects_bad_items_and_oversized_work():
    from ps_claude_opt_b200 import native

    obj = prepared("tiny")
    with pytest.raises(native.PsError):
        native.fit_items_noalloc(obj, np.array([0]), np.array([0]))   # frequency index < 1
    # 1.1 million items: their items and results alone exceed the 64 MiB arena
    n = 1_100_000
    with pytest.raises(native.PsError, match="64 MiB"):
        native.fit_items_noalloc(obj, np.ones(n, dtype=np.int32), np.zeros(n, dtype=np.int32))
    # the arena is still usable afterwards
    got, _, _ = native.fit_items_noalloc(obj, np.array([1, 2]), np.array([0, 3]))
    assert np.all(np.isfinite(got[:, 0]))
