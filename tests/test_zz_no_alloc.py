"""ps_fit_items_noalloc, the allocation-free entry point, against
ps_gpu_fit_items on the same object and items.

Who needs it: callers that cannot call cudaMalloc -- a host framework whose
caching allocator owns all device memory, or a pipeline that forbids
allocation once it runs (cudaMalloc can synchronise the device).  The entry
point keeps every device byte in one static 64 MiB arena, so it must give
the same fits as the allocating path.  Both run the same kernel and every
fit is computed by one CTA on its own, so the results must agree bit for bit
whatever the grid size; the tests compare with exact equality.  Two calls in
a row check that the arena's leftover contents from the first call (queue
counter, status word, scratch) do not leak into the second.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test.
"""
import numpy as np
import pytest

from conftest import prepared

pytestmark = pytest.mark.gpu


def _reference(obj, nf, pl):
    from ps_claude_opt_b200 import native

    with native.Engine(obj) as eng:
        eng.configure()
        return eng.fit_items(nf, pl)


def test_noalloc_warm_up_reserves_the_arena():
    """n = 0 with every array NULL only loads the module (reserving the
    arena) and succeeds, repeatedly; a later call with work still runs."""
    from ps_claude_opt_b200 import native

    native.reserve_noalloc(0)
    native.reserve_noalloc(0)
    obj = prepared("tiny")
    got, _, _ = native.fit_items_noalloc(obj, np.array([1, 2]), np.array([0, 3]))
    assert np.all(np.isfinite(got[:, 0]))


@pytest.mark.parametrize("kind", ["mixed", "c2"])
def test_noalloc_matches_allocating_entry_point(kind):
    from ps_claude_opt_b200 import native

    obj = prepared(kind)
    nfq = 3 if kind == "mixed" else 2
    nf = np.repeat(np.arange(1, nfq + 1), 10)
    pl = np.tile(np.arange(10), nfq)
    ref, ref_it, ref_st = _reference(obj, nf, pl)
    for _ in range(2):
        got, it, st = native.fit_items_noalloc(obj, nf, pl)
        assert np.array_equal(it, ref_it)
        assert np.array_equal(st, ref_st)
        assert np.array_equal(got, ref)


def test_noalloc_grid_limited_by_arena_scratch():
    """A production-size object: 3983 points x 58 doubles of derivative
    rows make one CTA's scratch about 1.85 MB, so the 64 MiB arena holds
    at most 36 CTAs -- fewer than the 60 items below and than the resident
    maximum of the allocating path (148).  The queue then hands each CTA
    several fits; the results must not change."""
    from ps_claude_opt_b200 import native

    obj = prepared("c2")
    nf = np.repeat(np.arange(1, 7), 10)
    pl = np.tile(np.arange(10), 6)
    ref, ref_it, ref_st = _reference(obj, nf, pl)
    got, it, st = native.fit_items_noalloc(obj, nf, pl)
    assert np.array_equal(it, ref_it)
    assert np.array_equal(st, ref_st)
    assert np.array_equal(got, ref)


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
