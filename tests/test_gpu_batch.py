"""ps_gpu_scan_batch against one object at a time: objects of three sizes
(16, 32 and 56 padded coefficients) searched and scanned in one call give
the same convexity weight and the same lines, bit for bit, as run_object
on each alone -- every fit runs the same kernel whatever runs beside it."""
import numpy as np
import pytest

from conftest import prepared

pytestmark = pytest.mark.gpu


def test_batch_equals_objects_one_by_one():
    from ps_claude_opt_b200 import native

    objs = [prepared("tiny"), prepared("mixed"), prepared("c2"), prepared("tiny", seed=5)]
    got = native.scan_batch(objs, max_freq=4)
    assert len(got) == len(objs)
    for obj, (lines, conw_r) in zip(objs, got):
        ref, ref_conw = native.run_object(obj, max_freq=4)
        assert conw_r == ref_conw
        assert lines.shape == ref.shape == (min(4, obj.grid.n_max), 6)
        assert np.array_equal(lines, ref)


def test_batch_with_repeated_object_and_quirk():
    from ps_claude_opt_b200 import native

    obj = prepared("mixed")
    a, b = native.scan_batch([obj, obj], quirks=native.QUIRK_PRECALC_CONW, max_freq=3)
    ref, ref_conw = native.run_object(obj, quirks=native.QUIRK_PRECALC_CONW, max_freq=3)
    for lines, conw_r in (a, b):
        assert conw_r == ref_conw and np.array_equal(lines, ref)
