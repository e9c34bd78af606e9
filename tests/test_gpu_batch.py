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


def test_autotuned_layouts_and_queue_order_change_no_line():
    """The batch's tile-layout autotuner (every layout that fits timed on a
    one-wave sample, the fastest kept) and its largest-object-first queue give
    the same lines as the first layout that fits; the report lists every
    group with the layouts it timed."""
    from ps_claude_opt_b200 import native

    objs = [prepared("tiny"), prepared("c2"), prepared("mixed"), prepared("lmax8rel")]
    native.batch_set_tuning(2)
    tuned = native.scan_batch(objs, max_freq=3)
    rep = native.batch_tuning_report()
    assert {g["ncp"] for g in rep} == {16, 32, 56, 88}
    for g in rep:
        assert g["source"] in ("timed", "only layout that fits")
        assert g["chosen"] in [{"tile_rows": c["tile_rows"], "cstat_smem": c["cstat_smem"]} for c in g["candidates"]]
        if g["source"] == "timed":
            assert all(c["sample_ms"] > 0 for c in g["candidates"])
    native.batch_set_tuning(0)
    try:
        first = native.scan_batch(objs, max_freq=3)
        assert all(g["source"] in ("first that fits", "only layout that fits")
                   for g in native.batch_tuning_report())
    finally:
        native.batch_set_tuning(1)
    for (a, ca), (b, cb) in zip(tuned, first):
        assert ca == cb and np.array_equal(a, b)
