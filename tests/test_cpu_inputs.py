"""The generated inputs the parity tests, the golden files and the bench
share: the reference-run inputs (synth.reference_input_text) and the batched
workload's objects (synth.config3_object)."""
import numpy as np
import pytest


@pytest.mark.parametrize("name", ["c1", "c2rel"])
def test_reference_inputs_variants_share_the_grid(name):
    import oracle
    from ps_claude_opt_b200 import objects, synth

    base = synth.reference_input_text(name)
    assert base.endswith(synth.NEUTRAL_WEIGHT_LINE)
    o = objects.parse_input(base, setup_fn=oracle.setup_shape)
    g = objects.scan_grid(base)
    assert (g.freq_start, g.freq_end, g.freq_step) == (o.grid.freq_start, o.grid.freq_end, o.grid.freq_step)
    assert o.grid.n_max == 200 and o.stop_condition == 50 and all(o.curve_rel)
    one = objects.parse_input(synth.reference_input_text(name, one_freq=True), setup_fn=oracle.setup_shape)
    assert one.grid.n_max == 1 and one.grid.freq_start == o.grid.freq_start
    long_ = objects.parse_input(synth.reference_input_text(name, n_freq=777), setup_fn=oracle.setup_shape)
    assert long_.grid.n_max == 777
    assert long_.grid.freq_start == o.grid.freq_start and long_.grid.freq_step == o.grid.freq_step
    five = synth.reference_input_text(name, stop=5)
    assert five == base.replace("50  stop condition", "5  stop condition")
    assert objects.parse_input(five, setup_fn=oracle.setup_shape).n_iter_max == 5


def test_batched_workload_spans_the_stated_ranges():
    from ps_claude_opt_b200 import synth

    cfgs = [synth.config3_object(i)[0] for i in range(synth.C3_OBJECTS)]
    pts = np.array([c.n_dense * c.dense_pts[0] for c in cfgs])
    assert pts.min() >= 300 and pts.max() <= 19900
    assert all(c.n_dense <= 199 for c in cfgs)            # with the pseudo-curve: the reference's MAX_LC
    assert {c.l_max for c in cfgs} == {4, 6, 8} and {c.nrows for c in cfgs} == {6, 8, 10}
    nf = np.array([c.n_freq for c in cfgs])
    assert nf.min() >= 500 and nf.max() <= 20000
    assert all(c.stop_condition < 1 for c in cfgs)        # converging fits: ragged iteration counts
    a, _ = synth.generate(*synth.config3_object(3))
    b, _ = synth.generate(*synth.config3_object(3))
    assert a == b                                          # seeded
