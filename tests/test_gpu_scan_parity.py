"""Whole scans and production-size fits against two checkers, under the
reference's own validation rules (hip/compare_out.py:30-52, restated in
ps_claude_opt_b200.compare): equal line counts, dark facet / lambda / beta
compared as printed, worst |dP| / |dRMS| / |dchi^2| inside the validator's
0.1 / 0.1 / 0.5.

Checkers:
  * the reference's OWN GPU application (PeriodSearch, unchanged, built for
    sm_100a against the project's BOINC stub by oracle/refapp/build.sh) run
    on a B200: tests/golden/refapp/, made by tests/golden/make_refapp_golden.py.
    Relative lightcurves only -- the reference's GPU code skips the
    brightness of calibrated curves;
  * the CPU oracle (strict FP64 restatement): tests/golden/oracle/, made by
    tests/golden/make_oracle_golden.py -- including the production object
    WITH its calibrated points.

Inputs (ps_claude_opt_b200.synth.reference_input_text): c1 = BASELINE config
1 object 0 (lmax 3, 288 facets, 1200 relative points, 200 frequencies x 10
poles); c2rel = the production object (lmax 6, 512 facets, 3298 relative
points) on 200 frequencies around its period.

What the measurements behind the bars show (numbers from B200 runs):
  * cut to a few LM iterations, every line agrees exactly as printed with
    the reference's GPU app (c1 and c2rel at 5 iterations; c2rel also at 2
    and 3) and with the oracle (c2rel at 3 and 10, c1 at 5): 200 of 200;
  * at 50 iterations the reference's GPU app is not repeatable on a B200:
    three runs of the same binary on c2rel differ on 43-48 of 200 lines as
    printed, and from about 10 iterations on its lines drift from both this
    engine and the oracle, almost always towards a worse rms (c2rel at 10
    iterations: 108 lines differ, 105 of them worse) -- so 50-iteration
    lines are held to the oracle, and to the reference only by the mean rms
    balance, the reference's second check;
  * this engine is repeatable (two runs identical) and, against the oracle
    at 50 iterations, c2rel agrees on 192 of 200 lines (5 printed poles
    differ, all inside the envelope); c1's 50-iteration fits are unconverged
    and rounding alone moves them: the oracle built with FMA contraction
    differs from the strict oracle on 59 lines (15 outside the envelope,
    another best line); this engine differs on 64 (7 outside, the same best
    frequency).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
ROOT = os.path.dirname(HERE)
sys.path.insert(0, GOLDEN)


def _run(text, tmp_path, tag, program=None, extra=()):
    from ps_claude_opt_b200 import native

    d = tmp_path / tag
    d.mkdir()
    (d / "period_search_in").write_text(text)
    cmd = program or [native.HOST_PROGRAM, "--fresh", *extra]
    r = subprocess.run(cmd, cwd=d, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    return str(d / "period_search_out")


def _compare(test, ref):
    from ps_claude_opt_b200 import compare

    c = compare.compare_files(test, ref)
    print(c.summary())
    return c


@pytest.mark.parametrize("name,stop,quirks", [("c1", 5, 1), ("c1", 5, 0), ("c2rel", 2, 0), ("c2rel", 5, 0)])
def test_lines_equal_the_reference_gpu_app_at_few_iterations(name, stop, quirks, tmp_path):
    """Every printed line equals the reference GPU app's, on both inputs.
    c1 runs with and without PS_QUIRK_PRECALC_CONW (the reference's
    convexity-weight search reads the pointer bits of conw_r,
    start_CUDA.cu:476); at 5 iterations both searches end on the same
    weight."""
    from ps_claude_opt_b200 import synth

    ref = os.path.join(GOLDEN, "refapp", "refapp_sm100a_%s_stop%d.out" % (name, stop))
    got = _run(synth.reference_input_text(name, stop=stop), tmp_path, "%s_%d_%d" % (name, stop, quirks),
               extra=("--quirks", str(quirks)))
    c = _compare(got, ref)
    assert c.line_count_ok and c.identical == c.n_ref_lines == 200


@pytest.mark.parametrize("name,stop", [("c2rel", 3), ("c2rel", 10), ("c1", 5)])
def test_lines_equal_the_oracle_at_few_iterations(name, stop, tmp_path):
    from ps_claude_opt_b200 import synth

    ref = os.path.join(GOLDEN, "oracle", "%s_stop%d_scan.out" % (name, stop))
    got = _run(synth.reference_input_text(name, stop=stop), tmp_path, "%s_%d" % (name, stop))
    c = _compare(got, ref)
    assert c.line_count_ok and c.identical == 200


def test_production_relative_scan_matches_the_oracle(tmp_path):
    """c2rel at 50 iterations: at least 190 of 200 lines identical, at most
    8 printed poles different, every line inside the envelope, the same best
    line (measured: 192 identical, 5 different poles)."""
    from ps_claude_opt_b200 import synth

    got = _run(synth.reference_input_text("c2rel"), tmp_path, "c2rel50")
    c = _compare(got, os.path.join(GOLDEN, "oracle", "c2rel_scan.out"))
    assert c.line_count_ok and c.malformed == 0 and c.nan_test == 0
    assert c.identical >= 190 and c.pole_mismatch <= 8 and c.envelope_violations == 0
    assert c.best_line_same


def test_full_config1_scan_matches_the_oracle(tmp_path):
    """c1 at 50 iterations, where rounding alone moves the unconverged fits
    (the FMA-contracted oracle differs from the strict one on 59 lines, 15
    outside the envelope): no more lines outside the envelope or with a
    different printed pole than that, and the best line at the same
    frequency within the envelope and a degree (measured: 64 / 7)."""
    from ps_claude_opt_b200 import compare, synth

    got = _run(synth.reference_input_text("c1"), tmp_path, "c150")
    ref = os.path.join(GOLDEN, "oracle", "c1_scan.out")
    c = _compare(got, ref)
    assert c.line_count_ok and c.malformed == 0 and c.nan_test == 0
    assert c.envelope_violations <= 15 and c.pole_mismatch <= 70
    assert c.best_line_test == c.best_line_ref
    a = compare.read_lines(got)[c.best_line_test].split()
    b = compare.read_lines(ref)[c.best_line_ref].split()
    assert abs(float(a[0]) - float(b[0])) < 0.1 and abs(float(a[1]) - float(b[1])) < 0.1
    dl = abs((float(a[4]) - float(b[4]) + 180.0) % 360.0 - 180.0)
    assert dl <= 1.0 and abs(float(a[5]) - float(b[5])) <= 1.0


@pytest.mark.parametrize("name,quirks", [("c1", 1), ("c2rel", 0)])
def test_fifty_iteration_scan_no_worse_than_the_reference_gpu_app(name, quirks, tmp_path):
    """Against the reference app's own 50-iteration run (not repeatable, see
    above): the reference's second check, the mean rms balance -- this
    engine's mean rms is not above the reference's -- every line present and
    finite, and the period of every line within the envelope."""
    from ps_claude_opt_b200 import synth

    got = _run(synth.reference_input_text(name), tmp_path, "%s_ref50" % name, extra=("--quirks", str(quirks)))
    c = _compare(got, os.path.join(GOLDEN, "refapp", "refapp_sm100a_%s.out" % name))
    assert c.line_count_ok and c.malformed == 0 and c.nan_test == 0
    assert c.mean_rms_test <= c.mean_rms_ref
    assert c.worst[0] < 0.1


def test_scans_are_repeatable(tmp_path):
    from ps_claude_opt_b200 import synth

    text = synth.reference_input_text("c2rel")
    a = _run(text, tmp_path, "rep_a")
    b = _run(text, tmp_path, "rep_b")
    assert open(a).read() == open(b).read()


def test_reference_main_on_the_b200_engine(tmp_path):
    """The reference's own host program (period_search_BOINC.cpp, unchanged)
    with start_CUDA.cu replaced by ps_claude_opt_b200/host/start_b200.cpp --
    the binding INTEGRATION.md gives -- writes the same file as this
    project's host program."""
    from ps_claude_opt_b200 import synth

    shim = os.path.join(ROOT, "oracle", "_ref", "refapp_b200shim")
    if not os.path.exists(shim):
        pytest.skip("refapp_b200shim not built (oracle/refapp/build.sh needs the reference source tree)")
    text = synth.reference_input_text("c1")
    a = _run(text, tmp_path, "refmain", program=[shim, "--device", "0"])
    b = _run(text, tmp_path, "ours")
    assert open(a).read() == open(b).read()


def test_production_fits_with_calibrated_points_match_the_oracle():
    """50-iteration fits of the production object (lmax 6, 512 facets, 40
    relative curves + 400 calibrated points, ia[1] fitted) at 20 frequencies
    x 10 poles against tests/golden/oracle/c2_fits.npz: every fit inside the
    validator envelope; near the true period (the 10 central frequencies)
    at most 4 fits end at another printed pole."""
    from make_oracle_golden import C2_SEED
    from ps_claude_opt_b200 import native, objects, synth

    gold = np.load(os.path.join(GOLDEN, "oracle", "c2_fits.npz"))
    text, truth = synth.generate(synth.C2, C2_SEED)
    obj = objects.parse_input(text)
    nf, pl = gold["n_freq"], gold["pole"]
    with native.Engine(obj) as eng:
        eng.configure()
        g, gi, gs = eng.fit_items(nf, pl)
    o = gold["res"]
    assert np.all(np.isfinite(g))
    dP = np.abs(g[:, 2] - o[:, 2]) * 24
    dR = np.abs(g[:, 0] - o[:, 0])
    dC = np.abs(g[:, 5] - o[:, 5])
    lam = np.round(g[:, 3]) != np.round(o[:, 3])
    bet = np.round(g[:, 4]) != np.round(o[:, 4])
    print("c2 fits: worst |dP| %.3g h, |dRMS| %.3g, |dchi2| %.3g; printed-pole mismatches %d of %d; "
          "iteration counts equal %d of %d" % (dP.max(), dR.max(), dC.max(), int(np.sum(lam | bet)), len(g),
                                                int(np.sum(gi == gold["niter"])), len(g)))
    assert dP.max() < 0.1 and dR.max() < 0.1 and dC.max() < 0.5
    g_ = obj.grid
    n_true = int(round((g_.freq_start - 1.0 / truth["period_h"]) / g_.freq_step)) + 1
    near = np.abs(nf - n_true) <= 5
    assert np.sum((lam | bet) & near) <= 4
