"""CUDA path vs the CPU oracle, through the C ABI (needs a B200).

Tolerances (FP64 throughout):
  * one function evaluation (chi^2, alpha, beta): relative 1e-9 -- both sides
    sum the same terms, only the rounding order differs;
  * a full LM fit: period, rms, chi^2 within the BOINC validator envelope
    0.1 / 0.1 / 0.5 (README.md:90 of the reference), and the same best pole
    (lambda, beta) and dark facet per output line as printed (%4.0f / %4.1f).
"""
import numpy as np
import pytest

from conftest import prepared

pytestmark = pytest.mark.gpu

REL_EVAL = 1e-9


def _close(g, o, rel):
    scale = max(np.abs(o).max(), 1e-300)
    return np.abs(g - o).max() <= rel * scale


@pytest.mark.parametrize("kind", ["tiny", "c1", "mixed", "c2"])
def test_eval_matches_oracle(kind):
    import oracle
    from ps_claude_opt_b200 import native, objects

    obj = prepared(kind)
    om = oracle.OracleModel(obj)
    rng = np.random.default_rng(3)
    with native.Engine(obj) as eng:
        eng.configure()
        for n, pole in [(1, 0), (3, 7), (5, 4)]:
            a = objects.initial_params(obj, n, pole)
            a[1:obj.n_coef + 1] += 0.05 * rng.standard_normal(obj.n_coef)
            chi_g, al_g, be_g, area_g = eng.eval(a)
            chi_o, al_o, be_o, _, area_o = om.eval(a)
            assert abs(chi_g - chi_o) <= REL_EVAL * abs(chi_o)
            assert _close(al_g, al_o, REL_EVAL)
            assert _close(be_g, be_o, REL_EVAL)
            assert abs(area_g - area_o) <= 1e-12 * area_o
            assert np.allclose(al_g, al_g.T, rtol=0, atol=0)


@pytest.mark.parametrize("kind", ["tiny", "mixed"])
def test_fits_match_oracle(kind):
    import oracle
    from ps_claude_opt_b200 import native

    obj = prepared(kind)
    om = oracle.OracleModel(obj)
    nf = np.repeat(np.arange(1, 4), 10)
    pl = np.tile(np.arange(10), 3)
    with native.Engine(obj) as eng:
        eng.configure()
        g, gi, gs = eng.fit_items(nf, pl)
    o, oi, os_ = om.fit_batch(obj.grid.freq_start, obj.grid.freq_step, nf, pl)
    assert np.array_equal(gi, oi)
    assert np.all(np.abs(g[:, 2] - o[:, 2]) * 24 < 0.1)          # period [h]
    assert np.all(np.abs(g[:, 0] - o[:, 0]) < 0.1)                # rms
    assert np.all(np.abs(g[:, 5] - o[:, 5]) < 0.5)                # chi^2
    # the bulk agree far inside the envelope
    rel = np.abs(g[:, 0] - o[:, 0]) / np.abs(o[:, 0])
    assert np.median(rel) < 1e-8


def _lines_equal(lg, lo):
    from ps_claude_opt_b200 import native

    tg = native.format_lines(lg).splitlines()
    to = native.format_lines(lo).splitlines()
    assert len(tg) == len(to)
    for a, b in zip(tg, to):
        fa, fb = a.split(), b.split()
        assert fa[3:] == fb[3:], (a, b)   # dark, lambda, beta exactly as printed
        assert abs(float(fa[0]) - float(fb[0])) < 0.1
        assert abs(float(fa[1]) - float(fb[1])) < 0.1
        assert abs(float(fa[2]) - float(fb[2])) < 0.5


@pytest.mark.parametrize("kind", ["tiny", "c1"])
def test_scan_lines_match_oracle(kind):
    import oracle
    from ps_claude_opt_b200 import native

    obj = prepared(kind)
    om = oracle.OracleModel(obj)
    g = obj.grid
    with native.Engine(obj) as eng:
        lines = eng.start(obj.conw_r, max_lines=6)
    ref = om.scan(g.freq_start, g.freq_end, g.freq_step, max_lines=6)
    ref[0, 3] = obj.conw_r * obj.escl * obj.escl
    _lines_equal(lines, ref)


def test_precalc_matches_oracle():
    import oracle
    from ps_claude_opt_b200 import native

    obj = prepared("tiny")
    om = oracle.OracleModel(obj)
    for quirks in (0, native.QUIRK_PRECALC_CONW):
        with native.Engine(obj) as eng:
            eng.set_quirks(quirks)
            cg, ng = eng.precalc(obj.conw_r)
        co, no = om.precalc(obj.grid.freq_start, obj.grid.freq_step, obj.conw_r, quirks=quirks)
        assert (cg, ng) == (co, no)


def test_status_and_argument_errors():
    from ps_claude_opt_b200 import native

    obj = prepared("tiny")
    with native.Engine(obj) as eng:
        eng.configure()
        with pytest.raises(native.PsError):
            eng.fit_items(np.array([0]), np.array([0]))      # frequency index < 1
        with pytest.raises(native.PsError):
            eng.fit_items(np.array([1]), np.array([10]))     # pole outside 0..9
        g, _, st = eng.fit_items(np.array([1, 2]), np.array([0, 1]))
        assert np.all(np.isfinite(g[:, 0]))
        assert eng.status() & native.DEVSTAT_NAN_CHISQ == 0
