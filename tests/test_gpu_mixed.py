"""The mixed-precision fit (PS_PRECISION_MIXED: FP32 facet sweep with 3xTF32
tensor-core shape derivatives, FP64 everywhere else) against the FP64
oracle and the FP64 engine.  Tolerances are those of a FP32 sweep: one
evaluation within 1e-4 (measured 1e-7 .. 4e-6), three-iteration fits within
1e-4 in rms, period and chi^2 and 1e-3 degrees in the pole, and a scan's best
line at the same frequency and pole as the FP64 scan (period and rms within
1e-4, the bar the FP64 scan meets against the oracle)."""
import numpy as np
import pytest

from conftest import prepared

pytestmark = pytest.mark.gpu
TOL_EVAL = 1e-4


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("kind", ["tiny", "c1", "mixed", "c2"])
def test_mixed_eval_matches_oracle(kind):
    import oracle
    from ps_claude_opt_b200 import native, objects

    obj = prepared(kind)
    om = oracle.OracleModel(obj)
    rng = np.random.default_rng(5)
    with native.Engine(obj) as eng:
        eng.set_precision(native.PRECISION_MIXED)
        eng.configure()
        for it in range(4):
            a = objects.initial_params(obj, 1 + it, (3 * it) % 10)
            ymax = np.abs(obj.dsph.reshape(obj.n_fac, obj.n_coef)).max(axis=0)
            a[1:obj.n_coef + 1] += 0.05 * rng.standard_normal(obj.n_coef) / ymax
            chi_g, al_g, be_g, _ = eng.eval(a)
            chi_o, al_o, be_o, _, _ = om.eval(a)
            assert abs(chi_g - chi_o) <= TOL_EVAL * abs(chi_o)
            assert _rel(al_g, al_o) <= TOL_EVAL
            assert _rel(be_g, be_o) <= TOL_EVAL


@pytest.mark.parametrize("kind", ["tiny", "mixed", "c2"])
def test_mixed_short_fits_match_oracle(kind):
    import oracle
    from ps_claude_opt_b200 import native

    obj = prepared(kind)
    om = oracle.OracleModel(obj)
    om.m.n_iter_max = 3
    nf = np.repeat(np.arange(1, 4), 10)
    pl = np.tile(np.arange(10), 3)
    with native.Engine(obj) as eng:
        eng.set_precision(native.PRECISION_MIXED)
        eng.configure(stop_condition=3.0)
        g, gi, gs = eng.fit_items(nf, pl)
    o, oi, os_ = om.fit_batch(obj.grid.freq_start, obj.grid.freq_step, nf, pl)
    assert np.array_equal(gi, oi)
    for col in (0, 2, 5):                        # rms, period, chi^2
        assert np.allclose(g[:, col], o[:, col], rtol=1e-4, atol=0)
    assert np.allclose(g[:, 3], o[:, 3], rtol=0, atol=1e-3)
    assert np.allclose(g[:, 4], o[:, 4], rtol=0, atol=1e-3)


@pytest.mark.parametrize("kind", ["c1", "c2"])
def test_mixed_scan_finds_the_fp64_best_line(kind):
    from ps_claude_opt_b200 import native

    obj = prepared(kind)
    l64, c64 = native.run_object(obj)
    lmx, cmx = native.run_object(obj, precision=native.PRECISION_MIXED)
    assert cmx == c64
    b64, bmx = int(np.argmin(l64[:, 1])), int(np.argmin(lmx[:, 1]))
    assert bmx == b64
    assert abs(lmx[bmx, 0] - l64[b64, 0]) < 1e-4                 # period [h]
    assert abs(lmx[bmx, 1] - l64[b64, 1]) < 1e-4                 # rms, as the FP64 scan against the oracle
    dl = abs((lmx[bmx, 4] - l64[b64, 4] + 180.0) % 360.0 - 180.0)
    assert dl < 1.0 and abs(lmx[bmx, 5] - l64[b64, 5]) < 1.0
    assert np.all(np.abs(lmx[:, 1] - l64[:, 1]) < 0.1)            # every line in the rms envelope


def test_mixed_rejects_the_largest_bases():
    from ps_claude_opt_b200 import native

    obj = prepared("lmax8")
    with native.Engine(obj) as eng:
        eng.set_precision(native.PRECISION_MIXED)
        with pytest.raises(native.PsError, match="mixed precision"):
            eng.configure()
        eng.set_precision(native.PRECISION_FP64)
        eng.configure()
