"""The oracle itself: pinned to the reference where the reference can run on a
CPU, and checked against the mathematics where it cannot."""
import os

import numpy as np
import pytest

import oracle
from conftest import prepared

REF_LIB = os.path.join(oracle.REF, "libref_setup.so")


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference setup library not built")
@pytest.mark.parametrize("lm,mm,nrows", [(3, 3, 6), (6, 6, 7), (4, 2, 5), (8, 8, 7), (1, 0, 1)])
def test_setup_bit_exact_with_reference_sources(lm, mm, nrows):
    """trifac/areanorm/sphfunc/ellfit restated == the reference's own C files."""
    a = oracle.setup_shape(lm, mm, nrows, 1.2, 1.0, 0.85)
    b = oracle.setup_shape(lm, mm, nrows, 1.2, 1.0, 0.85, reference=True)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_setup_golden_fixture():
    """The committed fixture was produced by the reference's own setup sources
    (tests/golden/make_golden.py); it pins the oracle where the reference tree
    is absent."""
    path = os.path.join(os.path.dirname(__file__), "golden", "setup_ref.npz")
    g = np.load(path)
    for key in g.files:
        if not key.startswith("case"):
            continue
        lm, mm, nrows = (int(v) for v in key.split("_")[1:4])
        which = key.split("_")[4]
        tabs = dict(zip(("normal", "darea", "dsph", "cg"), oracle.setup_shape(lm, mm, nrows, 1.2, 1.0, 0.85)))
        assert np.array_equal(tabs[which], g[key]), key


def test_setup_invariants():
    normal, darea, dsph, cg = oracle.setup_shape(6, 6, 8, 1.05, 1.0, 0.95)
    assert normal.shape == (512, 3) and dsph.shape == (512, 49)
    assert np.allclose(np.linalg.norm(normal, axis=1), 1.0, atol=1e-14)
    # inscribed polyhedron: total area a little below 4 pi, closed surface
    assert 4 * np.pi * 0.97 < darea.sum() < 4 * np.pi
    assert np.abs((darea[:, None] * normal).sum(axis=0)).max() < 1e-12
    assert np.all(dsph[:, 0] == 1.0)
    assert oracle.lib().pso_n_coef(8, 8) == 81


def test_gauss_jordan_solves():
    rng = np.random.default_rng(0)
    for n in (1, 5, 22, 56, 89):
        A = rng.standard_normal((n, n)) + n * np.eye(n)
        b = rng.standard_normal(n)
        rc, x = oracle.gauss_solve(A, b)
        assert rc == 0
        assert np.allclose(x, np.linalg.solve(A, b), rtol=1e-10, atol=1e-12)
    rc, _ = oracle.gauss_solve(np.zeros((3, 3)), np.ones(3))
    assert rc == 2


def test_gauss_jordan_known_answers():
    """The oracle's solve equals the exact rational solve, bit for bit, on
    tie-heavy systems whose elimination is exact (pivot order and tie-break
    included), and on rank-deficient ones its zero-pivot partial solution."""
    import numpy as np

    import solve_cases

    cases = solve_cases.exact_cases(np.random.default_rng(2024))
    assert len(cases) >= 20
    for A, b, (rerr, rx) in cases:
        rc, x = oracle.gauss_solve(A, b)
        assert rc == rerr == 0
        np.testing.assert_array_equal(x, np.array([float(v) for v in rx]))
    cases = solve_cases.rank_deficient_cases(np.random.default_rng(7))
    assert len(cases) >= 8
    for A, b, (rerr, rx) in cases:
        rc, x = oracle.gauss_solve(A, b)
        assert rc == rerr == 2
        np.testing.assert_array_equal(x, np.array([float(v) for v in rx]))


def _step(obj, a, p):
    # the rotation rate multiplies times of ~1000 days: a finite-difference step
    # of 1e-6 already turns the body by ~1e-3 rad and crosses facet terminators
    if p == obj.n_coef + 3:
        return 1e-9 * abs(a[p])
    return 1e-6 * max(1.0, abs(a[p]))


@pytest.mark.parametrize("kind", ["tiny", "mixed"])
def test_eval_beta_is_minus_half_chisq_gradient(kind):
    """beta = -1/2 d chi^2 / d a for every fitted parameter, and alpha is the
    Gauss-Newton matrix J^T W J (symmetric, positive semi-definite)."""
    from ps_claude_opt_b200 import objects

    obj = prepared(kind)
    om = oracle.OracleModel(obj)
    a = objects.initial_params(obj, 2, 5)
    chi, alpha, beta, rows, _ = om.eval(a, with_rows=True)
    fidx = [p for p in range(1, obj.ma + 1) if obj.ia[p]]
    assert np.array_equal(alpha, alpha.T)
    assert np.linalg.eigvalsh(alpha).min() > -1e-9 * np.abs(alpha).max()
    for j, p in enumerate(fidx):
        h = _step(obj, a, p)
        ap, am = a.copy(), a.copy()
        ap[p] += h
        am[p] -= h
        g = (om.eval(ap)[0] - om.eval(am)[0]) / (2 * h)
        assert abs(-0.5 * g - beta[j]) <= 2e-4 * (abs(beta).max() + 1e-12), (p, -0.5 * g, beta[j])


def test_eval_rows_are_brightness_derivatives():
    """Each raw row column p-1 is d ymod / d a_p (calibrated rows, no renorm)."""
    from ps_claude_opt_b200 import objects

    obj = prepared("mixed")
    om = oracle.OracleModel(obj)
    a = objects.initial_params(obj, 1, 2)
    _, _, _, rows, _ = om.eval(a, with_rows=True)
    ma = obj.ma
    for p in (1, 3, obj.n_coef + 1, obj.n_coef + 2, obj.n_coef + 3, obj.n_coef + 4, obj.n_coef + 5,
              obj.n_coef + 6, ma - 1, ma):
        h = _step(obj, a, p)
        ap, am = a.copy(), a.copy()
        ap[p] += h
        am[p] -= h
        yp = om.eval(ap, with_rows=True)[3][:, ma]
        ym = om.eval(am, with_rows=True)[3][:, ma]
        fd = (yp - ym) / (2 * h)
        an = rows[:, p - 1]
        scale = np.abs(an).max() + 1e-12
        # facets crossing the visibility terminator make ymod non-smooth; allow a few outliers
        bad = np.abs(fd - an) > 1e-4 * scale
        assert bad.mean() < 0.02, (p, bad.sum())


def test_oracle_recovers_injected_period():
    """Near the injected period the best line has the true period, a small
    rms and a pole close to the truth (an end-to-end check of the physics)."""
    from ps_claude_opt_b200 import objects, synth

    text, truth = synth.generate(synth.SynthConfig(n_freq=7, n_dense=12, dense_pts=(40, 40)), 1000003)
    import oracle as orc

    obj = objects.parse_input(text, setup_fn=orc.setup_shape)
    om = orc.OracleModel(obj)
    g = obj.grid
    lines = om.scan(g.freq_start, g.freq_end, g.freq_step)
    b = int(np.argmin(lines[:, 1]))
    assert abs(lines[b, 0] - truth["period_h"]) < 2e-3
    assert lines[b, 1] < 0.02
