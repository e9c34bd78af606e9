"""The facet sweep's bounding-cone pre-test (facet_cones and the group test
in ps_claude_opt_b200/csrc/fit_kernel.cuh), restated in numpy: for any
observer and Sun directions, a 4-facet group the test rules out has no
facet with mu > 1e-8 and mu0 > 1e-8 -- so the skipped groups are exactly
ones whose terms would all be zero -- while it rules out most of the
groups no facet of which is visible.  The test runs in FP32 on FP32-rounded
axes and directions; its stored margin (1e-5 on the sine) covers that."""
import numpy as np
import pytest

K_TINY = 1e-8


def _cones(normal):
    """Per group of 4 consecutive facets (the last one may be partial):
    FP32 axis and sine of the half-angle + 1e-5, as facet_cones builds them
    (a group wider than a hemisphere, or degenerate, gets sine 2)."""
    nf = len(normal)
    out = []
    for g in range(0, nf, 4):
        n = normal[g:g + 4]
        c = n.sum(0)
        length = np.sqrt((c * c).sum())
        cone = np.array([1.0, 0.0, 0.0, 2.0], dtype=np.float32)
        if length > 1e-3:
            c = c / length
            cmin = min(1.0, float((n @ c).min()))
            if cmin > 0.0:
                sn = np.sqrt(max(0.0, 1.0 - cmin * cmin))
                cone = np.array([c[0], c[1], c[2], sn + 1e-5], dtype=np.float32)
        out.append(cone)
    return np.array(out)


def _passes(cones, e, e0):
    """[points, groups]: the FP32 test c.e > -s and c.e0 > -s."""
    e32, s32 = e.astype(np.float32), e0.astype(np.float32)
    ce = e32 @ cones[:, :3].T
    c0 = s32 @ cones[:, :3].T
    return (ce > -cones[:, 3]) & (c0 > -cones[:, 3])


def _unit(rng, n):
    v = rng.standard_normal((n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


@pytest.mark.parametrize("kind", ["c1", "c2", "lmax8"])
def test_cone_test_never_skips_a_visible_facet(kind):
    from conftest import prepared

    obj = prepared(kind)
    normal = np.asarray(obj.normal, dtype=np.float64).reshape(-1, 3)
    cones = _cones(normal)
    rng = np.random.default_rng(11)
    e = _unit(rng, 4000)
    # Sun directions within 30 degrees of the observer, as the lightcurves' phase angles
    e0 = _unit(rng, 4000) * 0.5 + e
    e0 /= np.linalg.norm(e0, axis=1, keepdims=True)
    # also directions grazing a facet plane, where rounding matters most
    g = rng.integers(0, len(normal), 1000)
    t = _unit(rng, 1000)
    t -= (t * normal[g]).sum(1, keepdims=True) * normal[g]
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    e = np.vstack([e, t + 1e-7 * normal[g]])
    e0 = np.vstack([e0, t + 2e-7 * normal[g]])
    e /= np.linalg.norm(e, axis=1, keepdims=True)
    e0 /= np.linalg.norm(e0, axis=1, keepdims=True)
    vis = ((e @ normal.T) > K_TINY) & ((e0 @ normal.T) > K_TINY)
    ng = len(cones)
    pad = np.zeros((len(e), 4 * ng), dtype=bool)
    pad[:, :len(normal)] = vis
    group_vis = pad.reshape(len(e), ng, 4).any(2)
    passes = _passes(cones, e, e0)
    assert not np.any(group_vis & ~passes), "a group with a visible facet was ruled out"
    # the test is useful: it rules out most invisible groups
    invisible = ~group_vis
    assert (invisible & ~passes).sum() > 0.8 * invisible.sum()


def test_partial_and_degenerate_groups_always_pass():
    # a last group of 2 facets facing opposite ways: wider than a hemisphere
    normal = np.array([[0, 0, 1.0], [1.0, 0, 0], [0, 0, -1.0], [0, 0, 1.0], [0, 1.0, 0], [0, -1.0, 0]])
    cones = _cones(normal)
    assert cones.shape == (2, 4)
    assert cones[1, 3] == 2.0                       # opposite normals: the group always passes
    e = _unit(np.random.default_rng(3), 500)
    assert np.all(_passes(cones, e, e)[:, 1])
