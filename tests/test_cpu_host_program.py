"""The C++ host program's reader (period_search --dump-object) against the
Python reader on the same period_search_in text: every prepared array and
scalar bit-identical, plus its error handling.  No GPU: --dump-object stops
before the first CUDA call."""
import os
import subprocess

import numpy as np
import pytest

from conftest import synth_text


def _host():
    from ps_claude_opt_b200 import native

    if not os.path.exists(native.HOST_PROGRAM):
        pytest.fail("host program not built: run __graft_entry__.build()")
    return native.HOST_PROGRAM


def _dump(text, tmp_path):
    p = tmp_path / "period_search_in"
    p.write_text(text)
    r = subprocess.run([_host(), "--dump-object", str(p)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    out = {}
    for line in r.stdout.splitlines():
        t = line.split()
        vals = t[2:]
        assert len(vals) == int(t[1])
        if t[0] in ("ints", "curve_len", "curve_rel", "ia"):
            out[t[0]] = np.array([int(v) for v in vals])
        else:
            out[t[0]] = np.array([float.fromhex(v) for v in vals])
    return out


def _with_weights(text):
    return text.rstrip("\n") + "\n1 0.5\n3 2.5\n"


@pytest.mark.parametrize("kind,weights", [("tiny", False), ("mixed", False), ("mixed", True), ("c2", False),
                                          ("calonly", False), ("ragged", False)])
def test_reader_matches_python(kind, weights, tmp_path):
    from ps_claude_opt_b200 import objects

    text, _ = synth_text(kind, 11)
    if weights:
        text = _with_weights(text)
    d = _dump(text, tmp_path)
    obj = objects.parse_input(text)
    arrays = {"tim": obj.tim, "brightness": obj.brightness, "sig": obj.sig, "sigr2": obj.sigr2,
              "weight": obj.weight, "ee": obj.ee, "ee0": obj.ee0, "normal": obj.normal, "d_area": obj.d_area,
              "d_sphere": obj.dsph, "cg_first": obj.cg_first}
    for name, ref in arrays.items():
        assert np.array_equal(d[name], np.asarray(ref, dtype=np.float64)), name
    scal = [obj.phi0, *obj.par, obj.cl, obj.alamda_start, obj.alamda_incr, obj.alamda_incrr,
            obj.stop_condition, obj.conw_r, obj.escl, None, obj.grid.freq_start, obj.grid.freq_end,
            obj.grid.freq_step]
    for i, v in enumerate(scal):
        if v is not None:
            assert d["scalars"][i] == v, i
    assert list(d["ints"][[0, 1, 2, 3, 5, 6]]) == [obj.n_points, obj.n_curves, obj.n_coef, obj.n_fac,
                                                   obj.grid.n_max, int(obj.onlyrel)]
    assert np.array_equal(d["curve_len"], obj.curve_len)
    assert np.array_equal(d["curve_rel"], obj.curve_rel)
    assert np.array_equal(d["ia"], obj.ia)
    if weights:
        assert set(np.unique(obj.weight)) == {0.5, 1.0, 2.5}


def test_reader_errors(tmp_path):
    text, _ = synth_text("tiny", 11)
    lines = text.splitlines()
    bad = tmp_path / "truncated"
    bad.write_text("\n".join(lines[:20]) + "\n")          # lightcurve data cut short
    r = subprocess.run([_host(), "--dump-object", str(bad)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "bad data point" in r.stderr
    hdr = tmp_path / "header"
    hdr.write_text("\n".join(lines[:4]) + "\nx y\n")       # Laplace degree not a number
    r = subprocess.run([_host(), "--dump-object", str(hdr)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Laplace" in r.stderr
    r = subprocess.run([_host(), "--dump-object", str(tmp_path / "missing")], capture_output=True, text=True,
                       timeout=60)
    assert r.returncode == 1 and "cannot open" in r.stderr
    r = subprocess.run([_host(), "--no-such-flag"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "usage" in r.stderr
