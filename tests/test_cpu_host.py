"""Host side of the product without a GPU: the C ABI library loads and exports
every symbol the public header declares; the native shape setup is
bit-identical to the oracle (and therefore to the reference); input parsing
follows the reference's main()."""
import os
import re

import numpy as np
import pytest

import oracle
from conftest import ROOT, synth_text

HEADER = os.path.join(ROOT, "include", "ps_b200.h")


def _declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(ps_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from ps_claude_opt_b200 import native

    L = native.lib()
    names = _declared()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n
    assert set(names) <= set(native.exported_symbols())


def test_struct_layouts_match_the_header(tmp_path):
    """The ctypes mirrors of the ABI structs have the C compiler's layout."""
    import ctypes
    import subprocess

    from ps_claude_opt_b200 import native

    checks = {"ps_object": native.Object, "ps_curves": native.Curves, "ps_shape": native.Shape,
              "ps_line": native.Line, "ps_fit_result": native.FitResult}
    lines = []
    for cname, py in checks.items():
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
        lines.append(f'printf("{cname} sizeof %zu\\n", sizeof({cname}));')
    src = tmp_path / "layout.c"
    src.write_text("#include <stdio.h>\n#include <stddef.h>\n#include \"ps_b200.h\"\nint main(void) {\n" +
                   "\n".join(lines) + "\nreturn 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    for row in filter(None, out):
        cname, fname, val = row.split()
        py = checks[cname]
        want = ctypes.sizeof(py) if fname == "sizeof" else getattr(py, fname).offset
        assert int(val) == want, (cname, fname)


def test_scan_batch_validates_before_touching_the_gpu():
    import ctypes

    from ps_claude_opt_b200 import native

    assert native.scan_batch([]) == []
    o = (native.Object * 1)()          # n_start_from = 0 is invalid
    lines = (native.Line * 1)()
    off = (ctypes.c_int64 * 1)(0)
    nl = (ctypes.c_int32 * 1)(0)
    cw = (ctypes.c_double * 1)(0)
    rc = native.lib().ps_gpu_scan_batch(0, 1, o, 0, lines, off, nl, cw)
    assert rc == 1 and b"n_start_from" in native.lib().ps_last_error()


def test_version_string():
    from ps_claude_opt_b200 import native

    assert b"sm_100a" in native.lib().ps_version()


@pytest.mark.parametrize("lm,mm,nrows", [(3, 3, 6), (6, 6, 8), (8, 8, 10), (4, 3, 5)])
def test_native_setup_matches_oracle_bit_for_bit(lm, mm, nrows):
    from ps_claude_opt_b200 import native

    a = native.setup_shape(lm, mm, nrows, 1.1, 1.0, 0.9)
    b = oracle.setup_shape(lm, mm, nrows, 1.1, 1.0, 0.9)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_native_setup_rejects_bad_sizes():
    from ps_claude_opt_b200 import native

    with pytest.raises(native.PsError):
        native.setup_shape(16, 16, 4, 1, 1, 1)       # lmax > 15
    with pytest.raises(native.PsError):
        native.setup_shape(3, 3, 12, 1, 1, 1)        # 1152 facets > 1024


def test_parse_matches_reference_rules():
    from ps_claude_opt_b200 import objects

    text, truth = synth_text("mixed", 11)
    obj = objects.parse_input(text)
    assert obj.n_points == truth["n_points"]
    assert obj.n_curves == truth["n_curves"]
    assert not obj.onlyrel
    # calibrated data present: the first shape coefficient is fitted, cls never
    assert obj.ia[1] == 1 and obj.ia[obj.ma] == 0
    assert obj.mfit == obj.ma - 1
    # relative-only data: ia[1] = 0
    text1, _ = synth_text("tiny", 11)
    o1 = objects.parse_input(text1)
    assert o1.onlyrel and o1.ia[1] == 0 and o1.mfit == o1.ma - 2
    # sigma = per-curve mean brightness, jd0 = int(min JD), stop 50 -> 50 iterations
    c0 = o1.curve_len[0]
    assert np.all(o1.sig[:c0] == o1.sig[0])
    assert abs(o1.sig[0] - o1.brightness[:c0].mean()) < 1e-12
    assert 0 <= o1.tim.min() < 1
    assert o1.n_iter_max == 50 and o1.iter_diff_max == 0 and o1.n_iter_min == 0
    # frequency grid (period_search_BOINC.cpp:839-841)
    assert o1.grid.n_max == 6


def test_parse_weights_and_epoch():
    from ps_claude_opt_b200 import objects

    text, _ = synth_text("tiny", 11)
    lines = text.splitlines()
    lines[1] = "2455000.0  epoch of zero time t0"
    text2 = "\n".join(lines) + "\n2 0.5\n3 2.0\n"
    obj = objects.parse_input(text2)
    c = np.cumsum(np.r_[0, obj.curve_len])
    assert np.all(obj.weight[c[1]:c[2]] == 0.5)
    assert np.all(obj.weight[c[2]:c[3]] == 2.0)
    assert np.all(obj.weight[:c[1]] == 1.0)
    assert obj.tim.min() > 1          # explicit epoch used, not int(min JD)


def test_format_lines_matches_reference_printf():
    from ps_claude_opt_b200 import native

    s = native.format_lines(np.array([[7.12345678912, 0.0123456, 17.1234567, 3.25, 359.5, -44.5]]))
    assert s == "7.12345679  0.012346  17.123457  3.2  360  -45\n"
