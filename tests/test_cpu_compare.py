"""The period_search_out comparator (ps_claude_opt_b200.compare) on small
hand-made files: the reference's rules (hip/compare_out.py:30-52) -- carriage
returns ignored, equal line counts, dark / lambda / beta equal as printed on
every line, worst |dP| / |dRMS| / |dchi^2| -- and the added counts."""
from ps_claude_opt_b200 import compare

REF = ("7.29169748  0.084572  8.582834  1.6  356   79\n"
       "7.29183490  0.085616  8.796037  0.3    0   68\n"
       "7.29218660  0.083506  8.367860  0.0  102    5\n")


def test_identical_files_pass_with_crlf():
    c = compare.compare_lines(compare.read_lines(REF.replace("\n", "\r\n"), is_text=True),
                              compare.read_lines(REF, is_text=True))
    assert c.passes and c.identical == 3 and c.worst == (0.0, 0.0, 0.0)
    assert c.best_line_test == c.best_line_ref == 2 and c.best_line_same


def test_pole_and_dark_mismatches_are_counted():
    test = ("7.29169748  0.084572  8.582834  1.7  356   79\n"      # dark differs
            "7.29183490  0.085600  8.796000  0.3    1   68\n"      # lambda by 1 degree
            "7.29218660  0.083506  8.367860  0.0  282   -5\n")     # pole flipped
    c = compare.compare_lines(compare.read_lines(test, is_text=True), compare.read_lines(REF, is_text=True))
    assert not c.passes
    assert c.pole_mismatch == 3 and c.dark_mismatch == 1 and c.lambda_beta_mismatch == 2
    assert c.pole_off_gt1 == 1 and c.pole_off_gt30 == 1
    assert abs(c.worst[1] - 1.6e-5) < 1e-9 and abs(c.worst[2] - 3.7e-5) < 1e-9
    assert c.envelope_violations == 0
    assert c.rms_better == 1 and c.rms_worse == 0


def test_angle_wraps_at_360():
    test = REF.replace("356   79", "  0   79")
    c = compare.compare_lines(compare.read_lines(test, is_text=True), compare.read_lines(REF, is_text=True))
    assert c.lambda_beta_mismatch == 1 and c.pole_off_gt1 == 1 and c.pole_off_gt30 == 0


def test_envelope_line_count_and_nan():
    test = REF.replace("0.083506  8.367860", "0.283506  nan").splitlines()[1:]
    c = compare.compare_lines(test, compare.read_lines(REF, is_text=True))
    assert not c.line_count_ok and not c.passes
    # line-by-line on the first two lines of each
    assert c.n_lines == 2 and c.nan_test == 1


def test_cli_exit_codes(tmp_path):
    a, b = tmp_path / "a", tmp_path / "b"
    a.write_text(REF)
    b.write_text(REF)
    assert compare.main([str(a), str(b)]) == 0
    b.write_text(REF.replace("356   79", "355   79"))
    assert compare.main([str(a), str(b)]) == 1
