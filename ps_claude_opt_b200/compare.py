"""Line-by-line comparison of two ``period_search_out`` files.

The reference validates a GPU build by comparing its output with a trusted
run of the same input (hip/compare_out.py:30-52): carriage returns are
stripped, the line counts must agree, the dark-facet, lambda and beta fields
(fields 4-6) must match exactly as printed on every line, and the worst
absolute differences of period, rms and chi^2 (fields 1-3) are reported.  The
BOINC validator accepts 0.1 / 0.1 / 0.5 on those three.  A second check the
reference's notes use (OPTIMIZATION_NOTES.md:127-133) is the balance of lines
whose rms is better or worse than the trusted run's: a build that converges
worse shifts it even while every line passes the validator.

This module restates those rules and adds counts that explain a pole
mismatch (how far the printed pole moved, whether the best line moved).

    python -m ps_claude_opt_b200.compare TEST REF
"""
from __future__ import annotations

import dataclasses
import math
import sys

ENVELOPE = (0.1, 0.1, 0.5)   # |dP| [h], |dRMS|, |dchi^2| accepted by the validator


def read_lines(path_or_text: str, is_text: bool = False) -> list[str]:
    if is_text:
        raw = path_or_text
    else:
        with open(path_or_text, "rb") as f:
            raw = f.read().decode()
    return [l.rstrip("\n") for l in raw.replace("\r", "").splitlines() if l.strip()]


def _fields(line: str):
    p = line.split()
    return p if len(p) == 6 else None


def _angle_diff(a: float, b: float) -> float:
    d = abs(a - b) % 360.0
    return min(d, 360.0 - d)


@dataclasses.dataclass
class Comparison:
    n_lines: int = 0
    n_ref_lines: int = 0
    identical: int = 0
    pole_mismatch: int = 0          # lines whose dark / lambda / beta differ as printed
    dark_mismatch: int = 0
    lambda_beta_mismatch: int = 0
    pole_off_gt1: int = 0           # lambda or beta moved by more than 1 degree
    pole_off_gt30: int = 0
    malformed: int = 0
    worst: tuple = (0.0, 0.0, 0.0)  # |dP| [h], |dRMS|, |dchi^2|
    envelope_violations: int = 0    # lines outside 0.1 / 0.1 / 0.5
    rms_better: int = 0             # test rms below the reference's
    rms_worse: int = 0
    mean_rms_test: float = math.nan
    mean_rms_ref: float = math.nan
    best_line_test: int = -1        # 0-based index of the lowest-rms line
    best_line_ref: int = -1
    best_line_same: bool = False    # same index and identical pole fields
    nan_test: int = 0
    nan_ref: int = 0

    @property
    def line_count_ok(self) -> bool:
        return self.n_lines == self.n_ref_lines

    @property
    def passes(self) -> bool:
        """The reference's own bar: equal line counts and no pole/dark difference."""
        return self.line_count_ok and self.pole_mismatch == 0 and self.malformed == 0

    def summary(self) -> str:
        return ("%d lines (ref %d): %d identical; worst |dP|=%.3g |dRMS|=%.3g |dchi2|=%.3g; "
                "pole/dark mismatches %d (dark %d, lambda/beta %d, >1 deg %d, >30 deg %d); "
                "outside 0.1/0.1/0.5: %d; rms better/worse %d/%d (mean %.6f vs %.6f); "
                "best line %d vs %d (%s); nan %d/%d" % (
                    self.n_lines, self.n_ref_lines, self.identical, *self.worst, self.pole_mismatch,
                    self.dark_mismatch, self.lambda_beta_mismatch, self.pole_off_gt1, self.pole_off_gt30,
                    self.envelope_violations, self.rms_better, self.rms_worse, self.mean_rms_test,
                    self.mean_rms_ref, self.best_line_test, self.best_line_ref,
                    "same" if self.best_line_same else "DIFFERENT", self.nan_test, self.nan_ref))

    def as_dict(self) -> dict:
        d = dataclasses.asdict(self)
        d["worst"] = list(self.worst)
        d["passes"] = self.passes
        return d


def _best(lines):
    best, bi = math.inf, -1
    for i, l in enumerate(lines):
        f = _fields(l)
        if f is None:
            continue
        r = float(f[1])
        if r < best:      # NaN never compares below; the first minimum wins
            best, bi = r, i
    return bi


def compare_lines(test: list[str], ref: list[str]) -> Comparison:
    c = Comparison(n_lines=len(test), n_ref_lines=len(ref))
    worst = [0.0, 0.0, 0.0]
    rt, rr = [], []
    for a, b in zip(test, ref):
        fa, fb = _fields(a), _fields(b)
        if fa is not None and "nan" in a.lower():
            c.nan_test += 1
        if fb is not None and "nan" in b.lower():
            c.nan_ref += 1
        if a == b:
            c.identical += 1
        if fa is None or fb is None:
            c.malformed += 1
            continue
        if fa[3:] != fb[3:]:
            c.pole_mismatch += 1
            if fa[3] != fb[3]:
                c.dark_mismatch += 1
            if fa[4:] != fb[4:]:
                c.lambda_beta_mismatch += 1
                off = max(_angle_diff(float(fa[4]), float(fb[4])), abs(float(fa[5]) - float(fb[5])))
                c.pole_off_gt1 += off > 1.0
                c.pole_off_gt30 += off > 30.0
        d = [abs(float(fa[k]) - float(fb[k])) for k in range(3)]
        for k in range(3):
            if not math.isnan(d[k]):
                worst[k] = max(worst[k], d[k])
        if any(not (d[k] <= ENVELOPE[k]) for k in range(3)):
            c.envelope_violations += 1
        ra, rb = float(fa[1]), float(fb[1])
        if ra < rb:
            c.rms_better += 1
        elif ra > rb:
            c.rms_worse += 1
        rt.append(ra)
        rr.append(rb)
    c.worst = tuple(worst)
    if rt:
        c.mean_rms_test = sum(rt) / len(rt)
        c.mean_rms_ref = sum(rr) / len(rr)
    c.best_line_test, c.best_line_ref = _best(test), _best(ref)
    if c.best_line_test == c.best_line_ref and c.best_line_test >= 0:
        ft, fr = _fields(test[c.best_line_test]), _fields(ref[c.best_line_ref])
        c.best_line_same = ft[3:] == fr[3:]
    return c


def compare_files(test_path: str, ref_path: str) -> Comparison:
    return compare_lines(read_lines(test_path), read_lines(ref_path))


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 2:
        print("usage: python -m ps_claude_opt_b200.compare TEST REF", file=sys.stderr)
        return 2
    c = compare_files(argv[0], argv[1])
    print(c.summary())
    if not c.line_count_ok:
        print("LINE COUNT MISMATCH %d vs %d" % (c.n_lines, c.n_ref_lines))
    test, ref = read_lines(argv[0]), read_lines(argv[1])
    shown = 0
    for i, (a, b) in enumerate(zip(test, ref)):
        if a != b and shown < 12:
            fa, fb = _fields(a), _fields(b)
            tag = " POLE-DIFF" if (fa is None or fb is None or fa[3:] != fb[3:]) else ""
            print("  line %d%s:\n    test %s\n    ref  %s" % (i + 1, tag, a, b))
            shown += 1
    return 0 if c.passes else 1


if __name__ == "__main__":
    sys.exit(main())
