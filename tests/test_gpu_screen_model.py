"""The trained screening network on held-out production-size objects (not in
its training set): fitting about a tenth of the trial frequencies, the
screened scan finds the full scan's best line -- same frequency, same line --
on every object, which an equally large random choice of frequencies (the
method without the network) does not.  The full-scan best lines come from
tests/golden/screen_heldout.json (tests/golden/make_screen_fixture.py)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "screen_heldout.json")


def test_screen_finds_the_full_scan_best_line_with_a_tenth_of_the_fits():
    from ps_claude_opt_b200 import screen, screen_train

    rows = json.load(open(FIXTURE))
    net = screen.load_model()
    net_hits, random_hits = 0, 0
    for row in rows:
        obj, _ = screen_train.make_object(row["seed"])
        assert obj.grid.n_max == row["n_freq"]
        idx, lines, _ = screen.screened_scan(obj, net, row["conw_r"])
        assert len(idx) <= 0.125 * row["n_freq"]
        b = screen.best_line(lines)
        if idx[b] == row["best_freq"]:
            net_hits += 1
            assert np.allclose(lines[b], row["best_line"], rtol=1e-9, atol=1e-9)
        rng = np.random.default_rng(row["seed"])
        rand = rng.choice(row["n_freq"], size=len(idx), replace=False) + 1
        random_hits += int(row["best_freq"] in rand)
    assert net_hits == len(rows)
    assert random_hits < net_hits


def test_screened_scan_in_mixed_precision_finds_the_same_line():
    from ps_claude_opt_b200 import native, screen, screen_train

    row = json.load(open(FIXTURE))[0]
    obj, _ = screen_train.make_object(row["seed"])
    idx, lines, _ = screen.screened_scan(obj, screen.load_model(), row["conw_r"], precision=native.PRECISION_MIXED)
    b = screen.best_line(lines)
    assert idx[b] == row["best_freq"]
    assert abs(lines[b, 0] - row["best_line"][0]) < 1e-4 and abs(lines[b, 1] - row["best_line"][1]) < 1e-4
