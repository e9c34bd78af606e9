"""Writes tests/golden/screen_heldout.json: the full-scan best line of
held-out screening objects (seeds 8_000_000 + i of
ps_claude_opt_b200.screen_train.make_object), read from the npz of full scans
that `python -m ps_claude_opt_b200.screen_train --fulls PATH` writes.

    python tests/golden/make_screen_fixture.py PATH [n_objects]
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    d = np.load(sys.argv[1])
    n = int(sys.argv[2]) if len(sys.argv) > 2 else 3
    rows = []
    for i in range(min(n, len(d["seeds"]))):
        lines = d[f"lines{i}"]
        r = np.where(np.isnan(lines[:, 1]), np.inf, lines[:, 1])
        b = int(np.argmin(r))
        rows.append(dict(seed=int(d["seeds"][i]), n_freq=int(len(lines)), best_freq=b + 1,
                         best_line=[float(v) for v in lines[b]], conw_r=float(d["conw"][i])))
    with open(os.path.join(HERE, "screen_heldout.json"), "w") as f:
        json.dump(rows, f, indent=1)


if __name__ == "__main__":
    main()
