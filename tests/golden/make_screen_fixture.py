"""Writes tests/golden/screen_heldout.json: the plain FP64 full scan's best
line of held-out screening objects (seeds 8_000_000 + i of
ps_claude_opt_b200.screen_train.make_object), for the GPU test that replays
their screened scans.

    python tests/golden/make_screen_fixture.py ROWS.jsonl [n_objects]

ROWS.jsonl is the held-out judgement that
`python -m ps_claude_opt_b200.screen_train --judge-out ROWS.jsonl` streams
(one JSON line per object: the FP64 full scan's best frequency and printed
line, the convexity weight it ended with, the screened scan's result).
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    rows = [json.loads(l) for l in open(sys.argv[1]) if l.strip()]
    n = int(sys.argv[2]) if len(sys.argv) > 2 else 10
    out = [dict(seed=r["seed"], n_freq=r["n_freq"], best_freq=r["full_best"], best_line_printed=r["full_line"],
                conw_r=r["conw_r"]) for r in rows[:n]]
    with open(os.path.join(HERE, "screen_heldout.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
