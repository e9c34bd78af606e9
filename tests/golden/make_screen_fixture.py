"""Fixtures of the held-out screening judgement (objects with seeds
8_000_000 + i of ps_claude_opt_b200.screen_train.make_object).

    python tests/golden/make_screen_fixture.py ROWS.jsonl [n_objects]
        writes screen_heldout.json: the plain FP64 full scan's best line of
        the first n_objects (default 10) objects, for the GPU test that
        replays their screened scans;
    python tests/golden/make_screen_fixture.py --fullscans ROWS.jsonl ...
        merges the full-scan fields of the rows (best frequency, printed best
        line, final convexity weight, seconds per object, true period) into
        screen_heldout_fullscans.jsonl, one line per object in seed order, so
        that `screen_train --judge-out OUT --rescreen
        tests/golden/screen_heldout_fullscans.jsonl` re-judges the screened
        scans without scanning the objects again;
    python tests/golden/make_screen_fixture.py --judgement ROWS.jsonl ...
        writes screen_heldout_judgement.jsonl: every object's judgement row
        (the last row of an object across the files wins), in seed order.

ROWS.jsonl are the rows that `python -m ps_claude_opt_b200.screen_train
--judge-out ROWS.jsonl` streams (one JSON line per object: the FP64 full
scan's best frequency and printed line, the convexity weight it ended with,
the screened scans' results) or that `--rescreen` writes.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
FULL_FIELDS = ("seed", "n_freq", "conw_r", "full_best", "full_line", "full_s_per_object", "true_period_h")


def _rows(paths):
    return [json.loads(l) for p in paths for l in open(p) if l.strip()]


def write_fullscans(paths):
    out = os.path.join(HERE, "screen_heldout_fullscans.jsonl")
    by_seed = {}
    if os.path.exists(out):
        for r in _rows([out]):
            by_seed[r["seed"]] = r
    for r in _rows(paths):
        row = {k: r[k] for k in FULL_FIELDS}
        old = by_seed.get(row["seed"])
        if old is not None and (old["full_best"], old["full_line"]) != (row["full_best"], row["full_line"]):
            raise SystemExit("seed %d: full scan differs from the kept one" % row["seed"])
        by_seed.setdefault(row["seed"], row)
    with open(out, "w") as f:
        for seed in sorted(by_seed):
            f.write(json.dumps(by_seed[seed]) + "\n")


def write_judgement(paths):
    by_seed = {r["seed"]: r for r in _rows(paths)}
    with open(os.path.join(HERE, "screen_heldout_judgement.jsonl"), "w") as f:
        for seed in sorted(by_seed):
            f.write(json.dumps(by_seed[seed]) + "\n")


def main():
    if sys.argv[1] == "--fullscans":
        write_fullscans(sys.argv[2:])
        return
    if sys.argv[1] == "--judgement":
        write_judgement(sys.argv[2:])
        return
    rows = _rows([sys.argv[1]])
    n = int(sys.argv[2]) if len(sys.argv) > 2 else 10
    out = [dict(seed=r["seed"], n_freq=r["n_freq"], best_freq=r["full_best"], best_line_printed=r["full_line"],
                conw_r=r["conw_r"]) for r in rows[:n]]
    with open(os.path.join(HERE, "screen_heldout.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
