"""Writes tests/golden/bench_object_fullscan.json: the plain FP64 full scan's
best line of the benchmarked production object (BASELINE config 2 object 0,
seed 2 000 006: 5000 frequencies x 10 poles after the convexity-weight
search), so that bench.py can state whether its screened + mixed-precision
scan of the same object found that line.  Needs a B200 (about 30 s).

    python tests/golden/make_bench_fixture.py [OUT.json]
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from ps_claude_opt_b200 import native, objects, synth  # noqa: E402

SEED = 1000003 * 2


def main():
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "bench_object_fullscan.json")
    text, _ = synth.generate(synth.C2, SEED)
    obj = objects.parse_input(text)
    t0 = time.time()
    lines, conw_r = native.run_object(obj)
    secs = time.time() - t0
    r = np.where(np.isnan(lines[:, 1]), np.inf, lines[:, 1])
    order = np.argsort(r, kind="stable")
    b = int(order[0])
    row = dict(seed=SEED, n_freq=int(len(lines)), conw_r=float(conw_r), best_freq=b + 1,
               best_line=[float(v) for v in lines[b]],
               runner_up=[dict(freq=int(i) + 1, line=[float(v) for v in lines[i]]) for i in order[1:6]],
               formatted_best=native.format_lines(lines[b:b + 1]).strip(), full_scan_wall_s=secs)
    with open(out, "w") as f:
        json.dump(row, f, indent=1)
    print(json.dumps(row))


if __name__ == "__main__":
    main()
