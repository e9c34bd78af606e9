"""Regenerates the oracle's golden outputs under tests/golden/oracle/ (CPU
only; the oracle is the strict FP64 build, identical on every x86-64 host).

  c1_scan.out     the full period_search_out of BASELINE config 1 object 0
                  (200 frequencies x 10 poles after the convexity-weight
                  search), the same input tests/golden/make_refapp_golden.py
                  gives the reference's GPU app
  c2rel_scan.out  the same for the production object without calibrated
                  points, 200 frequencies around the true period
  c1_stop5_scan.out, c2rel_stop{3,10,20}_scan.out
                  the same inputs cut to 5, 3, 10 and 20 LM iterations
  c2_fits.npz     50-iteration fits of the production object (with its 400
                  calibrated points) at 20 frequencies x 10 poles: the 10
                  grid frequencies nearest the true period and 10 spread
                  over the 2-100 h grid; per fit (rms, dark, period,
                  lambda, beta, chi^2), iteration count and status

    python tests/golden/make_oracle_golden.py [c1] [c2rel] [c2fits] [stops]

A few minutes on 8 cores (c1 ~80 s, c2rel ~5 min, c2fits ~1 min).
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import oracle  # noqa: E402
from make_refapp_golden import input_text  # noqa: E402
from ps_claude_opt_b200 import objects, synth  # noqa: E402

OUT = os.path.join(HERE, "oracle")
C2_SEED = 1000003 * 2


def c2_fit_items(obj, truth):
    """The 20 frequencies of c2_fits.npz: 10 nearest the true period, 10 spread."""
    g = obj.grid
    n_true = int(round((g.freq_start - 1.0 / truth["period_h"]) / g.freq_step)) + 1
    near = list(range(n_true - 4, n_true + 6))
    spread = [int(v) for v in np.linspace(1, g.n_max, 12)[1:-1].round()]
    freqs = sorted(set(near) | set(spread))
    nf = np.repeat(freqs, 10).astype(np.int32)
    pl = np.tile(np.arange(10), len(freqs)).astype(np.int32)
    return nf, pl


def scan(name, stop=None):
    with tempfile.TemporaryDirectory() as d:
        inp = os.path.join(d, "period_search_in")
        with open(inp, "w") as f:
            f.write(input_text(name, stop=stop))
        out = os.path.join(OUT, "%s%s_scan.out" % (name, "" if stop is None else "_stop%d" % stop))
        oracle.run_file(inp, out)
    print("wrote", out)


def c2fits():
    text, truth = synth.generate(synth.C2, C2_SEED)
    obj = objects.parse_input(text, setup_fn=oracle.setup_shape)
    nf, pl = c2_fit_items(obj, truth)
    res, niter, status = oracle.OracleModel(obj).fit_batch(obj.grid.freq_start, obj.grid.freq_step, nf, pl)
    path = os.path.join(OUT, "c2_fits.npz")
    np.savez_compressed(path, n_freq=nf, pole=pl, res=res, niter=niter, status=status)
    print("wrote", path)


def main(argv):
    os.makedirs(OUT, exist_ok=True)
    todo = argv or ["c1", "c2rel", "c2fits", "stops"]
    for t in todo:
        if t == "c2fits":
            c2fits()
        elif t == "stops":
            scan("c1", 5)
            for k in (3, 10, 20):
                scan("c2rel", k)
        else:
            scan(t)


if __name__ == "__main__":
    main(sys.argv[1:])
