"""How much relative error do the 50-iteration LM fits tolerate?  (Test
infrastructure: runs only the oracle.)

The strict oracle built with -DPSO_PERTURB (oracle/_build/libps_oracle_perturb.so)
multiplies every brightness term of an evaluation made during LM iteration
< UNTIL by 1 + EPS u, u uniform in [-1, 1] from a hash of (fit, iteration,
point, term).  This script scans a stretch of the relative-only production
object's grid with the noise off and with each (EPS, UNTIL) given, and
prints the comparator's counts against the noise-free scan.  It measures
what any reduced-precision evaluation (FP32 terms: relative errors near
1e-7) does to the printed lines, independent of the GPU.

    python oracle/perturbation_study.py [first_line n_lines eps_list until_list]
    python oracle/perturbation_study.py 41 40 1e-7,1e-10 50,40,30     # ~10 min on 8 cores
"""
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from ps_claude_opt_b200 import compare, native, objects, synth  # noqa: E402


def main(argv):
    lo, n = (int(argv[0]), int(argv[1])) if len(argv) >= 2 else (41, 40)
    eps_list = argv[2].split(",") if len(argv) >= 3 else ["1e-7", "1e-10"]
    until_list = argv[3].split(",") if len(argv) >= 4 else ["50", "30"]
    text = synth.reference_input_text("c2rel")
    obj = objects.parse_input(text, setup_fn=oracle.setup_shape)
    # the weight the full scan's convexity search ends with (first line's dark column / escl^2)
    cw_line = os.path.join(os.path.dirname(HERE), "tests", "golden", "oracle", "c2rel_scan.out")
    conw = float(open(cw_line).readline().split()[3]) / obj.escl ** 2
    om = oracle.OracleModel(obj, conw_r=conw)
    g = obj.grid
    base = None
    for eps, until in [("0", "1000")] + [(e, u) for e in eps_list for u in until_list]:
        os.environ["PSO_PERTURB_EPS"] = eps
        os.environ["PSO_PERTURB_UNTIL"] = until
        t0 = time.time()
        lines = om.scan(g.freq_start, g.freq_end, g.freq_step, n_start=lo, max_lines=n, perturb=True)
        txt = native.format_lines(lines).splitlines()
        if base is None:
            base = txt
            print("lines %d..%d of c2rel, noise off: %.1f s" % (lo, lo + n - 1, time.time() - t0), flush=True)
            continue
        c = compare.compare_lines(txt, base)
        print("eps %s in iterations < %s: %s" % (eps, until, c.summary()), flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
