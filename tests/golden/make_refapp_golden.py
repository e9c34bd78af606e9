"""Runs the reference's own GPU application and this project's host program
on the same inputs, and keeps the reference's output files as golden
fixtures (tests/golden/refapp/).

The reference app is built (unchanged, against the project's BOINC stub) by
``oracle/refapp/build.sh`` into ``oracle/_ref/refapp_sm100a`` (native sm_100a)
and ``oracle/_ref/refapp_lto100`` (the reference Makefile's own sm_100 entry,
compute_100 LTO-IR + sm_100).  Needs a B200.  Inputs are regenerated from
their seeds (ps_claude_opt_b200.synth.reference_input_text):

  c1     BASELINE config 1 object 0: lmax 3, 288 facets, 20 x 60 relative
         points, 200 trial frequencies around the true period (2000 fits)
  c2rel  the production object (lmax 6, 512 facets, 40 relative curves of
         50-120 points) without its calibrated points -- the reference's GPU
         code skips the brightness of calibrated curves, so it is an oracle
         only for relative data -- on 200 frequencies around the true period

Files written to OUTDIR:
  refapp_<build>_<input>.out         50 LM iterations (the inputs' stop condition)
  refapp_sm100a_<input>_stop<k>.out  the same input cut to k LM iterations
  refapp_sm100a_c2rel_run<r>.out     repeated runs of the same input and binary
  ours_<precision>_<input>.out       this project's host program, for comparison
  summary.json                       wall times, comparisons

    python tests/golden/make_refapp_golden.py OUTDIR
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from ps_claude_opt_b200 import compare, synth  # noqa: E402

input_text = synth.reference_input_text


def run(cmd, text, timeout):
    d = tempfile.mkdtemp(prefix="psrun_")
    try:
        with open(os.path.join(d, "period_search_in"), "w") as f:
            f.write(text)
        t0 = time.perf_counter()
        r = subprocess.run(cmd, cwd=d, capture_output=True, text=True, timeout=timeout)
        wall = time.perf_counter() - t0
        out_path = os.path.join(d, "period_search_out")
        out = open(out_path).read() if os.path.exists(out_path) else ""
        return r.returncode, wall, out, r.stdout[-3000:], r.stderr[-3000:]
    finally:
        shutil.rmtree(d, ignore_errors=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("outdir")
    ap.add_argument("--only", default="c1,c2rel")
    ap.add_argument("--variants", default="sm100a,lto100")
    ap.add_argument("--ours", default="fp64,mixed")
    ap.add_argument("--timeout", type=int, default=1200)
    args = ap.parse_args()
    os.makedirs(args.outdir, exist_ok=True)
    from ps_claude_opt_b200 import native

    progs = {}
    for v in filter(None, args.variants.split(",")):
        progs["refapp_" + v] = [os.path.join(ROOT, "oracle", "_ref", "refapp_" + v), "--device", "0"]
    for p in filter(None, args.ours.split(",")):
        progs["ours_" + p] = [native.HOST_PROGRAM, "--fresh", "--precision", p]
    summary = {}
    for name in filter(None, args.only.split(",")):
        full, one = input_text(name), input_text(name, one_freq=True)
        for prog, cmd in progs.items():
            rc1, w1, _, _, e1 = run(cmd, one, args.timeout)
            rc, w, out, so, se = run(cmd, full, args.timeout)
            base = os.path.join(args.outdir, "%s_%s" % (prog, name))
            with open(base + ".out", "w") as f:
                f.write(out)
            with open(base + ".log", "w") as f:
                f.write("rc %d wall %.3f s (one-frequency run: rc %d, %.3f s)\n--- stdout tail\n%s\n--- stderr tail\n%s\n"
                        "--- one-frequency stderr tail\n%s\n" % (rc, w, rc1, w1, so, se, e1))
            n_lines = len(compare.read_lines(out, is_text=True))
            summary["%s_%s" % (prog, name)] = {
                "rc": rc, "wall_s": w, "rc_one_freq": rc1, "wall_one_freq_s": w1, "lines": n_lines,
                "scan_fits": 10 * max(0, n_lines - 1),
                "scan_fits_per_s": (10 * (n_lines - 1) / (w - w1)) if (rc == 0 and w > w1 and n_lines > 1) else None,
                "nan_lines": sum("nan" in l.lower() for l in out.splitlines()),
            }
            print(prog, name, summary["%s_%s" % (prog, name)], flush=True)
        ref_key = "refapp_sm100a_%s" % name
        ref_path = os.path.join(args.outdir, ref_key + ".out")
        if os.path.exists(ref_path):
            for prog in progs:
                if prog == "refapp_sm100a":
                    continue
                c = compare.compare_files(os.path.join(args.outdir, "%s_%s.out" % (prog, name)), ref_path)
                summary["%s_%s" % (prog, name)]["vs_refapp_sm100a"] = c.as_dict()
                print("  %s vs refapp_sm100a: %s" % (prog, c.summary()), flush=True)
    app = progs.get("refapp_sm100a")
    if app:
        for name, stops in (("c1", (5,)), ("c2rel", (2, 3, 5, 10))):
            for k in stops:
                rc, w, out, _, _ = run(app, input_text(name, stop=k), args.timeout)
                with open(os.path.join(args.outdir, "refapp_sm100a_%s_stop%d.out" % (name, k)), "w") as f:
                    f.write(out)
                summary["refapp_sm100a_%s_stop%d" % (name, k)] = {"rc": rc, "wall_s": w}
        for r in range(2, 5):
            rc, w, out, _, _ = run(app, input_text("c2rel"), args.timeout)
            with open(os.path.join(args.outdir, "refapp_sm100a_c2rel_run%d.out" % r), "w") as f:
                f.write(out)
            summary["refapp_sm100a_c2rel_run%d" % r] = {"rc": rc, "wall_s": w}
    with open(os.path.join(args.outdir, "summary.json"), "w") as f:
        json.dump(summary, f, indent=1)


if __name__ == "__main__":
    main()
