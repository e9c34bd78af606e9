"""Throughput of the LM-fit hot path on the production-size object.

Workload: one seeded synthetic object of the production configuration
(lmax = mmax = 6 -> 49 shape coefficients, 8 triangulation rows -> 512
facets, 40 dense relative lightcurves of 50-120 points plus 400 sparse
calibrated points, periods 2-100 h on the reference's frequency grid, 10
initial poles, stop condition 50 = exactly 50 LM iterations, FP64).  One step
= one batch of (frequency, pole) fits, each run to termination, in one
persistent-kernel launch.  value = fits/s over all ranks; seconds per object
= (frequencies x 10 poles) / value.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

With N > 1 (torchrun) every rank fits its own disjoint frequency range (no
data-path collective); the timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SEED = 1000003 * 2          # production config, object 0
FITS_PER_CTA = 10           # fits per resident CTA in one step
L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2
# DRAM bytes per fit of the fit kernel on this workload: dram__bytes_read.sum +
# dram__bytes_write.sum = 12.41 + 14.32 = 26.73 GB over the 148 fits of one
# ncu capture of `bench.py --profile-case` (profiles/fit_kernel_production_object.md;
# the derivative-row scratch round trip, which grows with the number of fits,
# so a launch's traffic is this times its fits).
NCU_DRAM_BYTES_PER_FIT = 26.73e9 / 148
METRIC = ("LM fits/s of the plain FP64 full scan of the production object on 1 B200 (s/object of it and of "
          "the screened+mixed scan in the same line)")


def workload(setup_fn=None):
    """The production object.  setup_fn builds its shape tables: the
    library's (default) or, for the CPU arms, the oracle's, so that those
    arms load no product code."""
    from ps_claude_opt_b200 import objects, synth

    text, truth = synth.generate(synth.C2, SEED)
    return objects.parse_input(text, setup_fn=setup_fn), truth


def _c3_text(i):
    from ps_claude_opt_b200 import synth

    cfg, seed = synth.config3_object(i)
    return synth.generate(cfg, seed)[0]


def batch_texts(n_obj):
    """Input texts of the batched workload's objects, generated on host
    cores by a spawn pool (started before this process touches a GPU)."""
    import multiprocessing as mp

    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        return pool.map(_c3_text, range(n_obj))


def bench_batch(texts, max_freq, device=0, calls=3):
    """The batched form on the config-3 objects: the convexity-weight search
    and the first `max_freq` frequencies of every object's scan, all objects
    in one ps_gpu_scan_batch call (one persistent launch per coefficient
    group, the scans captured in one CUDA graph), against the same work
    object by object (run_object).  Wall times of whole calls (uploads,
    search rounds and scans; the fastest of `calls` calls), which vary by
    about 20 % from call to call on the host side.  The tile-layout
    autotuner's evidence is its own device-timed samples per group (in
    "tuning"): the first call times every layout that fits, later calls
    take the cached choice.  Lines must agree bit for bit across forms."""
    from ps_claude_opt_b200 import native, objects

    t0 = time.perf_counter()
    objs = [objects.parse_input(t) for t in texts]
    t_setup = time.perf_counter() - t0
    out = {}
    native.batch_set_tuning(2)
    t0 = time.perf_counter()
    first = native.scan_batch(objs, device=device, max_freq=max_freq)
    out["first_call_s"] = time.perf_counter() - t0   # includes timing the candidate layouts
    report = native.batch_tuning_report()
    times = []
    for _ in range(calls):
        t0 = time.perf_counter()
        batch = native.scan_batch(objs, device=device, max_freq=max_freq)
        times.append(time.perf_counter() - t0)
    out["batch_s"] = min(times)
    out["batch_call_s"] = times
    native.batch_set_tuning(0)
    first_fit = native.scan_batch(objs, device=device, max_freq=max_freq)
    first_fit_layouts = [g["chosen"] for g in native.batch_tuning_report()]
    native.batch_set_tuning(1)
    t0 = time.perf_counter()
    one = [native.run_object(o, device=device, max_freq=max_freq) for o in objs]
    out["one_by_one_s"] = time.perf_counter() - t0
    same = all(np.array_equal(a[0], b[0]) and np.array_equal(a[0], c[0]) and np.array_equal(a[0], d[0]) and
               a[1] == b[1] == c[1] == d[1] for a, b, c, d in zip(batch, first, first_fit, one))
    # fits: 100 per convexity-weight round (10 test periods x 10 poles; the
    # weight doubles each round after the first) plus the scan's
    fits = 0
    for o, (lines, cw) in zip(objs, batch):
        rounds = int(round(np.log2(cw / o.conw_r))) + 1
        fits += 100 * rounds + 10 * len(lines)
    pts = [o.n_points for o in objs]
    tuned_layouts = [g["chosen"] for g in report]
    out.update({
        "objects": len(objs), "fits": fits, "fits_per_s": fits / out["batch_s"],
        "s_per_object": out["batch_s"] / len(objs), "host_setup_s": t_setup,
        "batch_vs_one_by_one": out["one_by_one_s"] / out["batch_s"],
        "lines_identical_across_forms": bool(same), "tuning": report,
        "tuned_layouts_equal_first_fit": tuned_layouts == first_fit_layouts,
        "workload": "config 3: %d objects, %d-%d points, lmax %s, %d-%d facets, first %d frequencies of each "
                    "scan after the convexity-weight search, stop condition 0.005 (ragged iterations), FP64" % (
                        len(objs), min(pts), max(pts), sorted({o.l_max for o in objs}),
                        min(o.n_fac for o in objs), max(o.n_fac for o in objs), max_freq),
    })
    return out


def run_program(cmd, text, timeout=1200):
    """Runs a period_search-style program in a fresh directory on
    period_search_in = text; returns (rc, wall seconds, output lines)."""
    import shutil

    d = tempfile.mkdtemp(prefix="psbench_")
    try:
        with open(os.path.join(d, "period_search_in"), "w") as f:
            f.write(text)
        t0 = time.perf_counter()
        r = subprocess.run(cmd, cwd=d, capture_output=True, text=True, timeout=timeout)
        wall = time.perf_counter() - t0
        p = os.path.join(d, "period_search_out")
        lines = [l for l in open(p).read().splitlines() if l.strip()] if os.path.exists(p) else []
        return r.returncode, wall, lines
    finally:
        shutil.rmtree(d, ignore_errors=True)


def program_scan_rate(cmd, name, n_freq=None):
    """Scan fits/s of a period_search-style program on REFERENCE_INPUTS[name]
    (its grid extended to n_freq frequencies): (lines - 1) x 10 fits / (wall
    time of the whole input - wall time of its one-frequency copy), which
    takes start-up, tables and the convexity-weight search out of both."""
    from ps_claude_opt_b200 import synth

    one = synth.reference_input_text(name, one_freq=True)
    run_program(cmd, one)          # first start of the program: page in its libraries
    rc1, w1, _ = run_program(cmd, one)
    rc, w, lines = run_program(cmd, synth.reference_input_text(name, n_freq=n_freq))
    ok = rc == 0 and rc1 == 0 and len(lines) > 1 and w > w1
    fits = 10 * (len(lines) - 1)
    return {"rc": rc, "wall_s": w, "wall_one_freq_s": w1, "lines": len(lines),
            "scan_fits_per_s": fits / (w - w1) if ok else None,
            "s_per_object_scan": (w - w1) if ok else None}, lines


def reference_gpu_leg(grids=(("c1", 2000), ("c2rel", 1000))):
    """The reference's own GPU application (unchanged, sm_100a build) and
    this project's host program on the same inputs and the same B200, timed
    the same way (program_scan_rate; config 1 on 2000 frequencies, the
    relative-only production object on 1000, so the scan outweighs the
    fixed cost), with the comparator's counts of our lines against the
    reference's (whose 50-iteration lines are not repeatable run to run)."""
    from ps_claude_opt_b200 import compare, native

    app = os.path.join(ROOT, "oracle", "_ref", "refapp_sm100a")
    if not os.path.exists(app):
        return {"unavailable": "oracle/_ref/refapp_sm100a not built (oracle/refapp/build.sh)"}
    out = {}
    for name, n_freq in grids:
        ref, ref_lines = program_scan_rate([app, "--device", "0"], name, n_freq)
        ours, our_lines = program_scan_rate([native.HOST_PROGRAM, "--fresh"], name, n_freq)
        c = compare.compare_lines(our_lines, ref_lines)
        out[name] = {"frequencies": n_freq, "fits": 10 * n_freq, "reference_app": ref, "ours_host_program": ours,
                     "speedup_scan": (ours["scan_fits_per_s"] / ref["scan_fits_per_s"])
                     if ours["scan_fits_per_s"] and ref["scan_fits_per_s"] else None,
                     "speedup_whole_program": ref["wall_s"] / ours["wall_s"] if ours["wall_s"] else None,
                     "lines_vs_reference": {"pole_or_dark_mismatches": c.pole_mismatch, "worst": list(c.worst),
                                            "outside_envelope": c.envelope_violations,
                                            "best_line_same": c.best_line_same, "identical": c.identical,
                                            "n_lines": c.n_lines, "mean_rms_ours": c.mean_rms_test,
                                            "mean_rms_reference": c.mean_rms_ref,
                                            "reference_nan_lines": c.nan_ref}}
    return out


def c1_leg(steps, warmup, device, cpu=True):
    """Config 1 (lmax 3, 288 facets, 1200 relative points): the whole
    object's scan, 200 frequencies x 10 poles = 2000 fits, as ONE launch,
    device-timed with CUDA events (the convexity-weight search left out);
    and the oracle on all host cores on a bounded sample of the same fits."""
    import torch

    from ps_claude_opt_b200 import native, objects, synth

    text, _ = synth.generate(synth.C1, 1000003)
    obj = objects.parse_input(text)
    n = obj.grid.n_max * 10
    items = np.zeros((n, 2), dtype=np.int32)
    items[:, 0] = 1 + np.arange(n) // 10
    items[:, 1] = np.arange(n) % 10
    eng = native.Engine(obj, device=device)
    eng.configure(conw_r=obj.conw_r)
    stream = torch.cuda.ExternalStream(eng.stream)
    d_items = torch.from_numpy(items).cuda()
    d_out = torch.empty(n * ctypes.sizeof(native.FitResult), dtype=torch.uint8, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    ms = []
    with torch.cuda.stream(stream):
        for s in range(warmup + steps):
            flush.fill_(s & 0xFF)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            eng.fit_items_device(n, d_items.data_ptr(), d_out.data_ptr())
            e1.record(stream)
            if s >= warmup:
                ms.append((e0, e1))
    torch.cuda.synchronize()
    t = [a.elapsed_time(b) for a, b in ms]
    eng.close()
    value = n / (np.mean(t) / 1000.0)
    out = {"value": value, "unit": "fits/s", "s_per_object": n / value, "fits_per_launch": n, "steps": steps,
           "ms_per_step": float(np.mean(t)), "gpu_launches": steps,
           "workload": "config 1 object 0: lmax 3 (16 coeffs), 288 facets, 1200 relative points, "
                       "200 frequencies x 10 poles, 50 LM iterations, FP64, one launch per step"}
    if cpu:
        import oracle

        cobj = objects.parse_input(text, setup_fn=oracle.setup_shape)
        cores = os.cpu_count() or 1
        nc = 4 * cores
        om = oracle.OracleModel(cobj)
        t0 = time.perf_counter()
        om.fit_batch(cobj.grid.freq_start, cobj.grid.freq_step, items[:nc, 0], items[:nc, 1], threads=cores,
                     fast=True)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": nc / dt, "unit": "fits/s", "cores": cores, "kind": "port",
                               "s_per_object": n / (nc / dt),
                               "sample": "%d fits (frequencies 1..%d, 10 poles) of the same object, %.1f s" %
                                         (nc, nc // 10, dt)}
    return out


def _best_pole_lines(res, n_points):
    """One line per frequency (10 consecutive poles) as the reference prints
    it: NaN-safe best rms, the earliest pole wins ties (start_CUDA.cu:1200-1229)."""
    lines = []
    for q in range(len(res) // 10):
        r = res[10 * q:10 * q + 10]
        b = -1
        for p in range(10):
            if b < 0 or (not np.isnan(r["dev"][p]) and not (r["dev"][p] >= r["dev"][b])):
                b = p
        x = r[b]
        lines.append((24 * x["per"], x["dev"], x["dev"] ** 2 * n_points, x["dark"], x["la"], x["be"]))
    return np.array(lines)


def result_errors(test, ref, n_points):
    """Differences of two runs of the same (frequency, pole) items: per fit
    the worst |dP| [h], |d lambda| [deg], |d beta|, |d rms|, |d chi^2| and
    how many fits print a different pole; per line (best of each frequency's
    10 poles) the reference's comparator rules."""
    from ps_claude_opt_b200 import compare, native

    dl = np.abs((test["la"] - ref["la"] + 180.0) % 360.0 - 180.0)
    printed = (np.round(test["la"]) != np.round(ref["la"])) | (np.round(test["be"]) != np.round(ref["be"]))
    lt = native.format_lines(_best_pole_lines(test, n_points)).splitlines()
    lr = native.format_lines(_best_pole_lines(ref, n_points)).splitlines()
    c = compare.compare_lines(lt, lr)
    return {"fits": int(len(test)),
            "max_abs": {"period_h": float(np.max(np.abs(test["per"] - ref["per"])) * 24),
                        "lambda_deg": float(np.max(dl)), "beta_deg": float(np.max(np.abs(test["be"] - ref["be"]))),
                        "rms": float(np.max(np.abs(test["dev"] - ref["dev"]))),
                        "chi2": float(np.max(np.abs(test["chisq"] - ref["chisq"])))},
            "fits_printed_pole_differs": int(np.sum(printed)),
            "fits_pole_off_gt1deg": int(np.sum((dl > 1.0) | (np.abs(test["be"] - ref["be"]) > 1.0))),
            "lines": int(len(lt)), "lines_pole_or_dark_mismatch": c.pole_mismatch,
            "lines_outside_envelope": c.envelope_violations, "best_line_same": c.best_line_same}


def flops_per_fit(obj, niter):
    """Algorithmic FLOPs of one fit: (niter + 1) evaluations + niter solves,
    per-point cost F_pt = 150 + 10 Nf + V (60 + 2 nc) + mfit (mfit + 1) +
    2 mfit + 6 ma [relative], V = 0.45 Nf."""
    nf, nc, mfit, ma = obj.n_fac, obj.n_coef, obj.mfit, obj.ma
    V = 0.45 * nf
    base = 150 + 10 * nf + V * (60 + 2 * nc) + mfit * (mfit + 1) + 2 * mfit
    n_rel = int(sum(l for l, r in zip(obj.curve_len, obj.curve_rel) if r))
    f_eval = obj.n_points * base + n_rel * 6 * ma + 3 * (2 * nf * nc + 2 * nf) + 2 * nf * nc + nf
    return (niter + 1) * f_eval + niter * 2.0 * mfit ** 3


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def cpu_baseline(obj, n_fits, freq_offset=1):
    """The oracle (C FP64 restatement, -O3 -march=native) on all host cores."""
    import oracle

    cores = os.cpu_count() or 1
    om = oracle.OracleModel(obj)
    nf = freq_offset + np.arange(n_fits) // 10
    pl = np.arange(n_fits) % 10
    t0 = time.perf_counter()
    om.fit_batch(obj.grid.freq_start, obj.grid.freq_step, nf, pl, threads=cores, fast=True)
    dt = time.perf_counter() - t0
    return n_fits / dt, cores, dt


def workload_name(obj):
    return ("production object: lmax 6 (49 coeffs), 512 facets, %d points (%d curves, 400 calibrated), "
            "%d frequencies x 10 poles, 50 LM iterations" % (obj.n_points, obj.n_curves, obj.grid.n_max))


def reference_arm(args, rank, world):
    """The reference's fit has no runnable CPU form and its GPU form needs
    BOINC: the CPU port of the same algorithm (the oracle) on all host cores
    stands in.  Under torchrun rank 0 alone runs it; the others exit."""
    if rank != 0:
        return
    import oracle

    obj, _ = workload(setup_fn=oracle.setup_shape)
    cores = os.cpu_count() or 1
    per_step = max(8, cores)
    freq_at = lambda s: 1 + s * (per_step // 10 + 1)  # noqa: E731
    for s in range(max(1, args.warmup)):  # untimed: page in, spin up threads
        cpu_baseline(obj, per_step, freq_offset=freq_at(s))
    times = []
    for s in range(args.steps):
        rate, _, dt = cpu_baseline(obj, per_step, freq_offset=freq_at(args.warmup + s))
        times.append(dt)
    total = sum(times)
    value = per_step * args.steps / total
    n_obj = obj.grid.n_max * 10
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "fits/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator; no public dataset ships with the reference)",
        "config": {"workload": workload_name(obj), "sample": "%d fits per step" % per_step,
                   "parallelism": "host threads (CPU port of the fit on %d cores; no GPU)" % cores},
        "s_per_object": n_obj / value,
        "cpu_baseline": {"value": value, "unit": "fits/s", "cores": cores, "kind": "port",
                         "sample": "%d fits x %d steps of the production object on %d threads" %
                                   (per_step, args.steps, cores)},
        "e2e": {"value": value, "unit": "fits/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def profile_case(mixed=False):
    """One launch to capture under ncu: the production object, one fit per
    resident CTA (1 GPU), FP64 or mixed precision."""
    from ps_claude_opt_b200 import native

    obj, _ = workload()
    with native.Engine(obj, device=0) as eng:
        if mixed:
            eng.set_precision(native.PRECISION_MIXED)
        eng.configure(conw_r=obj.conw_r)
        ctas, nsm = eng.occupancy()
        n = ctas * nsm
        nf = 1 + np.arange(n) // 10
        pl = np.arange(n) % 10
        for _ in range(2):
            res, niter, _ = eng.fit_items(nf, pl)
        assert np.all(np.isfinite(res[:, 2]))
        print("profile case: %d fits, mean iterations %.1f, flops/launch %.4g" %
              (n, niter.mean(), flops_per_fit(obj, niter.mean()) * n))


RESULT_DTYPE = np.dtype([("dev", "f8"), ("dark", "f8"), ("per", "f8"), ("la", "f8"), ("be", "f8"),
                         ("chisq", "f8"), ("niter", "i4"), ("status", "i4")])
FIXTURE = os.path.join(ROOT, "tests", "golden", "bench_object_fullscan.json")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--fits-per-cta", type=int, default=FITS_PER_CTA)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="only the headline legs (FP64 timed steps, end to end, mixed); skip config 1, the "
                         "reference GPU app, the screened scan and the batch")
    ap.add_argument("--batch-objects", type=int, default=None)
    ap.add_argument("--batch-freqs", type=int, default=4)
    ap.add_argument("--profile-case", action="store_true",
                    help="two fit-kernel launches (warm-up + one to capture), one fit per resident CTA")
    ap.add_argument("--mixed", action="store_true", help="with --profile-case: the mixed-precision kernel")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return

    if args.profile_case:
        profile_case(args.mixed)
        return

    from ps_claude_opt_b200 import synth

    extra = rank == 0 and world == 1 and not args.no_extra
    # host-side generation of the batched workload, before this process touches a GPU
    n_batch = synth.C3_OBJECTS if args.batch_objects is None else args.batch_objects
    batch_in = batch_texts(n_batch) if extra and n_batch > 0 else None

    import torch

    from ps_claude_opt_b200 import native

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    obj, truth = workload()
    peak = native.measure_fp64_peak(local_rank)
    eng = native.Engine(obj, device=local_rank)
    eng.configure(conw_r=obj.conw_r)
    ctas, nsm = eng.occupancy()
    n_fits = ctas * nsm * args.fits_per_cta
    n_fits -= n_fits % 10
    freqs_per_step = n_fits // 10
    n_max = obj.grid.n_max
    steps_total = args.warmup + args.steps

    def items_for(step):
        base = ((rank * steps_total + step) * freqs_per_step) % max(1, n_max - freqs_per_step)
        it = np.zeros((n_fits, 2), dtype=np.int32)
        it[:, 0] = 1 + base + np.arange(n_fits) // 10
        it[:, 1] = np.arange(n_fits) % 10
        return it

    stream = torch.cuda.ExternalStream(eng.stream)
    d_items = [torch.from_numpy(items_for(s)).cuda() for s in range(steps_total)]
    rec = ctypes.sizeof(native.FitResult)   # one ps_fit_result per fit
    assert RESULT_DTYPE.itemsize == rec
    d_out = torch.empty(n_fits * rec, dtype=torch.uint8, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()

    def run_step(s):
        eng.fit_items_device(n_fits, d_items[s].data_ptr(), d_out.data_ptr())

    def timed_steps():
        evs = []
        with torch.cuda.stream(stream):
            for s in range(args.warmup, steps_total):
                flush.fill_(s & 0xFF)   # L2 flush between timed launches (not timed)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                run_step(s)
                e1.record(stream)
                evs.append((e0, e1))
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in evs]

    with torch.cuda.stream(stream):
        for s in range(args.warmup):
            flush.fill_(s & 0xFF)
            run_step(s)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()

    clocks = ClockSampler(local_rank)
    clocks.start()
    ms = timed_steps()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = float(sum(ms))

    # the last step's results: iteration counts for the FLOP count, a sanity check
    res = np.frombuffer(d_out.cpu().numpy().tobytes(), dtype=RESULT_DTYPE).copy()
    niter = float(np.mean(res["niter"]))
    if not np.all(np.isfinite(res["per"])):
        raise RuntimeError("non-finite fit results")

    if dist:
        t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = n_fits * args.steps * world / (total_ms / 1000.0)
    fl = flops_per_fit(obj, niter) * n_fits
    achieved = fl / (np.mean(ms) / 1000.0) / 1e12

    # end to end through the C ABI with host buffers: object upload, items,
    # kernel, results back -- what a caller of ps_gpu_configure + ps_gpu_fit_items pays
    it = items_for(args.warmup)
    h2d = (obj.n_points * (4 * 8 + 4 * 8 + 8 + 4) + obj.n_fac * (32 + 8 * ((obj.n_coef + 7) // 8 * 8))
           + it.nbytes)
    d2h = n_fits * rec
    e2e_ms = []
    e2e_clocks = ClockSampler(local_rank)
    e2e_clocks.start()
    for s in range(max(1, min(args.steps, 5))):
        flush.fill_(s)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng.configure(conw_r=obj.conw_r)
        eng.fit_items(it[:, 0], it[:, 1])
        e2e_ms.append((time.perf_counter() - t0) * 1000)
    e2e_clk = e2e_clocks.stop()
    e2e_value = n_fits * world / (np.mean(e2e_ms) / 1000.0)

    # the same steps with the mixed-precision sweep (FP32 facet terms, 3xTF32
    # tensor-core shape derivatives; FP64 elsewhere), device-timed the same way
    eng.set_precision(native.PRECISION_MIXED)
    eng.configure(conw_r=obj.conw_r)
    with torch.cuda.stream(stream):
        flush.fill_(1)
        run_step(0)
    torch.cuda.synchronize()
    mixed_ms = float(sum(timed_steps()))
    res_m = np.frombuffer(d_out.cpu().numpy().tobytes(), dtype=RESULT_DTYPE).copy()
    if dist:
        t = torch.tensor([mixed_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        mixed_ms = float(t.item())
    mixed_value = n_fits * args.steps * world / (mixed_ms / 1000.0)
    eng.close()

    line = None
    if rank == 0:
        n_obj = n_max * 10
        line = {
            "metric": METRIC, "value": value, "unit": "fits/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator; no public dataset ships with the reference)",
            "config": {"workload": workload_name(obj),
                       "fits_per_step_per_gpu": n_fits, "ctas_per_sm": ctas,
                       "l2": "256 MB buffer written between timed launches; per-launch scratch %.0f MB > L2" %
                             (ctas * nsm * (obj.n_points * (obj.ma + 2) + obj.n_curves * (obj.ma + 3)) * 8 / 1e6),
                       "parallelism": "dp%d (disjoint frequency ranges per GPU)" % world},
            "s_per_object": n_obj / (value / world),
            "roofline": {"bound": "tensor",
                         "bound_detail": "FP64 compute: the FP64 tensor-core (DMMA) and FMA pipes share one "
                                         "capacity on B200 (probe: 37.0 / 34.9 TF/s alone, 36.5 together); "
                                         "MEASURED_PEAKS.json's bf16 figure does not apply to FP64 work",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": NCU_DRAM_BYTES_PER_FIT * n_fits,
                         "traffic_source": "ncu capture of the profile case (148 fits), scaled by fits per launch",
                         "peak_source": "measured FP64 FMA probe (ps_measure_fp64_peak) on this GPU; "
                                        "MEASURED_PEAKS.json has no FP64 figure",
                         "flops_per_launch": fl, "mean_niter": niter},
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": "fits/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": float(np.mean(e2e_ms)),
                    "ms_per_step_each": [float(v) for v in e2e_ms], "clocks": e2e_clk},
            "gpu_launches": args.steps,
            "mixed": {"value": mixed_value, "unit": "fits/s", "ms_per_step": mixed_ms / args.steps,
                      "s_per_object": n_obj / (mixed_value / world), "gpu_launches": args.steps,
                      "speedup_vs_fp64": mixed_value / value,
                      "precision": "facet sweep FP32 (Newton-refined reciprocal, per-point sums flushed to FP64 "
                                   "every 8 facets) with 3xTF32 tensor-core shape derivatives; geometry, "
                                   "J^T W J, chi^2, Gauss-Jordan and lambda update FP64",
                      "errors_vs_fp64": result_errors(res_m, res, obj.n_points)},
        }
        if world == 1 and not args.no_cpu_baseline:
            cores = os.cpu_count() or 1
            n_cpu = 10 * cores     # about 10 s of CPU work at ~1 fit/s per core
            rate, cores, dt = cpu_baseline(obj, n_cpu)
            line["cpu_baseline"] = {"value": rate, "unit": "fits/s", "cores": cores, "kind": "port",
                                    "sample": "%d fits (frequencies 1.., 10 poles) of the same object, %.1f s" %
                                              (n_cpu, dt)}
    if extra:
        from ps_claude_opt_b200 import screen

        # the screened + mixed scan of the whole object, end to end on this
        # GPU: features of all trial frequencies, the network's ranking, the
        # mixed fits of the chosen frequencies (all 10 poles), widening at run
        # edges and the audit's fallback.  The convexity-weight search, the
        # same for both kinds of scan, is left out of both: the scan uses the
        # weight the full FP64 scan of the fixture ended with.
        fix = json.load(open(FIXTURE)) if os.path.exists(FIXTURE) else None
        conw_r = fix["conw_r"] if fix else obj.conw_r
        net = screen.load_model()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pred = net.predict(screen.normalise(screen.features(obj, screen.frequencies(obj), local_rank)))
        t_rank = time.perf_counter() - t0
        idx, lines, _, plan = screen.screened_scan(obj, net, conw_r, device=local_rank,
                                                   precision=native.PRECISION_MIXED, pred=pred)
        screened_s = time.perf_counter() - t0
        b = screen.best_line(lines)
        sm = {"s_per_object": screened_s, "ranking_s": t_rank, "fitted_frequencies": int(len(idx)),
              "first_selection": plan.initial, "edge_expansions": plan.expansions,
              "period_doubling_probes": plan.alias_probes, "fallback": plan.fallback,
              "fallback_reason": plan.reason, "n_frequencies": int(n_max),
              "fits": int(10 * (plan.first_pass + plan.polished)), "mixed_fitted_frequencies": plan.first_pass,
              "fp64_refitted_frequencies": plan.polished,
              "vs_plain_fp64_full_scan_s": n_max * 10 / value,
              "speedup_vs_plain_fp64_full_scan": (n_max * 10 / value) / screened_s,
              "best_frequency": int(idx[b]),
              "note": "top 3.4 % of the network's ranking with one neighbour each side plus a 2 % random audit, "
                      "widened around a best line at a run edge, its period-doubling partners probed, full grid "
                      "if the audit contradicts the ranking; "
                      "mixed-precision fits, then the candidate lines (best line, its period-doubling partners, "
                      "the lowest local minima) refitted in FP64; trained network ps_claude_opt_b200/screen_model.bin"}
        if fix:
            got = native.format_lines(lines[b:b + 1]).strip()
            sm["best_line_matches_full"] = bool(int(idx[b]) == fix["best_freq"] and
                                                got.split()[3:] == fix["formatted_best"].split()[3:] and
                                                abs(lines[b, 0] - fix["best_line"][0]) < 0.1 and
                                                abs(lines[b, 1] - fix["best_line"][1]) < 0.1)
            sm["best_line_printed_equal"] = got == fix["formatted_best"]
            sm["best_line"] = got
            sm["full_scan_best_line"] = fix["formatted_best"]
        line["screened_mixed"] = sm
        line["c1"] = c1_leg(args.steps, args.warmup, local_rank, cpu=not args.no_cpu_baseline)
        line["reference_gpu"] = reference_gpu_leg()
        if batch_in:
            line["batch"] = bench_batch(batch_in, args.batch_freqs, device=local_rank)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
