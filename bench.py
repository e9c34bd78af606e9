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
# dram__bytes_write.sum = 27.53 GB over the 148 fits of one ncu capture of
# `bench.py --profile-case` (the derivative-row scratch round trip; it grows
# with the number of fits, so a launch's traffic is this times its fits).
NCU_DRAM_BYTES_PER_FIT = 27.53e9 / 148
METRIC = ("LM fits/s of the plain FP64 full scan of the production object on 1 B200 (s/object of it and of "
          "the screened+mixed scan in the same line)")


def workload(setup_fn=None):
    """The production object.  setup_fn builds its shape tables: the
    library's (default) or, for the CPU arms, the oracle's, so that those
    arms load no product code."""
    from ps_claude_opt_b200 import objects, synth

    text, truth = synth.generate(synth.C2, SEED)
    return objects.parse_input(text, setup_fn=setup_fn), truth


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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--fits-per-cta", type=int, default=FITS_PER_CTA)
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
    d_out = torch.empty(n_fits * rec, dtype=torch.uint8, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()

    def run_step(s):
        eng.fit_items_device(n_fits, d_items[s].data_ptr(), d_out.data_ptr())

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
    ms = [a.elapsed_time(b) for a, b in evs]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = float(sum(ms))

    # read back the last step: iteration counts for the FLOP count, and a sanity check
    res = np.frombuffer(d_out.cpu().numpy().tobytes(), dtype=np.dtype(
        [("dev", "f8"), ("dark", "f8"), ("per", "f8"), ("la", "f8"), ("be", "f8"), ("chisq", "f8"),
         ("niter", "i4"), ("status", "i4")]))
    assert res.dtype.itemsize == rec
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
    for s in range(max(1, min(args.steps, 3))):
        flush.fill_(s)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng.configure(conw_r=obj.conw_r)
        eng.fit_items(it[:, 0], it[:, 1])
        e2e_ms.append((time.perf_counter() - t0) * 1000)
    e2e_value = n_fits * world / (np.mean(e2e_ms) / 1000.0)

    # the same steps with the mixed-precision sweep (FP32 facet terms, 3xTF32
    # tensor-core shape derivatives; FP64 elsewhere), device-timed the same way
    eng.set_precision(native.PRECISION_MIXED)
    eng.configure(conw_r=obj.conw_r)
    with torch.cuda.stream(stream):
        flush.fill_(1)
        run_step(0)
    torch.cuda.synchronize()
    evm = []
    with torch.cuda.stream(stream):
        for s in range(args.warmup, steps_total):
            flush.fill_(s & 0xFF)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            run_step(s)
            e1.record(stream)
            evm.append((e0, e1))
    torch.cuda.synchronize()
    mixed_ms = float(sum(a.elapsed_time(b) for a, b in evm))
    if dist:
        t = torch.tensor([mixed_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        mixed_ms = float(t.item())
    mixed_value = n_fits * args.steps * world / (mixed_ms / 1000.0)

    # the screened + mixed scan of the whole object, end to end on this GPU:
    # features of all trial frequencies, the network's ranking, the mixed
    # fits of the chosen frequencies (all 10 poles) -- the convexity-weight
    # search, the same for both kinds of scan, is left out of both
    from ps_claude_opt_b200 import screen

    net = screen.load_model()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pred = net.predict(screen.normalise(screen.features(obj, screen.frequencies(obj), local_rank)))
    sel = screen.select(pred) + 1
    t_rank = time.perf_counter() - t0
    eng.fit_items(np.repeat(sel, 10), np.tile(np.arange(10), len(sel)))
    screened_s = time.perf_counter() - t0

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
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": float(np.mean(e2e_ms))},
            "gpu_launches": args.steps,
            "screened_mixed": {"s_per_object": screened_s, "ranking_s": t_rank, "fitted_frequencies": int(len(sel)),
                               "n_frequencies": int(n_max), "fits": int(10 * len(sel)),
                               "vs_plain_fp64_full_scan_s": n_obj / (value / world),
                               "note": "top 3.4 % of the network's ranking with one neighbour each side plus a "
                                       "2 % random audit; mixed-precision fits; trained network from "
                                       "ps_claude_opt_b200/screen_model.bin"},
            "mixed": {"value": mixed_value, "unit": "fits/s", "ms_per_step": mixed_ms / args.steps,
                      "s_per_object": n_obj / (mixed_value / world), "gpu_launches": args.steps,
                      "precision": "facet sweep FP32 with 3xTF32 tensor-core shape derivatives; geometry, "
                                   "J^T W J, chi^2, Gauss-Jordan and lambda update FP64"},
        }
        if world == 1 and not args.no_cpu_baseline:
            cores = os.cpu_count() or 1
            n_cpu = 10 * cores     # about 10 s of CPU work at ~1 fit/s per core
            rate, cores, dt = cpu_baseline(obj, n_cpu)
            line["cpu_baseline"] = {"value": rate, "unit": "fits/s", "cores": cores, "kind": "port",
                                    "sample": "%d fits (frequencies 1.., 10 poles) of the same object, %.1f s" %
                                              (n_cpu, dt)}
        print(json.dumps(line), flush=True)
    eng.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
