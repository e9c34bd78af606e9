"""Trains the frequency-screening network and judges it against the full scan.

    python -m ps_claude_opt_b200.screen_train --objects 96 --out ps_claude_opt_b200/screen_model.bin

Training objects come from the production-size generator (lmax 6, 512 facets,
40 dense relative curves + 400 calibrated points, periods 2-100 h on the
reference's frequency grid), seeds 7_000_000 + i.  For each object the plain
FP64 LM (all 10 poles) labels a sample of its trial frequencies: the ones
nearest the true period, half and twice it, plus a uniform random share.
Label = log of the frequency's best rms, standardised per object with the
random share's mean and spread; features are standardised per object over
all its frequencies.  Held-out objects (seeds 8_000_000 + i) are scanned in
full and the screened scan (the top 3.4 % of frequencies with one neighbour
on either side, plus a 2 % random audit: at most 12.2 % of the grid) is
judged on whether its best line is the full scan's.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import native, objects, screen, synth

TRAIN_SEED = 7_000_000
EVAL_SEED = 8_000_000


def make_object(seed):
    cfg = synth.SynthConfig(l_max=6, m_max=6, nrows=8, n_dense=40, dense_pts=(50, 120), n_sparse=400,
                            sparse_curves=2, period_range=(2.0, 100.0), n_freq=5000)
    text, truth = synth.generate(cfg, seed)
    return objects.parse_input(text), truth


def label_frequencies(obj, truth, n_rand, n_near, rng):
    """1-based indices: n_near around each of P, P/2, 2P, and n_rand uniform."""
    g = obj.grid
    n_max = g.n_max
    picks = set()
    for mult in (1.0, 0.5, 2.0):
        f = 1.0 / (truth["period_h"] * mult)   # 1/hour, the grid's unit
        c = int(round((g.freq_start - f) / g.freq_step)) + 1
        for d in range(-(n_near // 2), n_near - n_near // 2):
            if 1 <= c + d <= n_max:
                picks.add(c + d)
    rand = rng.choice(np.arange(1, n_max + 1), size=min(n_rand, n_max), replace=False)
    return np.array(sorted(picks)), np.array(sorted(set(rand.tolist())))


def best_rms(res):
    """Per frequency (rows of 10 poles): the NaN-safe, earliest-wins best rms."""
    out = np.empty(res.shape[0])
    for q in range(res.shape[0]):
        r = res[q, :, 0]
        best = -1
        for p in range(native.N_POLES):
            if best < 0 or (not np.isnan(r[p]) and not (r[p] >= r[best])):
                best = p
        out[q] = r[best]
    return out


def fit_frequencies(eng, idx):
    nf = np.repeat(idx, native.N_POLES).astype(np.int32)
    pl = np.tile(np.arange(native.N_POLES), len(idx)).astype(np.int32)
    res, _, _ = eng.fit_items(nf, pl)
    return res.reshape(len(idx), native.N_POLES, 6)


def label_objects(n_obj, n_rand=240, n_near=20, seed0=TRAIN_SEED, log=print):
    """Per training object: (seed, labelled frequency indices, their best rms,
    the random share's indices), from plain FP64 fits of all 10 poles."""
    out = []
    rng = np.random.default_rng(seed0)
    for i in range(n_obj):
        t0 = time.time()
        obj, truth = make_object(seed0 + i)
        near, rand = label_frequencies(obj, truth, n_rand, n_near, rng)
        idx = np.array(sorted(set(near.tolist()) | set(rand.tolist())))
        with native.Engine(obj) as eng:
            eng.configure()
            rms = best_rms(fit_frequencies(eng, idx))
        out.append((seed0 + i, idx, rms, rand))
        log("object %d: %d labelled frequencies, %.1f s" % (i, len(idx), time.time() - t0))
    return out


def training_set(labels):
    """Features (standardised per object) and labels (log best rms,
    standardised with the random share's mean and spread)."""
    X, Y = [], []
    for seed, idx, rms, rand in labels:
        obj, _ = make_object(int(seed))
        feat = screen.normalise(screen.features(obj, screen.frequencies(obj)))
        lab = np.log(np.where(np.isfinite(rms) & (rms > 0), rms, np.nan))
        in_rand = np.isin(idx, rand) & np.isfinite(lab)
        mu, sd = lab[in_rand].mean(), lab[in_rand].std() + 1e-9
        ok = np.isfinite(lab)
        X.append(feat[idx[ok] - 1])
        Y.append(((lab[ok] - mu) / sd).astype(np.float32))
    return np.concatenate(X), np.concatenate(Y)


def save_labels(path, labels):
    np.savez_compressed(path, seeds=np.array([l[0] for l in labels]),
                        **{f"idx{i}": l[1] for i, l in enumerate(labels)},
                        **{f"rms{i}": l[2] for i, l in enumerate(labels)},
                        **{f"rand{i}": l[3] for i, l in enumerate(labels)})


def load_labels(path):
    d = np.load(path)
    return [(int(s), d[f"idx{i}"], d[f"rms{i}"], d[f"rand{i}"]) for i, s in enumerate(d["seeds"])]


def train(X, Y, epochs=60, batch=1024, lr=1e-3, seed=0, log=print):
    import torch

    net = screen.Mlp(seed=seed)
    xd = torch.from_numpy(X).cuda().to(torch.bfloat16)
    yd = torch.from_numpy(Y).cuda()
    rng = np.random.default_rng(seed)
    n = len(Y)
    for ep in range(epochs):
        perm = torch.from_numpy(rng.permutation(n)).cuda()
        tot = 0.0
        for i in range(0, n, batch):
            sel = perm[i:i + batch]
            tot += net.train_step(xd[sel], yd[sel], lr) * len(sel)
        if ep % 10 == 0 or ep == epochs - 1:
            log("epoch %d: mse %.4f" % (ep, tot / n))
    return net


def full_scans(n_obj, seed0=EVAL_SEED, log=print):
    """Per held-out object: (seed, full-scan lines, final conw_r, seconds)."""
    out = []
    for i in range(n_obj):
        obj, _ = make_object(seed0 + i)
        t0 = time.time()
        full, conw_r = native.run_object(obj)
        out.append((seed0 + i, full, conw_r, time.time() - t0))
        log("full scan %d: %.1f s" % (i, out[-1][3]))
    return out


def judge(net, fulls, top=0.034, halo=1, audit=0.02, log=print, precision=native.PRECISION_FP64):
    """Screened scan vs full scan on held-out objects: the screened best line
    must be the full scan's (same frequency, or period within 0.1 h, rms
    within 0.1 and pole within 1 degree).  Each row also records whether the
    scan expanded around an edge or fell back to the whole grid."""
    hits, rows = 0, []
    for i, (seed, full, conw_r, t_full) in enumerate(fulls):
        obj, _ = make_object(int(seed))
        t0 = time.time()
        idx, lines, _, plan = screen.screened_scan(obj, net, conw_r, top, halo, audit, seed=i,
                                                   precision=precision)
        t_scr = time.time() - t0
        bf, bs = screen.best_line(full), screen.best_line(lines)
        fb, sb = full[bf], lines[bs]
        dl = abs((fb[4] - sb[4] + 180.0) % 360.0 - 180.0)
        ok = (idx[bs] == bf + 1) or (abs(fb[0] - sb[0]) < 0.1 and abs(fb[1] - sb[1]) < 0.1 and dl < 1.0 and
                                     abs(fb[5] - sb[5]) < 1.0)
        hits += ok
        rows.append(dict(seed=int(seed), full_best=int(bf + 1), screened_best=int(idx[bs]), ok=bool(ok),
                         full_s=float(t_full), screened_s=t_scr, fitted=len(idx), n_freq=len(full),
                         initial=plan.initial, expansions=plan.expansions, fallback=plan.fallback,
                         reason=plan.reason))
        log(json.dumps(rows[-1]))
    return hits, rows


def _hit(full_best, full_fields, idx, lines, bs):
    """The screened best line (lines[bs] at frequency idx[bs]) is the full
    scan's: same frequency, or period within 0.1 h, rms within 0.1 and pole
    within 1 degree (full_fields: the full scan's printed best line, split)."""
    sb = lines[bs]
    fp, fr, fl, fbeta = float(full_fields[0]), float(full_fields[1]), float(full_fields[4]), float(full_fields[5])
    dl = abs((fl - sb[4] + 180.0) % 360.0 - 180.0)
    return bool(idx[bs] == full_best or (abs(fp - sb[0]) < 0.1 and abs(fr - sb[1]) < 0.1 and dl < 1.0 and
                                         abs(fbeta - sb[5]) < 1.0))


FP64_SCREEN_FIELDS = ("ok_fp64_screen", "fp64_screen_best", "fp64_screen_fallback", "fp64_screen_fitted")


def screen_row(net, i, obj, truth, n_freq, conw_r, full_best, full_line, t_full, precision=native.PRECISION_MIXED,
               fp64_row=None):
    """One held-out object's screened scans -- in `precision` (the screened
    + mixed form by default) and in FP64, which separates the ranking's
    misses from lines that only the precision moved -- judged against the
    full FP64 scan's best line (1-based frequency, printed line).  fp64_row:
    an earlier row of the same object whose FP64 screened-scan fields are
    reused instead of running that scan again (its inputs are unchanged)."""
    full_fields = full_line.split()
    t0 = time.time()
    idx, lines, _, plan = screen.screened_scan(obj, net, conw_r, seed=i, precision=precision)
    t_scr = time.time() - t0
    bs = screen.best_line(lines)
    if fp64_row is not None:
        fp64 = {k: fp64_row[k] for k in FP64_SCREEN_FIELDS}
    else:
        idx64, lines64, _, plan64 = screen.screened_scan(obj, net, conw_r, seed=i, precision=native.PRECISION_FP64)
        bs64 = screen.best_line(lines64)
        fp64 = dict(ok_fp64_screen=_hit(full_best, full_fields, idx64, lines64, bs64),
                    fp64_screen_best=int(idx64[bs64]), fp64_screen_fallback=plan64.fallback,
                    fp64_screen_fitted=int(len(idx64)))
    return dict(seed=EVAL_SEED + i, n_freq=n_freq, conw_r=conw_r, full_best=full_best, full_line=full_line,
                screened_best=int(idx[bs]), screened_line=native.format_lines(lines[bs:bs + 1]).strip(),
                ok=_hit(full_best, full_fields, idx, lines, bs), same_frequency=bool(idx[bs] == full_best),
                **fp64, fitted=int(len(idx)), initial=plan.initial,
                expansions=plan.expansions, alias_probes=plan.alias_probes, fallback=plan.fallback,
                reason=plan.reason, polished=plan.polished, polish_rounds=plan.polish_rounds,
                full_s_per_object=t_full, screened_s=t_scr,
                true_period_h=float(truth["period_h"]), precision=int(precision))


def judge_stream(net, start, count, out_path, precision=native.PRECISION_MIXED, group=8, log=print):
    """The held-out judgement at scale, one JSON line per object appended to
    out_path as soon as its group is done (a partial run keeps its rows).
    The judge is the plain FP64 full scan of object EVAL_SEED + start + i
    (convexity-weight search, then all 5000 frequencies x 10 poles), run
    `group` objects at a time through ps_gpu_scan_batch, whose lines are
    bit-identical to one object at a time; the screened scans (screen_row)
    use the judge's convexity weight."""
    done = set()
    try:
        with open(out_path) as f:
            done = {json.loads(l)["seed"] for l in f if l.strip()}
    except FileNotFoundError:
        pass
    todo = [i for i in range(start, start + count) if EVAL_SEED + i not in done]
    for g0 in range(0, len(todo), group):
        ids = todo[g0:g0 + group]
        objs = [make_object(EVAL_SEED + i) for i in ids]
        t0 = time.time()
        fulls = native.scan_batch([o for o, _ in objs])
        t_full = (time.time() - t0) / len(ids)
        for i, (obj, truth), (full, conw_r) in zip(ids, objs, fulls):
            bf = screen.best_line(full)
            row = screen_row(net, i, obj, truth, len(full), conw_r, bf + 1,
                             native.format_lines(full[bf:bf + 1]).strip(), t_full, precision)
            with open(out_path, "a") as f:
                f.write(json.dumps(row) + "\n")
            log(json.dumps(row))


def rescreen(net, rows_in, out_path, precision=native.PRECISION_MIXED, log=print):
    """Re-judges the screened scans of objects whose full FP64 scans a
    judge_stream run already made (its rows: best frequency, printed best
    line, convexity weight), with the current screen, without scanning them
    again; rows that carry the FP64 screened scan's fields keep them."""
    done = set()
    try:
        with open(out_path) as f:
            done = {json.loads(l)["seed"] for l in f if l.strip()}
    except FileNotFoundError:
        pass
    for l in open(rows_in):
        if not l.strip():
            continue
        r = json.loads(l)
        if r["seed"] in done:
            continue
        obj, truth = make_object(r["seed"])
        reuse = r if all(k in r for k in FP64_SCREEN_FIELDS) else None
        row = screen_row(net, r["seed"] - EVAL_SEED, obj, truth, r["n_freq"], r["conw_r"], r["full_best"],
                         r["full_line"], r["full_s_per_object"], precision, fp64_row=reuse)
        with open(out_path, "a") as f:
            f.write(json.dumps(row) + "\n")
        log(json.dumps(row))


def summarize(rows):
    """Totals of held-out judgement rows (judge_stream / rescreen output), one
    row per object: hits of the screened + mixed scan and of the screened
    FP64 scan against the FP64 full scan's best line, the one-sided 95 %
    lower bound of the hit rate (Clopper-Pearson), fallbacks to the full
    grid, frequencies fitted, and the period ratio of each miss to the full
    scan's best period (2 or 1/2: a period-doubling alias)."""
    from scipy.stats import beta as beta_dist

    n = len(rows)
    if n == 0:
        return dict(objects=0)
    hits = sum(bool(r["ok"]) for r in rows)
    hits64 = sum(bool(r.get("ok_fp64_screen", r["ok"])) for r in rows)
    lower = float(beta_dist.ppf(0.05, hits, n - hits + 1)) if hits > 0 else 0.0
    misses = []
    for r in rows:
        if r["ok"]:
            continue
        full_p = float(r["full_line"].split()[0])
        scr_p = float(r["screened_line"].split()[0]) if r.get("screened_line") else float("nan")
        misses.append(dict(seed=r["seed"], full_period_h=full_p, screened_period_h=scr_p,
                           ratio=scr_p / full_p if full_p else float("nan")))
    fitted = np.array([r["fitted"] for r in rows], dtype=float)
    return dict(objects=n, hits=hits, hit_rate=hits / n, hit_rate_lower95=lower, hits_fp64_screen=hits64,
                fallbacks=sum(bool(r["fallback"]) for r in rows),
                expansions=int(sum(int(r.get("expansions", 0)) for r in rows)),
                alias_probes=int(sum(int(r.get("alias_probes", 0)) for r in rows)),
                fitted_mean=float(fitted.mean()), fitted_max=int(fitted.max()),
                n_freq=int(rows[0]["n_freq"]),
                screened_s_mean=float(np.mean([r["screened_s"] for r in rows])),
                full_s_mean=float(np.mean([r["full_s_per_object"] for r in rows])),
                misses=misses)


def main():
    import os

    ap = argparse.ArgumentParser()
    ap.add_argument("--objects", type=int, default=96)
    ap.add_argument("--eval-objects", type=int, default=8)
    ap.add_argument("--epochs", type=int, default=150)
    ap.add_argument("--labels", default=None, help="npz of training labels: read if present, else written")
    ap.add_argument("--fulls", default=None, help="npz of held-out full scans: read if present, else written")
    ap.add_argument("--eval-start", type=int, default=0, help="first held-out object (seed offset)")
    ap.add_argument("--model", default=None, help="judge this trained network instead of training one")
    ap.add_argument("--out", default=None)
    ap.add_argument("--judge-out", default=None,
                    help="stream the held-out judgement (FP64 full scans as the judge) to this JSON-lines file")
    ap.add_argument("--rescreen", default=None,
                    help="with --judge-out: re-judge the screened scans of the objects in this rows file")
    ap.add_argument("--summarize", nargs="+", default=None,
                    help="print the totals of these judgement rows files (no GPU work)")
    args = ap.parse_args()
    if args.summarize:
        rows = [json.loads(l) for path in args.summarize for l in open(path) if l.strip()]
        print(json.dumps(summarize(rows), indent=1))
        return
    if args.judge_out:
        net = screen.load_model(args.model or screen.MODEL_PATH)
        if args.rescreen:
            rescreen(net, args.rescreen, args.judge_out)
        else:
            judge_stream(net, args.eval_start, args.eval_objects, args.judge_out)
        return
    t0 = time.time()
    if args.model:
        net = screen.load_model(args.model)
    else:
        if args.labels and os.path.exists(args.labels):
            labels = load_labels(args.labels)
        else:
            labels = label_objects(args.objects)
            if args.labels:
                save_labels(args.labels, labels)
        X, Y = training_set(labels)
        print("training set: %d samples from %d objects, %.1f s" % (len(Y), len(labels), time.time() - t0),
              flush=True)
        net = train(X, Y, args.epochs)
        if args.out:
            screen.save_model(args.out, net.state())
    if args.eval_objects:
        if args.fulls and os.path.exists(args.fulls):
            d = np.load(args.fulls)
            fulls = [(int(s), d[f"lines{i}"], float(d["conw"][i]), float(d["secs"][i]))
                     for i, s in enumerate(d["seeds"])]
        else:
            fulls = full_scans(args.eval_objects, seed0=EVAL_SEED + args.eval_start)
            if args.fulls:
                np.savez_compressed(args.fulls, seeds=np.array([f[0] for f in fulls]),
                                    conw=np.array([f[2] for f in fulls]), secs=np.array([f[3] for f in fulls]),
                                    **{f"lines{i}": f[1] for i, f in enumerate(fulls)})
        hits, _ = judge(net, fulls[:args.eval_objects])
        print("screened best line = full scan best line on %d of %d held-out objects" %
              (hits, min(args.eval_objects, len(fulls))))


if __name__ == "__main__":
    main()
