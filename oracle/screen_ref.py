"""CPU restatement of the frequency-screening features and of the BF16
multilayer perceptron's forward and backward passes.

Test infrastructure only: it checks the CUDA kernels of
ps_claude_opt_b200/csrc/screen.cu and is never called by the product.  The
screen has no counterpart in the reference (which fits every trial
frequency), so there is nothing of the reference to cite here; the feature
definition is the one stated in screen.cu.
"""
from __future__ import annotations

import numpy as np

N_BINS = 64


def bf16_round(x):
    """Round float32 values to bfloat16 (nearest, ties to even), as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def curve_stats(cnt, s1b, s2b):
    """The 8 per-curve statistics from 64-bin counts, sums and square sums."""
    cnt, s1b, s2b = (np.asarray(v, dtype=np.float64) for v in (cnt, s1b, s2b))
    n, s1, s2 = cnt.sum(), s1b.sum(), s2b.sum()
    total = s2 - (s1 * s1 / n if n > 0 else 0.0)
    st = np.zeros(8)
    for lev in range(4):
        w = 1 << lev
        c = cnt.reshape(-1, w).sum(1)
        a = s1b.reshape(-1, w).sum(1)
        q = s2b.reshape(-1, w).sum(1)
        within = np.sum(np.where(c > 0, q - a * a / np.where(c > 0, c, 1), 0.0))
        st[lev] = within / total if total > 0 else 1.0
    c32 = cnt.reshape(32, 2).sum(1)
    m32 = s1b.reshape(32, 2).sum(1)
    ok = c32 > 0
    b = np.arange(32)[ok]
    m = m32[ok] / c32[ok]
    pw = np.zeros(4)
    for k in range(4):
        ang = np.pi * (2 * (k + 1) * b) / 32.0
        pw[k] = np.sum(m * np.cos(ang)) ** 2 + np.sum(m * np.sin(ang)) ** 2
    tot = pw.sum()
    st[4:] = pw / tot if tot > 0 else 0.25
    return st


def features(tim, brightness, curve_len, freqs):
    """[n_freq, 88] features: 8 * statistic + aggregate over the curves, then
    64 + 8 * fold + statistic for the folds of all points."""
    tim = np.asarray(tim, dtype=np.float64)
    br = np.asarray(brightness, dtype=np.float64)
    starts = np.concatenate([[0], np.cumsum(curve_len)])
    y = np.zeros(len(br), dtype=np.float32)
    for c in range(len(curve_len)):
        p0, p1 = starts[c], starts[c + 1]
        mean = br[p0:p1].mean()
        y[p0:p1] = (br[p0:p1] / mean - 1.0).astype(np.float32)
    out = np.zeros((len(freqs), 88), dtype=np.float64)
    y64 = y.astype(np.float64)
    t_mid = 0.5 * (tim.min() + tim.max())
    folds = [np.ones(len(tim), bool), tim < t_mid, ~(tim < t_mid)]
    for fi, f in enumerate(freqs):
        ph = tim * f
        frac = ph - np.floor(ph)
        bins = np.clip((frac * N_BINS).astype(np.int64), 0, N_BINS - 1)
        st = np.zeros((len(curve_len), 8))
        for c in range(len(curve_len)):
            p0, p1 = starts[c], starts[c + 1]
            bb = bins[p0:p1]
            cnt = np.bincount(bb, minlength=N_BINS)
            s1 = np.bincount(bb, weights=y64[p0:p1], minlength=N_BINS)
            s2 = np.bincount(bb, weights=y64[p0:p1] ** 2, minlength=N_BINS)
            st[c] = curve_stats(cnt, s1, s2)
        w = np.asarray(curve_len, dtype=np.float64)
        for k in range(8):
            v = st[:, k]
            srt = np.sort(v)
            out[fi, 8 * k:8 * k + 8] = [np.sum(w * v) / w.sum(), v.mean(), np.sqrt(max(np.mean(v * v) - v.mean() ** 2, 0)),
                                        srt[0], np.quantile(v, 0.25), np.quantile(v, 0.5), np.quantile(v, 0.75), srt[-1]]
        for k, sel in enumerate(folds):
            cnt = np.bincount(bins[sel], minlength=N_BINS)
            s1 = np.bincount(bins[sel], weights=y64[sel], minlength=N_BINS)
            s2 = np.bincount(bins[sel], weights=y64[sel] ** 2, minlength=N_BINS)
            out[fi, 64 + 8 * k:72 + 8 * k] = curve_stats(cnt, s1, s2)
    return out


def mlp_forward_backward(x, target, weights, biases, round_bf16=True):
    """Forward and backward of the screening MLP in float64, rounding to BF16
    exactly where the device pipeline does: the input, the weights, each
    hidden activation (the next layer's operand) and each layer's output
    gradient (the operand of the backward products).  Loss = mean squared
    error.  Returns (loss, predictions, weight gradients, bias gradients).
    round_bf16=False keeps everything in float64 (for finite differences)."""
    rnd = bf16_round if round_bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    L = len(weights)
    h = [np.asarray(rnd(x), dtype=np.float64)]
    wq = [np.asarray(rnd(w), dtype=np.float64) for w in weights]
    for l in range(L):
        z = h[-1] @ wq[l].T + biases[l]
        if l < L - 1:
            z = np.maximum(z, 0.0)
            h.append(np.asarray(rnd(z.astype(np.float32) if round_bf16 else z), dtype=np.float64))
        else:
            yhat = z[:, 0]
    n = len(target)
    loss = float(np.mean((yhat - target) ** 2))
    dz = (2.0 * (yhat - target) / n)[:, None]
    gw, gb = [None] * L, [None] * L
    for l in range(L - 1, -1, -1):
        gb[l] = dz.sum(0)
        dzq = np.asarray(rnd(dz.astype(np.float32) if round_bf16 else dz), dtype=np.float64)
        gw[l] = dzq.T @ h[l]
        if l > 0:
            dh = dzq @ wq[l]
            dz = np.where(h[l] > 0, dh, 0.0)
    return loss, yhat, gw, gb
