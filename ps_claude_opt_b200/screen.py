"""Learned frequency screening: rank an object's trial frequencies by the chi^2
a small BF16 network predicts from phase-folded lightcurve features, fit the
top-ranked share plus a random audit sample with the plain LM, and keep the
best line of what was fitted.

No counterpart in the reference, which fits every trial frequency; the full
scan (native.run_object) stays the fallback and the judge of the screen.
All device work runs in the library's own kernels (csrc/screen.cu): the
feature kernel, BF16 tensor-core GEMMs, the ReLU backward, column sums and
Adam.  PyTorch only holds the device buffers.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native

import os

MODEL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "screen_model.bin")
MODEL_MAGIC = b"PSMLP001"
N_FEATURES = 88
SIZES = (N_FEATURES, 256, 256, 256, 1)   # features -> 3 x 256 hidden -> predicted log rms


def _lib():
    return native.lib()


def frequencies(obj, n_start=1, n=None):
    """Trial frequencies of the object's grid, 1/hour (the reference's unit)."""
    g = obj.grid
    n = g.n_max - n_start + 1 if n is None else n
    return g.freq_start - (np.arange(n_start, n_start + n) - 1) * g.freq_step


def features(obj, freqs, device=0):
    """[len(freqs), 88] float32 features of trial frequencies given in 1/hour
    (the lightcurve times are in days: the kernel folds at 24 f)."""
    freqs = np.ascontiguousarray(24.0 * np.asarray(freqs, dtype=np.float64))
    out = np.zeros((len(freqs), N_FEATURES), dtype=np.float32)
    tim = np.ascontiguousarray(obj.tim, dtype=np.float64)
    br = np.ascontiguousarray(obj.brightness, dtype=np.float64)
    cl = np.ascontiguousarray(obj.curve_len, dtype=np.int32)
    cr = np.ascontiguousarray(obj.curve_rel, dtype=np.int32)
    curves = native.Curves(len(cl), cl.ctypes.data_as(C.POINTER(C.c_int32)), cr.ctypes.data_as(C.POINTER(C.c_int32)))
    native._check(_lib().ps_screen_features(device, len(tim), tim.ctypes.data_as(C.POINTER(C.c_double)),
                                            br.ctypes.data_as(C.POINTER(C.c_double)), C.byref(curves), len(freqs),
                                            freqs.ctypes.data_as(C.POINTER(C.c_double)),
                                            out.ctypes.data_as(C.POINTER(C.c_float))))
    return out


def normalise(feat):
    """Per-object standardisation of each feature over the object's
    frequencies (in float64, as ps_screen_rank does): the network ranks
    frequencies within one object."""
    f = np.asarray(feat, dtype=np.float64)
    mu = f.mean(0)
    sd = np.sqrt(((f - mu) ** 2).mean(0))
    return ((f - mu) / np.where(sd > 1e-6, sd, 1.0)).astype(np.float32)


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class Mlp:
    """The screening network on the device: BF16 weights and activations for
    the tensor cores, FP32 master weights, Adam moments and gradients."""

    def __init__(self, sizes=SIZES, seed=0, device="cuda"):
        import torch

        self.torch = torch
        self.sizes = tuple(sizes)
        self.device = device
        rng = np.random.default_rng(seed)
        self.W, self.b, self.Wb = [], [], []
        for k, n in zip(self.sizes[:-1], self.sizes[1:]):
            w = rng.standard_normal((n, k)).astype(np.float32) * np.float32(np.sqrt(2.0 / k))
            self.W.append(torch.from_numpy(w).to(device))
            self.b.append(torch.zeros(n, dtype=torch.float32, device=device))
            self.Wb.append(torch.empty((n, k), dtype=torch.bfloat16, device=device))
        self.mW = [torch.zeros_like(w) for w in self.W]
        self.vW = [torch.zeros_like(w) for w in self.W]
        self.mb = [torch.zeros_like(b) for b in self.b]
        self.vb = [torch.zeros_like(b) for b in self.b]
        self.steps = 0
        self._sync_bf16()

    def _stream(self):
        return C.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    def _sync_bf16(self):
        for w, wb in zip(self.W, self.Wb):
            native._check(_lib().ps_to_bf16(w.numel(), _ptr(w), _ptr(wb), self._stream()))

    def forward(self, xb):
        """xb: [B, N_FEATURES] bfloat16 on the device.  Returns predictions [B] (FP32)
        and keeps the activations for backward."""
        torch = self.torch
        if xb.dim() != 2 or xb.shape[1] != self.sizes[0] or xb.dtype != torch.bfloat16 or not xb.is_contiguous():
            raise ValueError("Mlp.forward: input must be a contiguous [B, %d] bfloat16 tensor" % self.sizes[0])
        B = xb.shape[0]
        self.hb, self.hf = [xb], [None]
        L = len(self.W)
        for l in range(L):
            n, k = self.W[l].shape
            last = l == L - 1
            hf = torch.empty((B, n), dtype=torch.float32, device=self.device)
            hb = None if last else torch.empty((B, n), dtype=torch.bfloat16, device=self.device)
            native._check(_lib().ps_gemm_bf16(B, n, k, _ptr(self.hb[-1]), k, 1, _ptr(self.Wb[l]), 1, k, _ptr(hf), n,
                                              0, _ptr(self.b[l]), 0 if last else 1, _ptr(hb), n, self._stream()))
            self.hf.append(hf)
            self.hb.append(hb)
        return self.hf[-1][:, 0]

    def backward(self, dyhat):
        """dyhat: [B] FP32 loss gradient of the predictions.  Returns the
        gradients (weights, biases), FP32."""
        torch = self.torch
        B = dyhat.shape[0]
        if dyhat.dim() != 1 or B != self.hb[0].shape[0] or dyhat.dtype != torch.float32:
            raise ValueError("Mlp.backward: gradient must be FP32 [B] for the last forward batch")
        L = len(self.W)
        dz = dyhat.reshape(B, 1).contiguous()
        dzb = torch.empty((B, 1), dtype=torch.bfloat16, device=self.device)
        native._check(_lib().ps_to_bf16(B, _ptr(dz), _ptr(dzb), self._stream()))
        gW, gb = [None] * L, [None] * L
        for l in range(L - 1, -1, -1):
            n, k = self.W[l].shape
            gW[l] = torch.empty((n, k), dtype=torch.float32, device=self.device)
            gb[l] = torch.empty(n, dtype=torch.float32, device=self.device)
            native._check(_lib().ps_gemm_bf16(n, k, B, _ptr(dzb), 1, n, _ptr(self.hb[l]), k, 1, _ptr(gW[l]), k, 0,
                                              None, 0, None, 0, self._stream()))
            native._check(_lib().ps_column_sum(B, n, _ptr(dz), _ptr(gb[l]), self._stream()))
            if l > 0:
                dh = torch.empty((B, k), dtype=torch.float32, device=self.device)
                native._check(_lib().ps_gemm_bf16(B, k, n, _ptr(dzb), n, 1, _ptr(self.Wb[l]), k, 1, _ptr(dh), k, 0,
                                                  None, 0, None, 0, self._stream()))
                dz = torch.empty((B, k), dtype=torch.float32, device=self.device)
                dzb = torch.empty((B, k), dtype=torch.bfloat16, device=self.device)
                native._check(_lib().ps_relu_backward(B * k, _ptr(dh), _ptr(self.hf[l]), _ptr(dz), _ptr(dzb),
                                                      self._stream()))
        return gW, gb

    def adam(self, gW, gb, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        self.steps += 1
        for l in range(len(self.W)):
            native._check(_lib().ps_adam_step(self.W[l].numel(), _ptr(self.W[l]), _ptr(gW[l]), _ptr(self.mW[l]),
                                              _ptr(self.vW[l]), lr, beta1, beta2, eps, self.steps,
                                              _ptr(self.Wb[l]), self._stream()))
            native._check(_lib().ps_adam_step(self.b[l].numel(), _ptr(self.b[l]), _ptr(gb[l]), _ptr(self.mb[l]),
                                              _ptr(self.vb[l]), lr, beta1, beta2, eps, self.steps, None,
                                              self._stream()))

    def train_step(self, xb, y, lr=1e-3):
        """One Adam step on the mean squared error; returns the loss."""
        yhat = self.forward(xb)
        diff = yhat - y
        loss = float((diff * diff).mean())
        gW, gb = self.backward((2.0 / len(y)) * diff)
        self.adam(gW, gb, lr)
        return loss

    def predict(self, feat):
        torch = self.torch
        x = torch.from_numpy(np.ascontiguousarray(feat, dtype=np.float32)).to(self.device).to(torch.bfloat16)
        out = []
        for i in range(0, x.shape[0], 8192):
            out.append(self.forward(x[i:i + 8192]).cpu().numpy())
        return np.concatenate(out)

    def state(self):
        d = {"sizes": np.array(self.sizes)}
        for l in range(len(self.W)):
            d[f"W{l}"] = self.W[l].cpu().numpy()
            d[f"b{l}"] = self.b[l].cpu().numpy()
        return d

    @classmethod
    def from_state(cls, d, device="cuda"):
        net = cls(tuple(int(v) for v in d["sizes"]), device=device)
        for l in range(len(net.W)):
            net.W[l].copy_(net.torch.from_numpy(np.asarray(d[f"W{l}"], dtype=np.float32)))
            net.b[l].copy_(net.torch.from_numpy(np.asarray(d[f"b{l}"], dtype=np.float32)))
        net._sync_bf16()
        return net


def _lcg_uniform(seed, n):
    """n uniform integers in [0, 2^31) from the 64-bit linear congruential
    generator x <- 6364136223846793005 x + 1442695040888963407 (the host
    program draws the same audit sample)."""
    x = (int(seed) * 2654435761 + 1) & 0xFFFFFFFFFFFFFFFF
    out = []
    for _ in range(n):
        x = (6364136223846793005 * x + 1442695040888963407) & 0xFFFFFFFFFFFFFFFF
        out.append(x >> 33)
    return out


AUDIT_MARGIN = 0.10     # an audit line within 10 % of the screened best rms (the validator's rms envelope)
EDGE_WIDTH = 2          # frequencies fitted on each side of a best line that sits at the edge of a fitted run
MAX_EXPANSIONS = 8      # edge expansions before the scan falls back to the full grid
POLISH_MINIMA = 8       # mixed-precision scans: lowest local minima refitted in FP64 (with +-1 neighbours)
POLISH_ROUNDS = 4       # ... and at most this many rounds of FP64 refits around a moving best line


def select_parts(pred, top=0.034, halo=1, audit=0.02, seed=0):
    """(core, audit) frequency index sets (0-based) of a screened scan: the
    `top` share with the lowest predicted rms, each with `halo` neighbours on
    either side (an LM minimum in frequency is a few grid steps wide, finer
    than the folded features resolve), and an `audit` share drawn uniformly
    from the rest."""
    n = len(pred)
    k = max(1, int(round(top * n)))
    order = np.argsort(np.asarray(pred), kind="stable")
    chosen = set()
    for i in order[:k].tolist():
        for d in range(-halo, halo + 1):
            if 0 <= i + d < n:
                chosen.add(i + d)
    rest = [i for i in range(n) if i not in chosen]
    na = min(len(rest), max(1, int(round(audit * n))))
    # partial Fisher-Yates shuffle of the rest, driven by the LCG
    for j, r in enumerate(_lcg_uniform(seed, na)):
        pick = j + r % (len(rest) - j)
        rest[j], rest[pick] = rest[pick], rest[j]
    return chosen, set(rest[:na])


def select(pred, top=0.034, halo=1, audit=0.02, seed=0):
    """Frequency indices (0-based, sorted) a screened scan fits first: the
    core and the audit sample of select_parts.  The defaults fit at most
    12.2 % of the grid."""
    core, aud = select_parts(pred, top, halo, audit, seed)
    return np.array(sorted(core | aud), dtype=np.int64)


class Plan:
    """Outcome of a screened scan: the frequencies fitted (0-based, sorted),
    their rms, and how the scan got there."""

    def __init__(self, n):
        self.n = n
        self.rms = {}            # frequency -> best rms over the poles (NaN kept)
        self.initial = 0         # frequencies of the first selection
        self.expansions = 0      # edge expansions
        self.alias_probes = 0    # best lines whose period-doubling partners were fitted
        self.fallback = False    # the whole grid was fitted
        self.reason = ""         # why it fell back: "audit" or "edge"
        self.first_pass = 0      # frequencies fitted before any FP64 refit
        self.polished = 0        # mixed precision: frequencies refitted in FP64
        self.polish_rounds = 0

    @property
    def fitted(self):
        return sorted(self.rms)

    def best(self):
        """Lowest-rms fitted frequency (NaN never wins; the first minimum wins ties)."""
        b, br = -1, np.inf
        for i in self.fitted:
            r = self.rms[i]
            if r < br:
                b, br = i, r
        return b


def alias_indices(freqs, b):
    """0-based grid indices nearest the period-doubling partners of frequency
    index b (twice and half its frequency) that lie on the grid."""
    f0, df = float(freqs[0]), float(freqs[0] - freqs[1]) if len(freqs) > 1 else 0.0
    if df <= 0:
        return []
    out = []
    for t in (2.0 * freqs[b], 0.5 * freqs[b]):
        i = int(round((f0 - t) / df))
        if 0 <= i < len(freqs):
            out.append(i)
    return out


def plan_scan(pred, fit, top=0.034, halo=1, audit=0.02, seed=0, margin=AUDIT_MARGIN, edge=EDGE_WIDTH,
              max_expansions=MAX_EXPANSIONS, freqs=None):
    """The screened scan's control flow, independent of the device.

    fit(indices) fits the given 0-based frequencies (all poles) and returns
    each one's best rms.  Steps:
      1. fit the core (top-ranked share with halo) and the audit sample;
      2. while the best line sits at the edge of a fitted run (a neighbour is
         unfitted), fit `edge` more frequencies on each side of it -- at most
         `max_expansions` times, then fall back;
      3. with the grid's frequencies given (freqs), fit the neighbourhoods
         (+-edge) of the best line's period-doubling partners, twice and half
         its frequency -- a double-peaked lightcurve fits almost as well at
         twice its period, so the ranking can put the wrong one of the pair
         first -- and return to step 2 if one of them wins; each best line is
         probed once;
      4. judge by the audit sample: if an audit frequency away from the best
         line's neighbourhood comes within `margin` (relative) of the best
         rms, the network's ranking is not trustworthy for this object and
         the scan falls back;
      5. on fallback, fit every remaining frequency: the result is then the
         full scan's.
    Returns a Plan."""
    n = len(pred)
    plan = Plan(n)
    core, aud = select_parts(pred, top, halo, audit, seed)

    def run(idx):
        idx = sorted(i for i in set(idx) if 0 <= i < n and i not in plan.rms)
        if idx:
            for i, r in zip(idx, fit(np.array(idx, dtype=np.int64))):
                plan.rms[i] = float(r)

    run(core | aud)
    plan.initial = len(plan.rms)
    probed = set()
    while not plan.fallback:
        while True:
            b = plan.best()
            if b < 0:
                plan.fallback, plan.reason = True, "edge"
                break
            need = [j for j in (b - 1, b + 1) if 0 <= j < n and j not in plan.rms]
            if not need:
                break
            if plan.expansions >= max_expansions:
                plan.fallback, plan.reason = True, "edge"
                break
            run(range(b - edge, b + edge + 1))
            plan.expansions += 1
        if plan.fallback or freqs is None:
            break
        b = plan.best()
        if b in probed:
            break
        probed.add(b)
        around = set()
        for a in alias_indices(freqs, b):
            around.update(range(a - edge, a + edge + 1))
        run(around)
        plan.alias_probes += 1
        if plan.best() == b:
            break
    if not plan.fallback:
        b = plan.best()
        br = plan.rms[b]
        for a in aud:
            if abs(a - b) > edge and plan.rms.get(a, np.inf) <= br * (1.0 + margin):
                plan.fallback, plan.reason = True, "audit"
                break
    if plan.fallback:
        run(range(n))
    return plan


def polish_plan(plan, fit64, freqs, edge=EDGE_WIDTH, minima=POLISH_MINIMA, rounds=POLISH_ROUNDS):
    """FP64 decision for a scan whose fits ran in mixed precision.

    FP32 facet sums move a fit's rms at the 1e-3 level, enough to reorder
    two nearly equal minima -- most often a period and its double, which a
    double-peaked lightcurve fits almost equally well.  So the candidates
    are refitted in FP64 (fit64(indices) returns their best rms, and the
    caller replaces their lines): in the first round the `minima` lowest
    local minima of the rms over the fitted frequencies (an unfitted or NaN
    neighbour counts as higher) with one neighbour on either side; in every
    round the best line with `edge` neighbours on either side and the same
    neighbourhoods of its period-doubling partners (twice and half its
    frequency).  Rounds repeat while they add frequencies -- the best line
    can move to a refitted one -- at most `rounds` times.  Refitted
    frequencies may include ones the screen had not fitted; they become
    fitted lines.  Updates plan.rms, plan.polished, plan.polish_rounds."""
    n = plan.n
    done = set()

    def key(i):
        r = plan.rms.get(i, np.inf)
        return np.inf if np.isnan(r) else r

    for rnd in range(rounds):
        b = plan.best()
        if b < 0:
            break
        need = set(range(b - edge, b + edge + 1))
        for a in alias_indices(freqs, b):
            need.update(range(a - edge, a + edge + 1))
        if rnd == 0:
            loc = [i for i in plan.fitted if key(i) < np.inf and key(i) <= key(i - 1) and key(i) <= key(i + 1)]
            loc.sort(key=lambda i: (key(i), i))
            for i in loc[:minima]:
                need.update((i - 1, i, i + 1))
        need = sorted(i for i in need if 0 <= i < n and i not in done)
        if not need:
            break
        for i, r in zip(need, fit64(np.array(need, dtype=np.int64))):
            plan.rms[i] = float(r)
        done.update(need)
        plan.polished = len(done)
        plan.polish_rounds = rnd + 1
    return plan


def _best_pole_lines(obj, idx, res):
    """One line per frequency from the 10 poles' results, as the reference
    prints it (start_CUDA.cu:1200-1229): NaN-safe, the earliest pole wins ties."""
    lines = np.zeros((len(idx), 6))
    for q in range(len(idx)):
        r = res[q]
        best = -1
        for p in range(native.N_POLES):
            if best < 0 or (not np.isnan(r[p, 0]) and not (r[p, 0] >= r[best, 0])):
                best = p
        b = r[best]
        lines[q] = (24 * b[2], b[0], b[0] * b[0] * obj.n_points, b[1], b[3], b[4])
    return lines


def screened_scan(obj, net, conw_r, top=0.034, halo=1, audit=0.02, seed=0, device=0,
                  precision=native.PRECISION_FP64, margin=AUDIT_MARGIN, pred=None, polish=True):
    """Fits the screened frequencies (after the convexity-weight search,
    whose conw_r is passed in), expanding around a best line at the edge of
    a fitted run, probing its period-doubling partners and falling back to
    the whole grid when the audit sample contradicts the ranking
    (plan_scan); in mixed precision the candidate lines are then refitted
    in FP64 (polish_plan; polish=False leaves them mixed).  Returns (frequency indices
    1-based, lines, per-fit results [n, 10, 6], Plan)."""
    if pred is None:
        pred = net.predict(normalise(features(obj, frequencies(obj), device)))
    store = {}
    with native.Engine(obj, device) as eng:
        eng.set_precision(precision)
        eng.configure(conw_r=conw_r)

        def fit(idx0):
            nf = np.repeat(idx0 + 1, native.N_POLES).astype(np.int32)
            pl = np.tile(np.arange(native.N_POLES), len(idx0)).astype(np.int32)
            res, _, _ = eng.fit_items(nf, pl)
            res = res.reshape(len(idx0), native.N_POLES, 6)
            lines = _best_pole_lines(obj, idx0, res)
            for i, q in enumerate(idx0.tolist()):
                store[q] = (res[i], lines[i])
            return lines[:, 1]

        plan = plan_scan(pred, fit, top, halo, audit, seed, margin, freqs=frequencies(obj))
        plan.first_pass = len(plan.rms)
        if precision == native.PRECISION_MIXED and polish:
            # the candidates' final fits in FP64 (polish_plan)
            eng.set_precision(native.PRECISION_FP64)
            eng.configure(conw_r=conw_r)
            polish_plan(plan, fit, frequencies(obj))
    idx = np.array(plan.fitted, dtype=np.int64)
    res = np.stack([store[i][0] for i in idx])
    lines = np.stack([store[i][1] for i in idx])
    return idx + 1, lines, res, plan


def best_line(lines):
    """Index of the lowest-rms line (NaN lines never win)."""
    r = np.where(np.isnan(lines[:, 1]), np.inf, lines[:, 1])
    return int(np.argmin(r))


def save_model(path, state):
    """Writes a network state as MODEL_MAGIC, int32 layer count, int32 sizes,
    then per layer float32 weights [out][in] and biases [out]
    (little-endian) -- the layout ps_screen_rank takes."""
    sizes = [int(v) for v in state["sizes"]]
    with open(path, "wb") as f:
        f.write(MODEL_MAGIC)
        np.array([len(sizes) - 1] + sizes, dtype="<i4").tofile(f)
        for l in range(len(sizes) - 1):
            np.asarray(state[f"W{l}"], dtype="<f4").tofile(f)
            np.asarray(state[f"b{l}"], dtype="<f4").tofile(f)


def read_model(path=MODEL_PATH):
    """(sizes, flat float32 parameters, state dict) of a model file."""
    with open(path, "rb") as f:
        if f.read(8) != MODEL_MAGIC:
            raise ValueError("not a screening model file: " + path)
        nl = int(np.fromfile(f, dtype="<i4", count=1)[0])
        sizes = np.fromfile(f, dtype="<i4", count=nl + 1)
        params = np.fromfile(f, dtype="<f4")
    state, off = {"sizes": sizes}, 0
    for l in range(nl):
        n, k = int(sizes[l + 1]), int(sizes[l])
        state[f"W{l}"] = params[off:off + n * k].reshape(n, k)
        off += n * k
        state[f"b{l}"] = params[off:off + n]
        off += n
    if off != len(params):
        raise ValueError("screening model file size does not match its layer sizes: " + path)
    return sizes, params, state


def load_model(path=MODEL_PATH, device="cuda"):
    """The trained screening network (written by screen_train)."""
    return Mlp.from_state(read_model(path)[2], device=device)


def rank(obj, path=MODEL_PATH, device=0):
    """Scores of all grid frequencies through the C ABI (ps_screen_rank)."""
    sizes, params, _ = read_model(path)
    freqs = np.ascontiguousarray(frequencies(obj), dtype=np.float64)
    score = np.zeros(len(freqs), dtype=np.float32)
    tim = np.ascontiguousarray(obj.tim, dtype=np.float64)
    br = np.ascontiguousarray(obj.brightness, dtype=np.float64)
    cl = np.ascontiguousarray(obj.curve_len, dtype=np.int32)
    cr = np.ascontiguousarray(obj.curve_rel, dtype=np.int32)
    curves = native.Curves(len(cl), cl.ctypes.data_as(C.POINTER(C.c_int32)), cr.ctypes.data_as(C.POINTER(C.c_int32)))
    sz = np.ascontiguousarray(sizes, dtype=np.int32)
    native._check(native.lib().ps_screen_rank(device, len(tim), native._p(tim), native._p(br), C.byref(curves),
                                              len(freqs), native._p(freqs), len(sz) - 1,
                                              sz.ctypes.data_as(C.POINTER(C.c_int32)),
                                              params.ctypes.data_as(C.POINTER(C.c_float)),
                                              score.ctypes.data_as(C.POINTER(C.c_float))))
    return score
