"""Seeded synthetic asteroid objects in the ``period_search_in`` format.

No public benchmark data ship with PeriodSearch (its AsteroidsAtHome test
workunits are not distributed), so every workload here is generated: a convex
body whose Gaussian-image curvature is exp(sum a_lm Y_lm), seen on circular
orbits (asteroid at ``r_ast`` AU, Earth at 1 AU) in several apparitions, with
Lambert + Lommel-Seeliger scattering and an exponential-linear phase function.
Relative curves are mean-normalised; calibrated points keep absolute scale.

The truth brightness is computed on a finer direction grid than any fit uses,
so a fit never sees its own discretisation.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np
from scipy.special import lpmv

JD_BASE = 2455000.5


@dataclasses.dataclass
class SynthConfig:
    l_max: int = 3
    m_max: int = 3
    nrows: int = 6
    n_dense: int = 20               # relative lightcurves
    dense_pts: tuple = (60, 60)     # points per dense curve (inclusive range)
    n_sparse: int = 0               # calibrated sparse points
    sparse_curves: int = 1          # calibrated curves the sparse points are split into
    noise_dense: float = 0.01
    noise_sparse: tuple = (0.02, 0.05)
    apparitions: int = 3
    n_freq: int = 200               # trial frequencies (if period_range is None)
    period_range: tuple | None = None   # (P_start, P_end) hours, else centred on truth
    period_step_coef: float | None = None
    stop_condition: float = 50.0
    n_iter_min: int = 10
    conw: float = 0.1
    r_ast: float = 2.0
    truth_grid: tuple = (60, 120)   # (theta, phi) cells of the direction grid the truth brightness sums over


C1 = SynthConfig()
C2 = SynthConfig(l_max=6, m_max=6, nrows=8, n_dense=40, dense_pts=(50, 120), n_sparse=400,
                 sparse_curves=2, period_range=(2.0, 100.0), n_freq=5000)
# The production object with relative lightcurves only (the form the
# reference's GPU code evaluates correctly: it skips the brightness of
# calibrated curves) on 200 trial frequencies around the true period.
C2_REL = dataclasses.replace(C2, n_sparse=0, period_range=None, n_freq=200, period_step_coef=3.0)

# Trailing "lc# weight" pair appended to inputs run by the reference app: its
# weight loop (period_search_BOINC.cpp:524-533) prints weightLc[lcNumber]
# after the final failed read, so lcNumber must have been set once.  Weight 1
# for curve 1 equals the default and changes nothing.
NEUTRAL_WEIGHT_LINE = "1 1.0\n"


def _basis(l_max, m_max, theta, phi):
    """Orthonormal real spherical harmonics in the reference's coefficient
    order (m = 0..m_max, l = m..l_max; cos then sin for m > 0)."""
    x = np.cos(theta)
    cols = []
    for m in range(m_max + 1):
        for l in range(m, l_max + 1):
            norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - m) / math.factorial(l + m))
            p = norm * lpmv(m, l, x) * (math.sqrt(2.0) if m else 1.0)
            cols.append(p * np.cos(m * phi))
            if m:
                cols.append(p * np.sin(m * phi))
    return np.stack(cols, axis=1)


def _truth_grid(n_theta=60, n_phi=120):
    th = (np.arange(n_theta) + 0.5) * math.pi / n_theta
    ph = (np.arange(n_phi) + 0.5) * 2 * math.pi / n_phi
    T, P = np.meshgrid(th, ph, indexing="ij")
    T, P = T.ravel(), P.ravel()
    dom = np.sin(T) * (math.pi / n_theta) * (2 * math.pi / n_phi)
    nrm = np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], axis=1)
    return T, P, dom, nrm


def _rot(axis, ang):
    c, s = math.cos(ang), math.sin(ang)
    if axis == "x":
        return np.array([[1, 0, 0], [0, c, -s], [0, s, c]])
    return np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]])


def generate(cfg: SynthConfig, seed: int):
    """Returns (text of period_search_in, truth dict)."""
    rng = np.random.default_rng(seed)
    # shape
    ncoef = sum((2 if m else 1) for m in range(cfg.m_max + 1) for _ in range(m, cfg.l_max + 1))
    ls = [l for m in range(cfg.m_max + 1) for l in range(m, cfg.l_max + 1) for _ in range(2 if m else 1)]
    coef = rng.normal(0.0, 1.0, ncoef) * np.sqrt(0.3 / (np.array(ls) + 1.0) ** 2)
    coef[0] = 0.0
    lam = rng.uniform(0, 2 * math.pi)
    beta = math.asin(rng.uniform(-1, 1))
    period_h = rng.uniform(4.0, 12.0)
    omega = 2 * math.pi * 24.0 / period_h   # rad/day
    phi0 = rng.uniform(0, 2 * math.pi)
    cl_true, pA, pD, pK = 0.1, 0.5, 0.1, -0.5

    T, P, dom, nrm = _truth_grid(*cfg.truth_grid)
    area = dom * np.exp(_basis(cfg.l_max, cfg.m_max, T, P) @ coef)

    # orbit geometry (ecliptic frame): asteroid circular orbit, inclined
    inc = math.radians(rng.uniform(2, 12))
    node = rng.uniform(0, 2 * math.pi)
    Rorb = _rot("z", node) @ _rot("x", inc)
    n_ast = 2 * math.pi / (365.25 * cfg.r_ast ** 1.5)
    n_e = 2 * math.pi / 365.25
    th_a0, th_e0 = rng.uniform(0, 2 * math.pi), rng.uniform(0, 2 * math.pi)

    def positions(t):
        ta = th_a0 + n_ast * t
        te = th_e0 + n_e * t
        pa = (Rorb @ np.stack([cfg.r_ast * np.cos(ta), cfg.r_ast * np.sin(ta), np.zeros_like(ta)])).T
        pe = np.stack([np.cos(te), np.sin(te), np.zeros_like(te)], axis=1)
        return pa, pe

    # oppositions: relative angle te - ta = 0 mod 2pi
    syn = 2 * math.pi / (n_e - n_ast)
    t_opp0 = ((th_a0 - th_e0) % (2 * math.pi)) / (n_e - n_ast)
    opps = [t_opp0 + k * syn for k in range(cfg.apparitions)]

    Bpole = np.array([math.cos(beta) * math.cos(lam), math.cos(beta) * math.sin(lam), math.sin(beta)])

    def body_frame(t, v):
        # ecliptic -> body: rotate so the pole is z, then spin by omega t + phi0
        cb, sb, cl_, sl = math.cos(math.pi / 2 - beta), math.sin(math.pi / 2 - beta), math.cos(lam), math.sin(lam)
        B = np.array([[cb * cl_, cb * sl, -sb], [-sl, cl_, 0], [sb * cl_, sb * sl, cb]])
        f = omega * t + phi0
        c, s = np.cos(f), np.sin(f)
        vb = v @ B.T
        out = np.empty_like(vb)
        out[:, 0] = c * vb[:, 0] + s * vb[:, 1]
        out[:, 1] = -s * vb[:, 0] + c * vb[:, 1]
        out[:, 2] = vb[:, 2]
        return out

    def brightness(t, e_sun, e_obs):
        es = body_frame(t, e_sun)
        eo = body_frame(t, e_obs)
        mu = eo @ nrm.T
        mu0 = es @ nrm.T
        vis = (mu > 0) & (mu0 > 0)
        mu = np.where(vis, mu, 0.0)
        mu0 = np.where(vis, mu0, 0.0)
        den = np.where(vis, mu + mu0, 1.0)
        S = mu * mu0 * (cl_true + 1.0 / den)
        L = S @ area
        alpha = np.arccos(np.clip(np.sum(e_sun * e_obs, axis=1), -1, 1))
        return L * (1 + pA * np.exp(-alpha / pD) + pK * alpha), alpha

    curves = []  # (times, bright, e_sun_vec, e_obs_vec, rel)

    def geometry(t):
        pa, pe = positions(t)
        sun = -pa
        obs = pe - pa
        return sun, obs

    jd_nights = []
    for i in range(cfg.n_dense):
        app = opps[i % cfg.apparitions]
        for _ in range(1000):
            tn = app + rng.uniform(-70, 70)
            sun, obs = geometry(np.array([tn]))
            a = math.degrees(math.acos(np.clip(np.dot(sun[0], obs[0]) / np.linalg.norm(sun[0]) / np.linalg.norm(obs[0]), -1, 1)))
            if 2.0 <= a <= 30.0:
                break
        jd_nights.append(tn)
    jd_nights.sort()
    for tn in jd_nights:
        npt = int(rng.integers(cfg.dense_pts[0], cfg.dense_pts[1] + 1))
        dur = rng.uniform(4.0, 8.0) / 24.0
        t = tn + np.sort(rng.uniform(0, dur, npt))
        sun, obs = geometry(t)
        L, _ = brightness(t, sun / np.linalg.norm(sun, axis=1)[:, None], obs / np.linalg.norm(obs, axis=1)[:, None])
        L = L * (1 + cfg.noise_dense * rng.standard_normal(npt))
        L = L / L.mean()
        curves.append((t, L, sun, obs, 1))

    if cfg.n_sparse:
        per = [cfg.n_sparse // cfg.sparse_curves] * cfg.sparse_curves
        per[-1] += cfg.n_sparse - sum(per)
        span0, span1 = opps[0] - 80, opps[-1] + 80
        for k, npt in enumerate(per):
            noise = rng.uniform(*cfg.noise_sparse)
            ts = []
            while len(ts) < npt:
                tc = rng.uniform(span0, span1)
                sun, obs = geometry(np.array([tc]))
                a = math.degrees(math.acos(np.clip(np.dot(sun[0], obs[0]) / np.linalg.norm(sun[0]) / np.linalg.norm(obs[0]), -1, 1)))
                if 2.0 <= a <= 30.0:
                    ts.append(tc)
            t = np.sort(np.array(ts))
            sun, obs = geometry(t)
            L, _ = brightness(t, sun / np.linalg.norm(sun, axis=1)[:, None], obs / np.linalg.norm(obs, axis=1)[:, None])
            L = L * (1 + noise * rng.standard_normal(npt))
            curves.append((t, L, sun, obs, 0))

    tmin = min(c[0].min() for c in curves)
    tmax = max(c[0].max() for c in curves)
    span = tmax - tmin
    if cfg.period_range is None:
        coef_step = 0.8 if cfg.period_step_coef is None else cfg.period_step_coef
        df = 0.5 / span / 24 * coef_step
        f0 = 1.0 / period_h
        half = (cfg.n_freq - 1) / 2.0 + 0.25
        p_start, p_end = 1.0 / (f0 + half * df), 1.0 / (f0 - half * df)
    else:
        p_start, p_end = cfg.period_range
        if cfg.period_step_coef is None:
            df = (1 / p_start - 1 / p_end) / (cfg.n_freq - 0.5)
            coef_step = df * span * 24 / 0.5
        else:
            coef_step = cfg.period_step_coef

    lines = []
    lines.append(f"{p_start:.10f} {coef_step:.10f} {p_end:.10f} 1  period start/step/stop (free)")
    lines.append("0  epoch of zero time t0")
    lines.append("0  initial fixed rotation angle fi0")
    lines.append(f"{cfg.conw}  the weight factor for conv. reg.")
    lines.append(f"{cfg.l_max} {cfg.m_max}  degree and order of the Laplace series")
    lines.append(f"{cfg.nrows}  nr. of triangulation rows per octant")
    lines.append("0.5 1  initial guesses for phase funct. params.")
    lines.append("0.1 1")
    lines.append("-0.5 1")
    lines.append("0.1 1  initial Lambert coeff. (L-S=1)")
    lines.append(f"{cfg.stop_condition:g}  stop condition")
    lines.append(f"{cfg.n_iter_min}  minimum number of iterations")
    lines.append("10  Alamda multiplicative factor")
    lines.append("0.0001  initial Alamda")
    lines.append(f"{len(curves)}")
    for (t, L, sun, obs, rel) in curves:
        lines.append(f"{len(t)} {0 if rel else 1}")
        for k in range(len(t)):
            s, o = sun[k], obs[k]
            lines.append(f"{JD_BASE + t[k]:.8f} {L[k]:.10e} {s[0]:.10f} {s[1]:.10f} {s[2]:.10f} "
                         f"{o[0]:.10f} {o[1]:.10f} {o[2]:.10f}")
    text = "\n".join(lines) + "\n"
    truth = dict(period_h=period_h, lambda_deg=math.degrees(lam) % 360, beta_deg=math.degrees(beta),
                 coef=coef, phi0=phi0, n_points=sum(len(c[0]) for c in curves),
                 n_curves=len(curves), p_start=p_start, p_end=p_end, step_coef=coef_step)
    return text, truth


def write(cfg: SynthConfig, seed: int, path: str):
    text, truth = generate(cfg, seed)
    with open(path, "w") as f:
        f.write(text)
    return truth


def config3_object(i: int, seed0: int = 1000003 * 3):
    """Object i of the batched workload: points log-uniform in 300..19 900
    (relative curves of equal length, at most 199 of them -- with the
    pseudo-curve the reference's MAX_LC of 200), lmax = mmax in {4, 6, 8},
    nrows in {6, 8, 10}, trial-frequency count log-uniform in 500..20 000
    around the true period, stop condition 0.005 (fits run until the rms
    improves by less than that: ragged iteration counts).  Returns
    (SynthConfig, seed)."""
    rng = np.random.default_rng(seed0 + i)
    n_pts = int(round(math.exp(rng.uniform(math.log(300), math.log(19900)))))
    lmax = int(rng.choice([4, 6, 8]))
    nrows = int(rng.choice([6, 8, 10]))
    n_freq = int(round(math.exp(rng.uniform(math.log(500), math.log(20000)))))
    n_curves = min(199, max(5, n_pts // 80))
    per = max(1, n_pts // n_curves)
    # the truth sums over 30 x 60 directions (1800, still finer than the
    # fits' 288-800 facets) to keep generating 64 objects short
    cfg = SynthConfig(l_max=lmax, m_max=lmax, nrows=nrows, n_dense=n_curves, dense_pts=(per, per),
                      n_freq=n_freq, stop_condition=0.005, n_iter_min=10, truth_grid=(30, 60))
    return cfg, seed0 + i


C3_OBJECTS = 64


def config3_object(i: int, seed0: int = 1000003 * 3):
    """Object i of the batched workload: points log-uniform in 300..19 900
    (relative curves of equal length, at most 199 of them -- with the
    pseudo-curve the reference's MAX_LC of 200), lmax = mmax in {4, 6, 8},
    nrows in {6, 8, 10}, trial-frequency count log-uniform in 500..20 000
    around the true period, stop condition 0.005 (fits run until the rms
    improves by less than that: ragged iteration counts).  Returns
    (SynthConfig, seed)."""
    rng = np.random.default_rng(seed0 + i)
    n_pts = int(round(math.exp(rng.uniform(math.log(300), math.log(19900)))))
    lmax = int(rng.choice([4, 6, 8]))
    nrows = int(rng.choice([6, 8, 10]))
    n_freq = int(round(math.exp(rng.uniform(math.log(500), math.log(20000)))))
    n_curves = min(199, max(5, n_pts // 80))
    per = max(1, n_pts // n_curves)
    # the truth sums over 30 x 60 directions (1800, still finer than the
    # fits' 288-800 facets) to keep generating 64 objects short
    cfg = SynthConfig(l_max=lmax, m_max=lmax, nrows=nrows, n_dense=n_curves, dense_pts=(per, per),
                      n_freq=n_freq, stop_condition=0.005, n_iter_min=10, truth_grid=(30, 60))
    return cfg, seed0 + i


C3_OBJECTS = 64

# The two inputs both the reference's own GPU application and this project's
# host program are run on (golden files, parity tests, the bench's
# reference_gpu leg): BASELINE config 1 object 0 and the relative-only
# production object, each with the neutral trailing weight line.
REFERENCE_INPUTS = {"c1": (C1, 1000003 * 1), "c2rel": (C2_REL, 1000003 * 2)}


def reference_input_text(name: str, one_freq: bool = False, stop: float | None = None,
                         n_freq: int | None = None) -> str:
    """period_search_in text of REFERENCE_INPUTS[name].  one_freq=True sets
    period end = period start, a grid of one frequency (its wall time is the
    program's fixed cost: start-up, tables and the convexity-weight search);
    n_freq moves the period end so the same grid (same start and step) holds
    n_freq frequencies; stop replaces the stop condition (e.g. 5: exactly 5
    LM iterations per fit)."""
    cfg, seed = REFERENCE_INPUTS[name]
    text, _ = generate(cfg, seed)
    first, rest = text.split("\n", 1)
    p = first.split()
    if one_freq:
        p[2] = p[0]
    elif n_freq is not None:
        from .objects import scan_grid

        g = scan_grid(text)
        p[2] = "%.17g" % (1.0 / (g.freq_start - (n_freq - 0.5) * g.freq_step))
    text = "%s %s %s %s  period start/step/stop (free)\n%s" % (p[0], p[1], p[2], p[3], rest)
    if stop is not None:
        lines = text.splitlines(True)
        k = [i for i, l in enumerate(lines) if "stop condition" in l][0]
        lines[k] = "%g  stop condition\n" % stop
        text = "".join(lines)
    return text + NEUTRAL_WEIGHT_LINE
