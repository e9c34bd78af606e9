"""Reading ``period_search_in`` and preparing one object for the fit engine.

Mirrors the host part of PeriodSearch's ``main`` (period_search_BOINC.cpp):
input parsing (:343-533), epoch and weights (:537-571), the initial ellipsoid
scale (:573-585), the ``ia`` mask (:843-857, start_CUDA.cu:850-853), the stop
condition (start_CUDA.cu:855-869) and the frequency grid (:839-841).  The
shape tables come from the native setup in the extension library
(``ps_setup_shape``), a restatement of trifac/areanorm/sphfunc/ellfit.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

PI = 3.14159265358979323846
DEG2RAD = PI / 180
MAX_N_ITER = 60
LAMBDA_POLES = (0, 90, 180, 270, 60, 180, 300, 60, 180, 300)   # period_search_BOINC.cpp:229-238
BETA_POLES = (0, 0, 0, 0, 60, 60, 60, -60, -60, -60)


def n_coef(l_max: int, m_max: int) -> int:
    return sum((2 if m else 1) for m in range(m_max + 1) for _ in range(m, l_max + 1))


@dataclasses.dataclass
class ScanGrid:
    freq_start: float
    freq_end: float
    freq_step: float

    @property
    def n_max(self) -> int:
        return int((self.freq_start - self.freq_end) / self.freq_step) + 1


@dataclasses.dataclass
class PreparedObject:
    # data
    n_points: int
    n_curves: int
    curve_len: np.ndarray
    curve_rel: np.ndarray
    tim: np.ndarray
    ee: np.ndarray
    ee0: np.ndarray
    brightness: np.ndarray
    sig: np.ndarray
    sigr2: np.ndarray
    weight: np.ndarray
    # shape model
    l_max: int
    m_max: int
    nrows: int
    n_fac: int
    n_coef: int
    normal: np.ndarray
    d_area: np.ndarray
    dsph: np.ndarray
    cg_first: np.ndarray
    # fit constants
    phi0: float
    par: np.ndarray
    lcl: float                # ln(cl), the fitted Lambert parameter's start value
    cl: float                 # Lambert coefficient as read
    alamda_start: float
    alamda_incr: float
    alamda_incrr: float
    beta_pole: np.ndarray
    lambda_pole: np.ndarray
    ia: np.ndarray            # 1-based, length ma + 1
    n_iter_max: int
    n_iter_min: int
    iter_diff_max: float
    stop_condition: float     # as read: > 1 fixed iteration count, < 1 rms-improvement threshold
    conw_r: float             # initial conw / escl^2
    escl: float
    grid: ScanGrid
    onlyrel: bool

    @property
    def ma(self) -> int:
        return self.n_coef + 8

    @property
    def mfit(self) -> int:
        return int(np.count_nonzero(self.ia[1:]))


def _tokens(line: str):
    return line.split()


def scan_grid(text: str) -> ScanGrid:
    """The trial-frequency grid of a period_search_in text without preparing
    the object: 1/P_start, 1/P_end and 0.5 coef / (24 (JD_max - JD_min))
    (period_search_BOINC.cpp:839-841)."""
    lines = text.splitlines()
    p_start, p_coef, p_end = (float(v) for v in _tokens(lines[0])[:3])
    rest = " ".join(lines[14:]).split()
    pos, jd_min, jd_max = 1, math.inf, -math.inf
    for _ in range(int(rest[0])):
        lp = int(rest[pos])
        pos += 2
        for j in range(lp):
            t = float(rest[pos + 8 * j])
            jd_min, jd_max = min(jd_min, t), max(jd_max, t)
        pos += 8 * lp
    return ScanGrid(1 / p_start, 1 / p_end, 0.5 / (jd_max - jd_min) / 24 * p_coef)


def parse_input(text: str, setup_fn=None) -> PreparedObject:
    """Parses a period_search_in text and prepares the object."""
    lines = text.splitlines()
    hdr = [_tokens(l) for l in lines[:14]]
    p_start, p_coef, p_end, ia_prd = float(hdr[0][0]), float(hdr[0][1]), float(hdr[0][2]), int(hdr[0][3])
    jd00 = float(hdr[1][0])
    phi0 = float(hdr[2][0])
    conw = float(hdr[3][0])
    l_max, m_max = int(hdr[4][0]), int(hdr[4][1])
    nrows = int(hdr[5][0])
    par = np.array([float(hdr[6 + i][0]) for i in range(3)])
    ia_par = [int(hdr[6 + i][1]) for i in range(3)]
    cl, ia_cl = float(hdr[9][0]), int(hdr[9][1])
    stop = float(hdr[10][0])
    n_iter_min = int(hdr[11][0])
    lincr = float(hdr[12][0])
    lstart = float(hdr[13][0])
    rest = " ".join(lines[14:]).split()
    pos = 0
    n_curves = int(rest[pos]); pos += 1
    clen, crel = [], []
    tim, br, ee, ee0, sig = [], [], [], [], []
    al0 = al0_abs = PI
    ial0 = ial0_abs = -1
    onlyrel = True
    np_ = 0
    for i in range(n_curves):
        lp, itemp = int(rest[pos]), int(rest[pos + 1]); pos += 2
        rel = 1 - itemp
        clen.append(lp)
        crel.append(rel)
        if rel == 0:
            onlyrel = False
        blk = np.array(rest[pos:pos + 8 * lp], dtype=np.float64).reshape(lp, 8); pos += 8 * lp
        t, b, e0, e = blk[:, 0], blk[:, 1], blk[:, 2:5], blk[:, 5:8]
        e0len = np.sqrt(e0[:, 0] * e0[:, 0] + e0[:, 1] * e0[:, 1] + e0[:, 2] * e0[:, 2])
        elen = np.sqrt(e[:, 0] * e[:, 0] + e[:, 1] * e[:, 1] + e[:, 2] * e[:, 2])
        cosa = (e[0, 0] * e0[0, 0] + e[0, 1] * e0[0, 1] + e[0, 2] * e0[0, 2]) / (elen[0] * e0len[0])
        a = math.acos(cosa)
        if a < al0:
            al0, ial0 = a, np_
        if a < al0_abs and rel == 0:
            al0_abs, ial0_abs = a, np_
        ave = 0.0
        for v in b:
            ave += v
        ave /= lp
        tim.append(t)
        br.append(b)
        ee.append(e / elen[:, None])
        ee0.append(e0 / e0len[:, None])
        sig.append(np.full(lp, ave))
        np_ += lp
    wlc = [-1.0] * n_curves
    while pos + 1 < len(rest):
        lc, wv = int(rest[pos]), float(rest[pos + 1]); pos += 2
        if 1 <= lc <= n_curves:
            wlc[lc - 1] = wv
    tim = np.concatenate(tim)
    jd_min, jd_max = float(tim.min()), float(tim.max())
    jd0 = jd00 if jd00 > 0 else float(int(jd_min))
    tim = tim - jd0
    sig = np.concatenate(sig)
    if not onlyrel:
        al0, ial0 = al0_abs, ial0_abs
    ea, eb, ec = 1.05, 1.00, 0.95
    rfit = math.sqrt(2 * sig[ial0] / (0.5 * PI * (1 + math.cos(al0))))
    escl = rfit / math.sqrt((ea * eb + eb * ec + ea * ec) / 3)
    if not onlyrel:
        escl *= 0.8
    ea, eb, ec = ea * escl, eb * escl, ec * escl
    nc = n_coef(l_max, m_max)
    if setup_fn is None:
        from . import native
        setup_fn = native.setup_shape
    normal, d_area, dsph, cg_first = setup_fn(l_max, m_max, nrows, ea, eb, ec)
    ma = nc + 8
    ia = np.zeros(ma + 1, dtype=np.int32)
    ia[1:nc + 1] = 1
    if onlyrel:
        ia[1] = 0
    ia[nc + 1] = 1
    ia[nc + 2] = 1
    ia[nc + 3] = ia_prd
    ia[nc + 4:nc + 7] = ia_par
    ia[ma - 1] = ia_cl
    ia[ma] = 0
    if stop > 1:
        n_iter_max, iter_diff_max, nimin = int(stop), 0.0, 0
    elif stop < 1:
        n_iter_max, iter_diff_max, nimin = MAX_N_ITER, stop, n_iter_min
    else:
        n_iter_max, iter_diff_max, nimin = 0, -1.0, n_iter_min
    weight = np.concatenate([np.full(l, 1.0 if w == -1 else w) for l, w in zip(clen, wlc)])
    grid = ScanGrid(1 / p_start, 1 / p_end, 0.5 / (jd_max - jd_min) / 24 * p_coef)
    return PreparedObject(
        n_points=np_, n_curves=n_curves, curve_len=np.array(clen, dtype=np.int32),
        curve_rel=np.array(crel, dtype=np.int32), tim=tim, ee=np.concatenate(ee).ravel(),
        ee0=np.concatenate(ee0).ravel(), brightness=np.concatenate(br), sig=sig,
        sigr2=1.0 / (sig * sig), weight=weight, l_max=l_max, m_max=m_max, nrows=nrows,
        n_fac=8 * nrows * nrows, n_coef=nc, normal=np.ascontiguousarray(normal).ravel(),
        d_area=np.ascontiguousarray(d_area), dsph=np.ascontiguousarray(dsph).ravel(),
        cg_first=np.ascontiguousarray(cg_first), phi0=phi0 * DEG2RAD, par=par, lcl=math.log(cl), cl=cl,
        alamda_start=lstart, alamda_incr=lincr,
        alamda_incrr=(1.0 / lincr) if lincr != 0.0 else np.finfo(np.float64).max,
        beta_pole=np.array(BETA_POLES, dtype=np.float64),
        lambda_pole=np.array(LAMBDA_POLES, dtype=np.float64), ia=ia, n_iter_max=n_iter_max,
        n_iter_min=nimin, iter_diff_max=iter_diff_max, stop_condition=stop, conw_r=conw / escl / escl, escl=escl,
        grid=grid, onlyrel=onlyrel)


def load(path: str, setup_fn=None) -> PreparedObject:
    with open(path) as f:
        return parse_input(f.read(), setup_fn)


def initial_params(obj: PreparedObject, n_freq: int, pole: int) -> np.ndarray:
    """1-based parameter vector of one (frequency, pole) item
    (CudaCalculatePreparePole, Start.cu:4346-4418)."""
    nc, ma = obj.n_coef, obj.ma
    a = np.zeros(ma + 1)
    a[1:nc + 1] = obj.cg_first
    period = 1.0 / (obj.grid.freq_start - (n_freq - 1) * obj.grid.freq_step)
    a[nc + 1] = DEG2RAD * 90 - DEG2RAD * obj.beta_pole[pole]
    a[nc + 2] = DEG2RAD * obj.lambda_pole[pole]
    a[nc + 3] = (24.0 * 2.0 * PI) / period
    a[nc + 4:nc + 7] = obj.par
    a[ma - 1] = obj.lcl
    a[ma] = 1
    return a
