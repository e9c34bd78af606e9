"""ctypes binding of the CPU FP64 oracle (test infrastructure only).

The oracle is a plain-C restatement of PeriodSearch's LM-fit hot path
(oracle/ps_oracle.c).  Only the test suite, ``__graft_entry__.smoke`` and the
CPU-baseline leg of ``bench.py`` import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF = os.path.join(HERE, "_ref")

MAX_PAR = 128
N_POLES = 10
QUIRK_PRECALC_CONW = 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class Model(C.Structure):
    _fields_ = [
        ("n_points", C.c_int), ("n_curves", C.c_int),
        ("curve_len", _ip), ("curve_rel", _ip),
        ("tim", _dp), ("ee", _dp), ("ee0", _dp), ("bright", _dp),
        ("sig", _dp), ("sigr2", _dp), ("weight", _dp),
        ("n_fac", C.c_int), ("n_coef", C.c_int),
        ("normal", _dp), ("d_area", _dp), ("dsph", _dp), ("cg_first", _dp),
        ("phi0", C.c_double), ("par", C.c_double * 3), ("lcl", C.c_double),
        ("alamda_start", C.c_double), ("alamda_incr", C.c_double), ("alamda_incrr", C.c_double),
        ("beta_pole", C.c_double * N_POLES), ("lambda_pole", C.c_double * N_POLES),
        ("ia", C.c_int * (MAX_PAR + 1)),
        ("n_iter_max", C.c_int), ("n_iter_min", C.c_int),
        ("iter_diff_max", C.c_double), ("conw_r", C.c_double), ("conw_r_dev", C.c_double),
    ]


class FitResult(C.Structure):
    _fields_ = [("dev", C.c_double), ("dark", C.c_double), ("per", C.c_double),
                ("lambda_deg", C.c_double), ("beta_deg", C.c_double), ("chisq", C.c_double),
                ("niter", C.c_int), ("status", C.c_int)]


class Line(C.Structure):
    _fields_ = [("period_h", C.c_double), ("rms", C.c_double), ("chisq", C.c_double),
                ("dark", C.c_double), ("lambda_deg", C.c_double), ("beta_deg", C.c_double),
                ("valid", C.c_int)]


def build(quiet: bool = True) -> None:
    """Compile the oracle (and, where the reference tree exists, oracle/_ref)."""
    out = subprocess.run(["make", "-C", HERE, "-j4"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


_LIBS: dict = {}


def lib(fast: bool = False, fma: bool = False, perturb: bool = False) -> C.CDLL:
    """The strict oracle; fast=True the -O3 -march=native build (timed CPU
    baseline); fma=True the build with FMA contraction (the same algorithm
    under a different rounding); perturb=True the strict build with the
    seeded brightness noise of oracle/perturbation_study.py."""
    name = ("libps_oracle_perturb.so" if perturb else "libps_oracle_fma.so" if fma else
            "libps_oracle_fast.so" if fast else "libps_oracle.so")
    if name not in _LIBS:
        path = os.path.join(BUILD, name)
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.pso_n_coef.restype = C.c_int
        L.pso_setup_shape.restype = C.c_int
        L.pso_setup_shape.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                      _dp, _dp, _dp, _dp]
        L.pso_eval.restype = C.c_double
        L.pso_eval.argtypes = [C.POINTER(Model), _dp, _dp, _dp, _dp, _dp]
        L.pso_fit_batch.argtypes = [C.POINTER(Model), C.c_double, C.c_double, _ip, _ip, C.c_int,
                                    C.POINTER(FitResult), C.c_int]
        L.pso_precalc.argtypes = [C.POINTER(Model), C.c_double, C.c_double, _dp, _ip, C.c_int, C.c_int]
        L.pso_scan.restype = C.c_int
        L.pso_scan.argtypes = [C.POINTER(Model), C.c_double, C.c_double, C.c_double, C.c_int,
                               C.POINTER(Line), C.c_int, C.c_int]
        L.pso_run_file.restype = C.c_int
        L.pso_run_file.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_int]
        L.pso_gauss_solve.restype = C.c_int
        L.pso_gauss_solve.argtypes = [_dp, C.c_int, _dp]
        _LIBS[name] = L
    return _LIBS[name]


def _p(a, ct=C.c_double):
    return a.ctypes.data_as(C.POINTER(ct))


def setup_shape(l_max, m_max, nrows, a, b, c, reference=False):
    """Shape tables from the oracle restatement (or, reference=True, from the
    reference's own setup sources in oracle/_ref)."""
    nfac = 8 * nrows * nrows
    nc = int(lib().pso_n_coef(l_max, m_max))
    normal = np.zeros((nfac, 3))
    darea = np.zeros(nfac)
    dsph = np.zeros((nfac, nc))
    cg = np.zeros(nc)
    if reference:
        L = C.CDLL(os.path.join(REF, "libref_setup.so"))
        L.ref_setup_shape.restype = C.c_int
        L.ref_setup_shape.argtypes = lib().pso_setup_shape.argtypes
        rc = L.ref_setup_shape(l_max, m_max, nrows, a, b, c, _p(normal), _p(darea), _p(dsph), _p(cg))
    else:
        rc = lib().pso_setup_shape(l_max, m_max, nrows, a, b, c, _p(normal), _p(darea), _p(dsph), _p(cg))
    if rc != 0:
        raise RuntimeError(f"setup failed ({rc})")
    return normal, darea, dsph, cg


class OracleModel:
    """Holds numpy arrays alive behind a ctypes Model built from a prepared object
    (ps_claude_opt_b200.objects.PreparedObject or any object with the same fields)."""

    def __init__(self, obj, conw_r=None, conw_r_dev=None):
        self._keep = []

        def arr(x, dt=np.float64):
            x = np.ascontiguousarray(x, dtype=dt)
            self._keep.append(x)
            return x

        m = Model()
        m.n_points = int(obj.n_points)
        m.n_curves = int(obj.n_curves)
        m.curve_len = _p(arr(obj.curve_len, np.int32), C.c_int)
        m.curve_rel = _p(arr(obj.curve_rel, np.int32), C.c_int)
        m.tim = _p(arr(obj.tim))
        m.ee = _p(arr(obj.ee))
        m.ee0 = _p(arr(obj.ee0))
        m.bright = _p(arr(obj.brightness))
        m.sig = _p(arr(obj.sig))
        m.sigr2 = _p(arr(obj.sigr2))
        m.weight = _p(arr(obj.weight))
        m.n_fac = int(obj.n_fac)
        m.n_coef = int(obj.n_coef)
        m.normal = _p(arr(obj.normal))
        m.d_area = _p(arr(obj.d_area))
        m.dsph = _p(arr(obj.dsph))
        m.cg_first = _p(arr(obj.cg_first))
        m.phi0 = float(obj.phi0)
        for i in range(3):
            m.par[i] = float(obj.par[i])
        m.lcl = float(obj.lcl)
        m.alamda_start = float(obj.alamda_start)
        m.alamda_incr = float(obj.alamda_incr)
        m.alamda_incrr = float(obj.alamda_incrr)
        for i in range(N_POLES):
            m.beta_pole[i] = float(obj.beta_pole[i])
            m.lambda_pole[i] = float(obj.lambda_pole[i])
        for i, v in enumerate(obj.ia):
            m.ia[i] = int(v)
        m.n_iter_max = int(obj.n_iter_max)
        m.n_iter_min = int(obj.n_iter_min)
        m.iter_diff_max = float(obj.iter_diff_max)
        cw = float(obj.conw_r if conw_r is None else conw_r)
        m.conw_r = cw
        m.conw_r_dev = cw if conw_r_dev is None else float(conw_r_dev)
        self.m = m
        self.obj = obj

    @property
    def ma(self):
        return self.m.n_coef + 8

    def mfit(self):
        return sum(1 for p in range(1, self.ma + 1) if self.m.ia[p])

    def eval(self, a, with_rows=False):
        """One mrqcof evaluation at the 1-based parameter vector a[0..ma]."""
        a = np.ascontiguousarray(a, dtype=np.float64)
        mf = self.mfit()
        alpha = np.zeros((mf, mf))
        beta = np.zeros(mf)
        area = np.zeros(1)
        rows = np.zeros((self.m.n_points + 3, self.ma + 1)) if with_rows else None
        chisq = lib().pso_eval(C.byref(self.m), _p(a), _p(alpha), _p(beta),
                               _p(rows) if with_rows else None, _p(area))
        return chisq, alpha, beta, rows, float(area[0])

    def fit_batch(self, freq_start, freq_step, n_freq, pole, threads=0, fast=False):
        n_freq = np.ascontiguousarray(n_freq, dtype=np.int32)
        pole = np.ascontiguousarray(pole, dtype=np.int32)
        n = len(n_freq)
        res = (FitResult * n)()
        threads = threads or os.cpu_count() or 1
        lib(fast).pso_fit_batch(C.byref(self.m), freq_start, freq_step, _p(n_freq, C.c_int),
                                _p(pole, C.c_int), n, res, threads)
        out = np.zeros((n, 6))
        niter = np.zeros(n, dtype=np.int32)
        status = np.zeros(n, dtype=np.int32)
        for i in range(n):
            r = res[i]
            out[i] = (r.dev, r.dark, r.per, r.lambda_deg, r.beta_deg, r.chisq)
            niter[i] = r.niter
            status[i] = r.status
        return out, niter, status

    def precalc(self, freq_start, freq_step, conw_r, quirks=0, threads=0):
        cw = np.array([conw_r], dtype=np.float64)
        nc = np.zeros(1, dtype=np.int32)
        lib().pso_precalc(C.byref(self.m), freq_start, freq_step, _p(cw), _p(nc, C.c_int), quirks,
                          threads or os.cpu_count() or 1)
        return float(cw[0]), int(nc[0])

    def scan(self, freq_start, freq_end, freq_step, n_start=1, max_lines=None, threads=0, fast=False,
             perturb=False):
        n_max = int((freq_start - freq_end) / freq_step) + 1
        cap = n_max - n_start + 1 if max_lines is None else max_lines
        lines = (Line * max(cap, 1))()
        n = lib(fast, perturb=perturb).pso_scan(C.byref(self.m), freq_start, freq_end, freq_step, n_start, lines, cap,
                               threads or os.cpu_count() or 1)
        return np.array([(l.period_h, l.rms, l.chisq, l.dark, l.lambda_deg, l.beta_deg)
                         for l in lines[:n]])


def gauss_solve(a, b):
    a = np.array(a, dtype=np.float64, order="C")
    b = np.array(b, dtype=np.float64)
    rc = lib().pso_gauss_solve(_p(a), a.shape[0], _p(b))
    return rc, b


def run_file(in_path, out_path, quirks=0, threads=0, max_freq=0, fma=False):
    rc = lib(fma=fma).pso_run_file(in_path.encode(), out_path.encode(), quirks, threads or os.cpu_count() or 1,
                            max_freq)
    if rc != 0:
        raise RuntimeError(f"oracle run failed ({rc})")
