"""ctypes binding of the native library ``_lib/libps_b200.so`` (include/ps_b200.h).

There is no Python or CPU fallback: if the library is missing or a CUDA call
fails, the call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libps_b200.so")
# the C++ host program (period_search_in -> period_search_out) built beside the library
HOST_PROGRAM = os.path.join(HERE, "_lib", "period_search")

N_POLES = 10
QUIRK_PRECALC_CONW = 1
PRECISION_FP64 = 0
PRECISION_MIXED = 1
DEVSTAT_SINGULAR = 1
DEVSTAT_NAN_CHISQ = 2
DEVSTAT_TIMEOUT = 4

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class Curves(C.Structure):
    _fields_ = [("n_curves", C.c_int32), ("curve_len", _ip), ("curve_rel", _ip)]


class Shape(C.Structure):
    _fields_ = [("n_coef", C.c_int32), ("normal", _dp), ("d_area", _dp), ("d_sphere", _dp)]


class Line(C.Structure):
    _fields_ = [("period_h", C.c_double), ("rms", C.c_double), ("chisq", C.c_double),
                ("dark", C.c_double), ("lambda_deg", C.c_double), ("beta_deg", C.c_double)]


class FitResult(C.Structure):
    _fields_ = [("dev", C.c_double), ("dark", C.c_double), ("per", C.c_double),
                ("lambda_deg", C.c_double), ("beta_deg", C.c_double), ("chisq", C.c_double),
                ("niter", C.c_int32), ("status", C.c_int32)]


class Object(C.Structure):
    """ps_object: one object of ps_gpu_scan_batch."""
    _fields_ = [("beta_pole", _dp), ("lambda_pole", _dp), ("par", _dp),
                ("cl", C.c_double), ("alamda_start", C.c_double), ("alamda_incr", C.c_double),
                ("alamda_incrr", C.c_double), ("phi0", C.c_double), ("ndata", C.c_int32),
                ("tim", _dp), ("ee", _dp), ("ee0", _dp), ("weight", _dp), ("brightness", _dp), ("sig", _dp),
                ("sigr2", _dp), ("ia", _ip), ("ia_par", _ip), ("cg_first", _dp), ("numfac", C.c_int32),
                ("curves", Curves), ("shape", Shape), ("freq_start", C.c_double), ("freq_end", C.c_double),
                ("freq_step", C.c_double), ("stop_condition", C.c_double), ("n_iter_min", C.c_int32),
                ("escl", C.c_double), ("conw_r", C.c_double), ("n_start_from", C.c_int32),
                ("max_lines", C.c_int32)]


PROGRESS_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int32, C.c_int32)

# name -> (restype, argtypes)
_SIGS = {
    "ps_gpu_prepare": (C.c_int, [C.c_int32, _dp, _dp, _dp, C.c_double, C.c_double, C.c_double, C.c_double,
                                 _dp, _dp, _dp, C.c_double, C.c_int32, _dp, C.POINTER(C.c_void_p)]),
    "ps_gpu_precalc": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int32, _dp,
                                 C.c_int32, _ip, _ip, _ip, _dp, _dp, _dp, C.c_int32, _dp,
                                 C.POINTER(Curves), C.POINTER(Shape)]),
    "ps_gpu_start": (C.c_int, [C.c_void_p, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int32,
                               C.c_double, C.c_int32, _ip, _ip, _dp, C.c_double, _dp, _dp, C.c_int32, _dp,
                               C.POINTER(Curves), C.POINTER(Shape), C.POINTER(Line), C.c_int32, _ip,
                               PROGRESS_FN, C.c_void_p]),
    "ps_gpu_unprepare": (None, [C.c_void_p]),
    "ps_gpu_configure": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int32, C.c_double,
                                   C.c_double, C.c_int32, _ip, _ip, _dp, _dp, _dp, C.c_int32, _dp,
                                   C.POINTER(Curves), C.POINTER(Shape)]),
    "ps_gpu_fit_items": (C.c_int, [C.c_void_p, C.c_int32, _ip, _ip, C.POINTER(FitResult)]),
    "ps_gpu_fit_items_device": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "ps_gpu_eval": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp, _dp]),
    "ps_gpu_status": (C.c_int, [C.c_void_p, _ip]),
    "ps_gpu_set_quirks": (C.c_int, [C.c_void_p, C.c_int32]),
    "ps_gpu_phase_clocks": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int64)]),
    "ps_gpu_stream": (C.c_void_p, [C.c_void_p]),
    "ps_gpu_occupancy": (C.c_int, [C.c_void_p, _ip, _ip]),
    "ps_setup_shape": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                 _dp, _dp, _dp, _dp]),
    "ps_fit_items_noalloc": (C.c_int, [C.c_int32, C.c_void_p, _dp, _dp, _dp, C.c_double, C.c_double, C.c_double,
                                       C.c_double, _dp, _dp, _dp, C.c_double, _dp, C.c_double, C.c_double,
                                       C.c_double, C.c_int32, C.c_double, C.c_double, C.c_int32, _ip, _ip, _dp,
                                       _dp, _dp, C.c_int32, _dp, C.POINTER(Curves), C.POINTER(Shape), C.c_int32,
                                       _ip, _ip, C.POINTER(FitResult)]),
    "ps_gpu_scan_batch": (C.c_int, [C.c_int32, C.c_int32, C.POINTER(Object), C.c_int32, C.POINTER(Line),
                                    C.POINTER(C.c_int64), _ip, _dp]),
    "ps_gpu_set_precision": (C.c_int, [C.c_void_p, C.c_int32]),
    "ps_batch_set_tuning": (C.c_int, [C.c_int32]),
    "ps_batch_tuning_report": (C.c_int32, [C.c_char_p, C.c_int32]),
    "ps_screen_features": (C.c_int, [C.c_int32, C.c_int32, _dp, _dp, C.POINTER(Curves), C.c_int32, _dp,
                                     C.POINTER(C.c_float)]),
    "ps_screen_rank": (C.c_int, [C.c_int32, C.c_int32, _dp, _dp, C.POINTER(Curves), C.c_int32, _dp, C.c_int32,
                                 _ip, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "ps_gemm_bf16": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p,
                               C.c_int64, C.c_int64, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_int32,
                               C.c_void_p, C.c_int32, C.c_void_p]),
    "ps_relu_backward": (C.c_int, [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ps_column_sum": (C.c_int, [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ps_adam_step": (C.c_int, [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_float,
                               C.c_float, C.c_float, C.c_int32, C.c_void_p, C.c_void_p]),
    "ps_to_bf16": (C.c_int, [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ps_n_coef": (C.c_int32, [C.c_int32, C.c_int32]),
    "ps_measure_fp64_peak": (C.c_int, [C.c_int32, _dp]),
    "ps_probe_reciprocal": (C.c_int, [C.c_int32, _dp, _dp]),
    "ps_probe_wait_timeout": (C.c_int, [C.c_int32, _ip]),
    "ps_probe_solve": (C.c_int, [C.c_int32, _dp, _dp, _dp, _ip]),
    "ps_last_error": (C.c_char_p, []),
    "ps_version": (C.c_char_p, []),
}

_lib = None


def lib() -> C.CDLL:
    """The loaded native library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"native library missing: {LIB_PATH} (run __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS)


class PsError(RuntimeError):
    pass


def _check(rc):
    if rc != 0:
        raise PsError(f"ps_b200 error {rc}: {lib().ps_last_error().decode()}")


def _p(a, ct=C.c_double):
    return a.ctypes.data_as(C.POINTER(ct))


def setup_shape(l_max, m_max, nrows, a, b, c):
    """Gaussian-image tables (normals, areas, Laplace basis, ellipsoid fit)."""
    nfac = 8 * nrows * nrows
    nc = int(lib().ps_n_coef(l_max, m_max))
    normal = np.zeros((nfac, 3))
    d_area = np.zeros(nfac)
    dsph = np.zeros((nfac, nc))
    cg = np.zeros(nc)
    _check(lib().ps_setup_shape(l_max, m_max, nrows, a, b, c, _p(normal), _p(d_area), _p(dsph), _p(cg)))
    return normal, d_area, dsph, cg


def measure_fp64_peak(device=0):
    t = np.zeros(1)
    _check(lib().ps_measure_fp64_peak(device, _p(t)))
    return float(t[0])


def probe_reciprocal(d):
    d = np.ascontiguousarray(d, dtype=np.float64)
    r = np.zeros_like(d)
    _check(lib().ps_probe_reciprocal(len(d), _p(d), _p(r)))
    return r


def probe_solve(a, b):
    """The fit kernel's Gauss-Jordan solve of a x = b on the GPU: (err, x)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    n = b.shape[0]
    if a.shape != (n, n):
        raise ValueError("probe_solve: a must be n x n")
    x = np.zeros(n)
    err = np.zeros(1, dtype=np.int32)
    _check(lib().ps_probe_solve(n, _p(a), _p(b), _p(x), _p(err, C.c_int32)))
    return int(err[0]), x


class Engine:
    """One prepared object on one GPU (the reference's CUDAPrepare state)."""

    def __init__(self, obj, device: int = 0):
        self.obj = obj
        self._keep = []
        L = lib()
        h = C.c_void_p()
        self._ee = self._arr(obj.ee)
        self._ee0 = self._arr(obj.ee0)
        self._tim = self._arr(obj.tim)
        _check(L.ps_gpu_prepare(device, _p(self._arr(obj.beta_pole)), _p(self._arr(obj.lambda_pole)),
                                _p(self._arr(obj.par)), float(obj.cl), obj.alamda_start,
                                obj.alamda_incr, obj.alamda_incrr, _p(self._ee), _p(self._ee0), _p(self._tim),
                                obj.phi0, obj.n_points, _p(self._arr(obj.weight)), C.byref(h)))
        self.h = h
        self._ia = self._arr(obj.ia, np.int32)
        self._ia_par = self._arr(obj.ia[obj.n_coef + 4:obj.n_coef + 7], np.int32)
        self._cg = self._arr(obj.cg_first)
        self._sig = self._arr(obj.sig)
        self._sigr2 = self._arr(obj.sigr2)
        self._br = self._arr(obj.brightness)
        self.curves = Curves(obj.n_curves, _p(self._arr(obj.curve_len, np.int32), C.c_int32),
                             _p(self._arr(obj.curve_rel, np.int32), C.c_int32))
        self.shape = Shape(obj.n_coef, _p(self._arr(obj.normal)), _p(self._arr(obj.d_area)),
                           _p(self._arr(obj.dsph)))

    def _arr(self, x, dt=np.float64):
        a = np.ascontiguousarray(x, dtype=dt)
        self._keep.append(a)
        return a

    def close(self):
        if self.h:
            lib().ps_gpu_unprepare(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_quirks(self, q):
        _check(lib().ps_gpu_set_quirks(self.h, q))

    def set_precision(self, precision):
        """PRECISION_FP64 or PRECISION_MIXED; applies from the next configure."""
        _check(lib().ps_gpu_set_precision(self.h, precision))

    def configure(self, conw_r=None, conw_r_rms=None, stop_condition=None, grid=None):
        o = self.obj
        g = grid or o.grid
        cw = o.conw_r if conw_r is None else conw_r
        stop = stop_condition if stop_condition is not None else self._stop()
        _check(lib().ps_gpu_configure(self.h, g.freq_start, g.freq_step, stop, o.n_iter_min, cw,
                                      cw if conw_r_rms is None else conw_r_rms, o.n_points,
                                      _p(self._ia, C.c_int32), _p(self._ia_par, C.c_int32), _p(self._cg),
                                      _p(self._sig), _p(self._sigr2), o.n_fac, _p(self._br),
                                      C.byref(self.curves), C.byref(self.shape)))

    def _stop(self):
        return float(self.obj.stop_condition)

    def fit_items(self, n_freq, pole):
        n_freq = np.ascontiguousarray(n_freq, dtype=np.int32)
        pole = np.ascontiguousarray(pole, dtype=np.int32)
        n = len(n_freq)
        res = (FitResult * max(n, 1))()
        _check(lib().ps_gpu_fit_items(self.h, n, _p(n_freq, C.c_int32), _p(pole, C.c_int32), res))
        out = np.array([(r.dev, r.dark, r.per, r.lambda_deg, r.beta_deg, r.chisq) for r in res[:n]])
        niter = np.array([r.niter for r in res[:n]], dtype=np.int32)
        status = np.array([r.status for r in res[:n]], dtype=np.int32)
        return out.reshape(n, 6), niter, status

    def fit_items_device(self, n, d_items_ptr, d_out_ptr):
        _check(lib().ps_gpu_fit_items_device(self.h, n, C.c_void_p(d_items_ptr), C.c_void_p(d_out_ptr)))

    def eval(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        mf = self.obj.mfit
        alpha = np.zeros((mf, mf))
        beta = np.zeros(mf)
        chisq = np.zeros(1)
        area = np.zeros(1)
        _check(lib().ps_gpu_eval(self.h, _p(a), _p(chisq), _p(alpha), _p(beta), _p(area)))
        return float(chisq[0]), alpha, beta, float(area[0])

    def precalc(self, conw_r, grid=None):
        o = self.obj
        g = grid or o.grid
        cw = np.array([conw_r], dtype=np.float64)
        nc = np.zeros(1, dtype=np.int32)
        _check(lib().ps_gpu_precalc(self.h, g.freq_start, g.freq_end, g.freq_step, self._stop(), o.n_iter_min,
                                    _p(cw), o.n_points, _p(self._ia, C.c_int32), _p(self._ia_par, C.c_int32),
                                    _p(nc, C.c_int32), _p(self._cg), _p(self._sig), _p(self._sigr2), o.n_fac,
                                    _p(self._br), C.byref(self.curves), C.byref(self.shape)))
        return float(cw[0]), int(nc[0])

    def start(self, conw_r, n_start_from=1, max_lines=None, grid=None, progress=None):
        o = self.obj
        g = grid or o.grid
        cap = g.n_max - n_start_from + 1 if max_lines is None else max_lines
        lines = (Line * max(cap, 1))()
        nl = np.zeros(1, dtype=np.int32)
        cb = PROGRESS_FN(progress) if progress else PROGRESS_FN()
        _check(lib().ps_gpu_start(self.h, n_start_from, g.freq_start, g.freq_end, g.freq_step, self._stop(),
                                  o.n_iter_min, conw_r, o.n_points, _p(self._ia, C.c_int32),
                                  _p(self._ia_par, C.c_int32), _p(self._cg), o.escl, _p(self._sig),
                                  _p(self._sigr2), o.n_fac, _p(self._br), C.byref(self.curves),
                                  C.byref(self.shape), lines, cap, _p(nl, C.c_int32), cb, None))
        n = int(nl[0])
        return np.array([(l.period_h, l.rms, l.chisq, l.dark, l.lambda_deg, l.beta_deg) for l in lines[:n]])

    def status(self):
        f = np.zeros(1, dtype=np.int32)
        _check(lib().ps_gpu_status(self.h, _p(f, C.c_int32)))
        return int(f[0])

    PHASES = ("curv", "sort", "sweep", "curve_stats", "jtwj_other", "pseudo", "solve", "rest", "tile_wait",
              "tile_stage", "tile_syrk")

    def phase_clocks(self, enable=True):
        """Cycles per phase since the last call (dict), then restarts counting."""
        out = np.zeros(12, dtype=np.int64)
        _check(lib().ps_gpu_phase_clocks(self.h, 1 if enable else 0, out.ctypes.data_as(C.POINTER(C.c_int64))))
        d = dict(zip(self.PHASES, out[:11].tolist()))
        d["evals"] = int(out[11])
        return d

    def occupancy(self):
        a = np.zeros(1, dtype=np.int32)
        b = np.zeros(1, dtype=np.int32)
        _check(lib().ps_gpu_occupancy(self.h, _p(a, C.c_int32), _p(b, C.c_int32)))
        return int(a[0]), int(b[0])

    @property
    def stream(self):
        return lib().ps_gpu_stream(self.h)


def fit_items_noalloc(obj, n_freq, pole, device=0, conw_r=None):
    """ps_fit_items_noalloc on a prepared object: the allocation-free variant of
    Engine.fit_items (host inputs, host results, one static device arena)."""
    keep = []

    def arr(x, dt=np.float64):
        a = np.ascontiguousarray(x, dtype=dt)
        keep.append(a)
        return a

    n_freq = arr(n_freq, np.int32)
    pole = arr(pole, np.int32)
    n = len(n_freq)
    res = (FitResult * max(n, 1))()
    cw = obj.conw_r if conw_r is None else conw_r
    curves = Curves(obj.n_curves, _p(arr(obj.curve_len, np.int32), C.c_int32),
                    _p(arr(obj.curve_rel, np.int32), C.c_int32))
    shape = Shape(obj.n_coef, _p(arr(obj.normal)), _p(arr(obj.d_area)), _p(arr(obj.dsph)))
    ia = arr(obj.ia, np.int32)
    ia_par = arr(obj.ia[obj.n_coef + 4:obj.n_coef + 7], np.int32)
    g = obj.grid
    _check(lib().ps_fit_items_noalloc(
        device, None, _p(arr(obj.beta_pole)), _p(arr(obj.lambda_pole)), _p(arr(obj.par)), float(obj.cl),
        obj.alamda_start, obj.alamda_incr, obj.alamda_incrr, _p(arr(obj.ee)), _p(arr(obj.ee0)), _p(arr(obj.tim)),
        obj.phi0, _p(arr(obj.weight)), g.freq_start, g.freq_step, float(obj.stop_condition), obj.n_iter_min, cw, cw,
        obj.n_points, _p(ia, C.c_int32), _p(ia_par, C.c_int32), _p(arr(obj.cg_first)), _p(arr(obj.sig)),
        _p(arr(obj.sigr2)), obj.n_fac, _p(arr(obj.brightness)), C.byref(curves), C.byref(shape), n,
        _p(n_freq, C.c_int32), _p(pole, C.c_int32), res))
    out = np.array([(r.dev, r.dark, r.per, r.lambda_deg, r.beta_deg, r.chisq) for r in res[:n]])
    niter = np.array([r.niter for r in res[:n]], dtype=np.int32)
    status = np.array([r.status for r in res[:n]], dtype=np.int32)
    return out.reshape(n, 6), niter, status


def reserve_noalloc(device=0):
    """ps_fit_items_noalloc with no work (n = 0, every array NULL): selects
    the device and loads the library's module there, which reserves the
    entry point's static device arena.  Call it at start-up, before another
    allocator fills the device."""
    _check(lib().ps_fit_items_noalloc(device, None, None, None, None, 0.0, 0.0, 0.0, 0.0, None, None, None, 0.0,
                                      None, 0.0, 0.0, 0.0, 0, 0.0, 0.0, 0, None, None, None, None, None, 0, None,
                                      None, None, 0, None, None, None))


def scan_batch(objs, device=0, quirks=0, max_freq=None):
    """ps_gpu_scan_batch over prepared objects: each object's convexity-weight
    search and scan, all on one GPU at once.  Returns [(lines, conw_r)] in the
    order of objs, as run_object gives them one by one."""
    keep = []

    def arr(x, dt=np.float64):
        a = np.ascontiguousarray(x, dtype=dt)
        keep.append(a)
        return a

    n = len(objs)
    cs = (Object * max(n, 1))()
    offs = np.zeros(max(n, 1), dtype=np.int64)
    total = 0
    for i, o in enumerate(objs):
        g = o.grid
        nl = g.n_max if max_freq is None else min(g.n_max, max_freq)
        offs[i] = total
        total += nl
        c = cs[i]
        c.beta_pole, c.lambda_pole, c.par = _p(arr(o.beta_pole)), _p(arr(o.lambda_pole)), _p(arr(o.par))
        c.cl, c.alamda_start, c.alamda_incr, c.alamda_incrr = float(o.cl), o.alamda_start, o.alamda_incr, o.alamda_incrr
        c.phi0, c.ndata = o.phi0, o.n_points
        c.tim, c.ee, c.ee0, c.weight = _p(arr(o.tim)), _p(arr(o.ee)), _p(arr(o.ee0)), _p(arr(o.weight))
        c.brightness, c.sig, c.sigr2 = _p(arr(o.brightness)), _p(arr(o.sig)), _p(arr(o.sigr2))
        c.ia = _p(arr(o.ia, np.int32), C.c_int32)
        c.ia_par = _p(arr(o.ia[o.n_coef + 4:o.n_coef + 7], np.int32), C.c_int32)
        c.cg_first, c.numfac = _p(arr(o.cg_first)), o.n_fac
        c.curves = Curves(o.n_curves, _p(arr(o.curve_len, np.int32), C.c_int32),
                          _p(arr(o.curve_rel, np.int32), C.c_int32))
        c.shape = Shape(o.n_coef, _p(arr(o.normal)), _p(arr(o.d_area)), _p(arr(o.dsph)))
        c.freq_start, c.freq_end, c.freq_step = g.freq_start, g.freq_end, g.freq_step
        c.stop_condition, c.n_iter_min = float(o.stop_condition), o.n_iter_min
        c.escl, c.conw_r, c.n_start_from, c.max_lines = o.escl, o.conw_r, 1, nl
    lines = (Line * max(total, 1))()
    nl = np.zeros(max(n, 1), dtype=np.int32)
    cw = np.zeros(max(n, 1))
    _check(lib().ps_gpu_scan_batch(device, n, cs, quirks, lines, offs.ctypes.data_as(C.POINTER(C.c_int64)),
                                   _p(nl, C.c_int32), _p(cw)))
    out = []
    for i in range(n):
        ls = lines[int(offs[i]):int(offs[i]) + int(nl[i])]
        out.append((np.array([(l.period_h, l.rms, l.chisq, l.dark, l.lambda_deg, l.beta_deg) for l in ls]),
                    float(cw[i])))
    return out


def batch_set_tuning(mode):
    """ps_batch_set_tuning: 1 = autotuned tile layouts (default; choices
    cached per group shape), 2 = the same after clearing the cache, 0 = the
    first layout that fits."""
    _check(lib().ps_batch_set_tuning(int(mode)))


def batch_tuning_report():
    """The last scan_batch's per-group layout choices (parsed JSON)."""
    import json

    n = lib().ps_batch_tuning_report(None, 0)
    buf = C.create_string_buffer(n + 1)
    lib().ps_batch_tuning_report(buf, n + 1)
    return json.loads(buf.value.decode())


def run_object(obj, device=0, quirks=0, max_freq=None, progress=None, precision=PRECISION_FP64):
    """The reference's main flow after parsing: conw precalc loop, then the scan.
    Returns (lines, final conw_r)."""
    with Engine(obj, device) as eng:
        eng.set_quirks(quirks)
        eng.set_precision(precision)
        conw_r = obj.conw_r
        new_conw = 0
        while new_conw != 1 and conw_r * obj.escl * obj.escl < 10.0:
            conw_r, new_conw = eng.precalc(conw_r)
        lines = eng.start(conw_r, max_lines=max_freq, progress=progress)
    return lines, conw_r


def format_lines(lines):
    """period_search_out text (start_CUDA.cu:1220-1227)."""
    out = []
    for l in lines:
        out.append("%.8f  %.6f  %.6f %4.1f %4.0f %4.0f\n" % (l[0], l[1], l[2], l[3], _round(l[4]), _round(l[5])))
    return "".join(out)


def _round(x):
    # C round(): half away from zero
    return float(np.sign(x) * np.floor(abs(x) + 0.5))
