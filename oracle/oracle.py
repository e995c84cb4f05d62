"""ctypes front-end of the CPU parity oracle (oracle/pf_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline legs of ``bench.py``.  The product package never imports it.

``OracleNR`` mirrors the method set of the reference's ``KLUSolverSingleSlack`` /
``KLUSolver`` pybind11 classes (src/main.cpp:228-254): ``compute_pf``/``solve``,
``get_V``, ``get_Va``, ``get_Vm``, ``get_J``, ``get_nb_iter``, ``get_error``,
``converged``, ``reset``.
"""
import ctypes
import os
import subprocess

import numpy as np
from scipy import sparse

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libpf_oracle.so")
_lib = None

_i32p = ctypes.POINTER(ctypes.c_int32)
_f64p = ctypes.POINTER(ctypes.c_double)


def build():
    """Compile the oracle with its Makefile (gcc)."""
    subprocess.check_call(["make", "-s", "-C", _HERE])
    return _LIB_PATH


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    lib = ctypes.CDLL(_LIB_PATH)
    lib.oracle_solver_create.restype = ctypes.c_void_p
    lib.oracle_solver_create.argtypes = [ctypes.c_int]
    lib.oracle_solver_destroy.argtypes = [ctypes.c_void_p]
    lib.oracle_solver_reset.argtypes = [ctypes.c_void_p]
    lib.oracle_solver_compute_pf.restype = ctypes.c_int
    lib.oracle_solver_compute_pf.argtypes = [
        ctypes.c_void_p, ctypes.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, _i32p, ctypes.c_int, _f64p,
        _i32p, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_double]
    for nm in ("oracle_solver_get_V", "oracle_solver_get_Vm", "oracle_solver_get_Va"):
        getattr(lib, nm).argtypes = [ctypes.c_void_p, _f64p]
    for nm in ("oracle_solver_get_nb_iter", "oracle_solver_get_error", "oracle_solver_get_n",
               "oracle_solver_lu_nnz"):
        getattr(lib, nm).restype = ctypes.c_int
        getattr(lib, nm).argtypes = [ctypes.c_void_p]
    lib.oracle_solver_get_J.restype = ctypes.c_int
    lib.oracle_solver_get_J.argtypes = [ctypes.c_void_p, _i32p, _i32p, _i32p, _f64p]
    lib.oracle_contingency_analysis.restype = ctypes.c_int
    lib.oracle_contingency_analysis.argtypes = [
        ctypes.c_int, ctypes.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, _i32p, ctypes.c_int, _f64p,
        _i32p, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
        ctypes.c_int, ctypes.c_int, _i32p, _i32p, _i32p, _f64p, _f64p, _i32p, _i32p, _i32p]
    lib.oracle_time_series.restype = ctypes.c_int
    lib.oracle_time_series.argtypes = [
        ctypes.c_int, ctypes.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, ctypes.c_int, _f64p, _i32p,
        ctypes.c_int, _f64p, _i32p, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
        ctypes.c_double, ctypes.c_int, _f64p, _i32p, _i32p, _i32p]
    _lib = lib
    return lib


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).ravel())


def _c128(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.complex128).ravel())


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())


def _p(a, t):
    return a.ctypes.data_as(t)


def _csc(Ybus):
    Y = sparse.csc_matrix(Ybus)
    Y.sum_duplicates()
    Y.sort_indices()
    return Y


class OracleNR:
    """CPU restatement of KLUSolverSingleSlack (distributed=False) / KLUSolver (True)."""

    def __init__(self, distributed=False):
        self._lib = _load()
        self._h = self._lib.oracle_solver_create(1 if distributed else 0)
        self.distributed = bool(distributed)
        self._keep = None

    def __del__(self):
        try:
            if self._h:
                self._lib.oracle_solver_destroy(self._h)
                self._h = None
        except Exception:
            pass

    def reset(self):
        self._lib.oracle_solver_reset(self._h)

    def compute_pf(self, Ybus, V, Sbus, slack_ids, slack_weights, pv, pq, max_iter, tol):
        Y = _csc(Ybus)
        n = Y.shape[0]
        V = _c128(V)
        Sbus = _c128(Sbus)
        if Sbus.size != n or V.size != n or Y.shape[1] != n:
            raise RuntimeError("size mismatch between Ybus, V and Sbus")
        Yp, Yi, Yx = _i32(Y.indptr), _i32(Y.indices), _c128(Y.data)
        sl, w, pv, pq = _i32(slack_ids), _f64(slack_weights), _i32(pv), _i32(pq)
        if w.size != n:
            w = np.zeros(n)
            w[sl] = 1.0 / max(sl.size, 1)
        self._keep = (Yp, Yi, Yx, V, Sbus, sl, w, pv, pq)
        r = self._lib.oracle_solver_compute_pf(
            self._h, n, _p(Yp, _i32p), _p(Yi, _i32p), _p(Yx.view(np.float64), _f64p),
            _p(V.view(np.float64), _f64p), _p(Sbus.view(np.float64), _f64p), _p(sl, _i32p), sl.size,
            _p(w, _f64p), _p(pv, _i32p), pv.size, _p(pq, _i32p), pq.size, int(max_iter), float(tol))
        if r < 0:
            raise RuntimeError("oracle: invalid sizes")
        return bool(r)

    solve = compute_pf

    def _n(self):
        return self._lib.oracle_solver_get_n(self._h)

    def get_V(self):
        out = np.zeros(self._n(), dtype=np.complex128)
        self._lib.oracle_solver_get_V(self._h, _p(out.view(np.float64), _f64p))
        return out

    def get_Vm(self):
        out = np.zeros(self._n())
        self._lib.oracle_solver_get_Vm(self._h, _p(out, _f64p))
        return out

    def get_Va(self):
        out = np.zeros(self._n())
        self._lib.oracle_solver_get_Va(self._h, _p(out, _f64p))
        return out

    def get_nb_iter(self):
        return self._lib.oracle_solver_get_nb_iter(self._h)

    def get_error(self):
        return self._lib.oracle_solver_get_error(self._h)

    def converged(self):
        return self.get_error() == 0

    def lu_nnz(self):
        return self._lib.oracle_solver_lu_nnz(self._h)

    def get_J(self):
        m = ctypes.c_int(0)
        nz = self._lib.oracle_solver_get_J(self._h, ctypes.byref(m), None, None, None)
        if nz < 0:
            raise RuntimeError("J is not available before a call to compute_pf")
        Jp = np.zeros(m.value + 1, dtype=np.int32)
        Ji = np.zeros(nz, dtype=np.int32)
        Jx = np.zeros(nz)
        self._lib.oracle_solver_get_J(self._h, None, _p(Jp, _i32p), _p(Ji, _i32p), _p(Jx, _f64p))
        return sparse.csc_matrix((Jx, Ji, Jp), shape=(m.value, m.value))


def contingency_analysis(Ybus, Sbus, Vinit, slack_ids, slack_weights, pv, pq, coeffs, max_iter=10,
                         tol=1e-8, sn_mva=1.0, distributed=False, init_from_n=False):
    """Sequential N-1/N-k loop (ContingencyAnalysis::compute semantics).

    ``coeffs`` is a list (one entry per case) of lists of ``(row, col, y)`` Ybus
    coefficients to remove.  Returns ``(n_conv, V[ncases, n], conv, iters, errs)``.
    """
    lib = _load()
    Y = _csc(Ybus)
    n = Y.shape[0]
    Yp, Yi, Yx = _i32(Y.indptr), _i32(Y.indices), _c128(Y.data)
    Sbus, Vinit = _c128(Sbus), _c128(Vinit)
    sl, w, pv, pq = _i32(slack_ids), _f64(slack_weights), _i32(pv), _i32(pq)
    ncases = len(coeffs)
    cptr = np.zeros(ncases + 1, dtype=np.int32)
    rows, cols, vals = [], [], []
    for c, lst in enumerate(coeffs):
        cptr[c + 1] = cptr[c] + len(lst)
        for (r, cc, y) in lst:
            rows.append(r)
            cols.append(cc)
            vals.append(y)
    crow, ccol, cval = _i32(rows), _i32(cols), _c128(vals)
    if crow.size == 0:
        crow, ccol, cval = np.zeros(1, np.int32), np.zeros(1, np.int32), np.zeros(1, np.complex128)
    Vout = np.zeros((ncases, n), dtype=np.complex128)
    conv = np.zeros(ncases, dtype=np.int32)
    iters = np.zeros(ncases, dtype=np.int32)
    errs = np.zeros(ncases, dtype=np.int32)
    ok = lib.oracle_contingency_analysis(
        1 if distributed else 0, n, _p(Yp, _i32p), _p(Yi, _i32p), _p(Yx.view(np.float64), _f64p),
        _p(Sbus.view(np.float64), _f64p), _p(Vinit.view(np.float64), _f64p), _p(sl, _i32p), sl.size,
        _p(w, _f64p), _p(pv, _i32p), pv.size, _p(pq, _i32p), pq.size, int(max_iter), float(tol),
        float(sn_mva), 1 if init_from_n else 0, ncases, _p(cptr, _i32p), _p(crow, _i32p), _p(ccol, _i32p),
        _p(cval.view(np.float64), _f64p), _p(Vout.view(np.float64), _f64p), _p(conv, _i32p),
        _p(iters, _i32p), _p(errs, _i32p))
    return ok, Vout, conv.astype(bool), iters, errs


def time_series(Ybus, Sbus0, Sbuses, Vinit, slack_ids, slack_weights, pv, pq, max_iter=10, tol=1e-8,
                sn_mva=1.0, distributed=False, init_from_n=False):
    """Sequential warm-started time series (TimeSeries::compute_Vs semantics).

    Returns ``(status, V[nsteps, n], conv, iters, errs)``.
    """
    lib = _load()
    Y = _csc(Ybus)
    n = Y.shape[0]
    Yp, Yi, Yx = _i32(Y.indptr), _i32(Y.indices), _c128(Y.data)
    Sb = np.ascontiguousarray(np.asarray(Sbuses, dtype=np.complex128))
    nsteps = Sb.shape[0]
    Sbus0, Vinit = _c128(Sbus0), _c128(Vinit)
    sl, w, pv, pq = _i32(slack_ids), _f64(slack_weights), _i32(pv), _i32(pq)
    Vout = np.zeros((nsteps, n), dtype=np.complex128)
    conv = np.zeros(nsteps, dtype=np.int32)
    iters = np.zeros(nsteps, dtype=np.int32)
    errs = np.zeros(nsteps, dtype=np.int32)
    st = lib.oracle_time_series(
        1 if distributed else 0, n, _p(Yp, _i32p), _p(Yi, _i32p), _p(Yx.view(np.float64), _f64p),
        _p(Sbus0.view(np.float64), _f64p), _p(Sb.view(np.float64), _f64p), nsteps,
        _p(Vinit.view(np.float64), _f64p), _p(sl, _i32p), sl.size, _p(w, _f64p), _p(pv, _i32p), pv.size,
        _p(pq, _i32p), pq.size, int(max_iter), float(tol), float(sn_mva), 1 if init_from_n else 0,
        _p(Vout.view(np.float64), _f64p), _p(conv, _i32p), _p(iters, _i32p), _p(errs, _i32p))
    return st, Vout, conv.astype(bool), iters, errs
