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


def _coeff_arrays(coeffs):
    """CSR of the removal coefficients of each case: (cptr, rows, cols, values)."""
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
    return cptr, crow, ccol, cval


class ContingencyBatch:
    """An N-1 / N-k batch prepared for the oracle's C loop: Ybus, injections, start voltages and
    the removal coefficients converted to the C layout once, so that ``run`` times only the
    loop itself (ContingencyAnalysis::compute, ContingencyAnalysis.cpp:166-233: the base power
    flow, then every case).  ``run(threads)`` splits the cases into contiguous slices, one
    independent computer per host thread (the pattern of the reference's
    examples/computers_with_grid2op_multithreading.py:98-108); ctypes releases the GIL during
    the C call, so the slices run in parallel."""

    def __init__(self, Ybus, Sbus, Vinit, slack_ids, slack_weights, pv, pq, coeffs, max_iter=10, tol=1e-8,
                 sn_mva=1.0, distributed=False, init_from_n=False):
        self._lib = _load()
        Y = _csc(Ybus)
        self.n = n = Y.shape[0]
        self.Y = (_i32(Y.indptr), _i32(Y.indices), _c128(Y.data))
        self.Sbus, self.Vinit = _c128(Sbus), _c128(Vinit)
        self.sl, self.w, self.pv, self.pq = _i32(slack_ids), _f64(slack_weights), _i32(pv), _i32(pq)
        self.ncases = len(coeffs)
        self.coeffs = list(coeffs)
        self.args = (int(max_iter), float(tol), float(sn_mva), 1 if init_from_n else 0)
        self.distributed = 1 if distributed else 0
        self.Vout = np.zeros((self.ncases, n), dtype=np.complex128)
        self.conv = np.zeros(self.ncases, dtype=np.int32)
        self.iters = np.zeros(self.ncases, dtype=np.int32)
        self.errs = np.zeros(self.ncases, dtype=np.int32)
        self._slices = {}

    def _slice_arrays(self, threads):
        if threads not in self._slices:
            edges = (np.arange(threads + 1) * self.ncases) // threads
            self._slices[threads] = [(int(a), int(b), _coeff_arrays(self.coeffs[a:b]))
                                     for a, b in zip(edges[:-1], edges[1:])]
        return self._slices[threads]

    def _run_slice(self, lo, hi, arrs):
        if hi <= lo:
            return 1
        cptr, crow, ccol, cval = arrs
        Yp, Yi, Yx = self.Y
        max_iter, tol, sn_mva, init_n = self.args
        return self._lib.oracle_contingency_analysis(
            self.distributed, self.n, _p(Yp, _i32p), _p(Yi, _i32p), _p(Yx.view(np.float64), _f64p),
            _p(self.Sbus.view(np.float64), _f64p), _p(self.Vinit.view(np.float64), _f64p), _p(self.sl, _i32p),
            self.sl.size, _p(self.w, _f64p), _p(self.pv, _i32p), self.pv.size, _p(self.pq, _i32p), self.pq.size,
            max_iter, tol, sn_mva, init_n, hi - lo, _p(cptr, _i32p), _p(crow, _i32p), _p(ccol, _i32p),
            _p(cval.view(np.float64), _f64p), _p(self.Vout[lo:hi].view(np.float64), _f64p),
            _p(self.conv[lo:hi], _i32p), _p(self.iters[lo:hi], _i32p), _p(self.errs[lo:hi], _i32p))

    def prepare(self, threads):
        """Converts the slices for ``threads`` host threads (outside any timed region)."""
        self._slice_arrays(max(1, int(threads)))

    def run(self, threads=1):
        """Runs every case; returns (ok, V[ncases, n], conv, iters, errs, seconds of the loop)."""
        import threading
        import time

        threads = max(1, int(threads))
        parts = self._slice_arrays(threads)
        oks = [1] * len(parts)

        def work(t):
            oks[t] = self._run_slice(*parts[t])

        t0 = time.perf_counter()
        if threads == 1:
            work(0)
        else:
            th = [threading.Thread(target=work, args=(t,)) for t in range(len(parts))]
            for x in th:
                x.start()
            for x in th:
                x.join()
        dt = time.perf_counter() - t0
        return int(all(oks)), self.Vout, self.conv.astype(bool), self.iters, self.errs, dt


def contingency_analysis(Ybus, Sbus, Vinit, slack_ids, slack_weights, pv, pq, coeffs, max_iter=10,
                         tol=1e-8, sn_mva=1.0, distributed=False, init_from_n=False, threads=1):
    """N-1/N-k loop (ContingencyAnalysis::compute semantics), sequential per computer.

    ``coeffs`` is a list (one entry per case) of lists of ``(row, col, y)`` Ybus
    coefficients to remove.  ``threads`` > 1 splits the cases into contiguous slices, each
    solved by its own computer on its own host thread (same results: every case starts from
    ``Vinit`` and re-adds its coefficients).  Returns ``(ok, V[ncases, n], conv, iters, errs)``.
    """
    b = ContingencyBatch(Ybus, Sbus, Vinit, slack_ids, slack_weights, pv, pq, coeffs, max_iter, tol, sn_mva,
                         distributed, init_from_n)
    ok, V, conv, iters, errs, _ = b.run(threads)
    return ok, V, conv, iters, errs


def time_series_chunks(Ybus, Sbus0, Sbuses, Vinit, slack_ids, slack_weights, pv, pq, job_first, job_count,
                       max_iter=10, tol=1e-8, threads=1):
    """The chunked chains of a device time series, each chunk the reference's exact chain
    (TimeSeries::compute_Vs) over its snapshots from ``Vinit``, chunks spread over host
    threads.  Returns (V[nsteps, n], conv, iters, errs) with each chunk's rows in place (rows
    after a chunk's first divergence stay zero, errs NotInitError)."""
    import threading

    Sb = np.ascontiguousarray(np.asarray(Sbuses, dtype=np.complex128))
    nsteps, n = Sb.shape
    V = np.zeros((nsteps, n), np.complex128)
    conv = np.zeros(nsteps, bool)
    iters = np.zeros(nsteps, np.int32)
    errs = np.full(nsteps, 8, np.int32)
    jobs = [(int(a), int(c)) for a, c in zip(job_first, job_count)]
    threads = max(1, min(int(threads), len(jobs)))

    def work(t):
        for k in range(t, len(jobs), threads):
            a, c = jobs[k]
            _, Vk, ck, ik, ek = time_series(Ybus, Sbus0, Sb[a:a + c], Vinit, slack_ids, slack_weights, pv, pq,
                                            max_iter, tol)
            V[a:a + c], conv[a:a + c], iters[a:a + c], errs[a:a + c] = Vk, ck, ik, ek

    th = [threading.Thread(target=work, args=(t,)) for t in range(threads)]
    for x in th:
        x.start()
    for x in th:
        x.join()
    return V, conv, iters, errs


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
