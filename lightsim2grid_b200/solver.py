"""Solver classes with the reference's pybind11 method set, on the GPU engine.

Reference bindings: ``KLUSolverSingleSlack`` / ``KLUSolver`` (src/main.cpp:228-254), the
``SolverType`` and ``ErrorType`` enums (src/main.cpp:118-160, src/ChooseSolver.hpp:17-25,
src/Utils.hpp:47-56).  The new solver types are appended after the reference's members so
that every reference ordinal keeps its value.
"""
import enum
import time

import numpy as np
from scipy import sparse

from . import _native as nat


class SolverType(enum.IntEnum):
    """Members 0-21 are the reference's (src/ChooseSolver.hpp:17-25); 22-28 are this engine's."""

    SparseLU = 0
    KLU = 1
    GaussSeidel = 2
    DC = 3
    GaussSeidelSynch = 4
    NICSLU = 5
    SparseLUSingleSlack = 6
    KLUSingleSlack = 7
    NICSLUSingleSlack = 8
    KLUDC = 9
    NICSLUDC = 10
    CKTSO = 11
    CKTSOSingleSlack = 12
    CKTSODC = 13
    FDPF_XB_SparseLU = 14
    FDPF_BX_SparseLU = 15
    FDPF_XB_KLU = 16
    FDPF_BX_KLU = 17
    FDPF_XB_NICSLU = 18
    FDPF_BX_NICSLU = 19
    FDPF_XB_CKTSO = 20
    FDPF_BX_CKTSO = 21
    #: Newton-Raphson on the GPU, distributed slack, FP64 LU (drop-in for KLU)
    GPUNR = 22
    #: Newton-Raphson on the GPU, single slack, FP64 LU (drop-in for KLUSingleSlack)
    GPUNRSingleSlack = 23
    #: distributed slack, FP32 LU and solves, FP64 mismatch / update / convergence test
    GPUNRMixed = 24
    #: single slack, FP32 LU and solves, FP64 mismatch / update / convergence test
    GPUNRMixedSingleSlack = 25
    #: DC power flow on the GPU, FP64 (drop-in for KLUDC)
    GPUDC = 26
    #: fast decoupled power flow on the GPU, XB method, FP64 (drop-in for FDPF_XB_KLU)
    GPUFDPF_XB = 27
    #: fast decoupled power flow on the GPU, BX method, FP64 (drop-in for FDPF_BX_KLU)
    GPUFDPF_BX = 28


class FDPFMethod(enum.IntEnum):
    """src/BaseConstants.hpp:35."""

    XB = 0
    BX = 1


class ErrorType(enum.IntEnum):
    """src/Utils.hpp:47-56."""

    NoError = 0
    SingularMatrix = 1
    TooManyIterations = 2
    InifiniteValue = 3
    SolverAnalyze = 4
    SolverFactor = 5
    SolverReFactor = 6
    SolverSolve = 7
    NotInitError = 8
    LicenseError = 9


GPU_SOLVERS = (SolverType.GPUNR, SolverType.GPUNRSingleSlack, SolverType.GPUNRMixed,
               SolverType.GPUNRMixedSingleSlack, SolverType.GPUFDPF_XB, SolverType.GPUFDPF_BX)

#: fast decoupled solver types and their method
FDPF_SOLVERS = {SolverType.GPUFDPF_XB: FDPFMethod.XB, SolverType.GPUFDPF_BX: FDPFMethod.BX}


def solver_flags(solver_type):
    """``(distributed, precision)`` of a GPU solver type (fast decoupled: ``(False, 0)``, the
    slack weights enter through pvpq and the mismatch)."""
    st = SolverType(solver_type)
    if st not in GPU_SOLVERS:
        raise RuntimeError("Solver type {} is not available in lightsim2grid_b200 (available: {})".format(
            st.name, ", ".join(s.name for s in GPU_SOLVERS)))
    distributed = st in (SolverType.GPUNR, SolverType.GPUNRMixed)
    precision = 1 if st in (SolverType.GPUNRMixed, SolverType.GPUNRMixedSingleSlack) else 0
    return distributed, precision


def canonical_csc(Ybus):
    """CSC with summed duplicates and sorted indices (newtonpf's requirement, _newtonpf.py:49-56)."""
    Y = Ybus if sparse.isspmatrix_csc(Ybus) else sparse.csc_matrix(Ybus)
    if not Y.has_canonical_format:
        Y = Y.copy()
        Y.sum_duplicates()
        if not Y.has_canonical_format:
            raise RuntimeError("Your matrix should be in a canonical format.")
    return Y


class Plan:
    """Owns one native plan (pattern, ordering, pivots, device schedules)."""

    def __init__(self, Ybus, V0, Sbus, slack_ids, slack_weights, pv, pq, distributed=False, precision=0,
                 threads=0, lu_placement=0, fuse_forward=0, fp64_fallback=0, max_ctas_per_sm=0, refine=0,
                 refine_threshold=0.0, lu_reuse_threshold=0.0, dc=False, fdpf=None, batch_layout=0, ordering=0,
                 placement=0, level_slack=0, handoff_lanes=0):
        self._lib = nat.load()
        Y = canonical_csc(Ybus)
        n = Y.shape[0]
        if Y.shape[1] != n:
            raise RuntimeError("Ybus must be square")
        self.n = n
        self.Yp, self.Yi = nat.as_i32(Y.indptr), nat.as_i32(Y.indices)
        self.Yx = nat.as_c128(Y.data).ravel()
        V0 = nat.as_c128(V0).ravel()
        Sbus = nat.as_c128(Sbus).ravel()
        if V0.size != n or Sbus.size != n:
            raise RuntimeError("Size of V (init voltages) and Sbus should be the same as the size of Ybus. "
                               "Currently: V ({}), Sbus ({}), Ybus ({}, {}).".format(V0.size, Sbus.size, n, n))
        self.slack_ids = nat.as_i32(slack_ids)
        w = nat.as_f64(slack_weights)
        if w.size != n:
            raise RuntimeError("slack_weights must have one entry per bus")
        self.weights = w
        self.pv, self.pq = nat.as_i32(pv), nat.as_i32(pq)
        self.distributed, self.precision = bool(distributed), int(precision)
        opt = nat.PfOptions(precision=self.precision, threads=int(threads), lu_placement=int(lu_placement),
                            fuse_forward=int(fuse_forward), pivot_threshold=0.0,
                            fp64_fallback=int(fp64_fallback), max_ctas_per_sm=int(max_ctas_per_sm),
                            refine=int(refine), refine_threshold=float(refine_threshold),
                            lu_reuse_threshold=float(lu_reuse_threshold), batch_layout=int(batch_layout),
                            ordering=int(ordering), placement=int(placement), level_slack=int(level_slack),
                            handoff_lanes=int(handoff_lanes))
        h = nat.ctypes.c_void_p()
        self.dc = bool(dc)
        self.fdpf = fdpf is not None
        if self.fdpf:
            # fast decoupled (BaseFDPFAlgo): fdpf = (B', B''), grid-level n x n real matrices
            self.precision = 0
            Bs = []
            for B in fdpf:
                B = sparse.csc_matrix(B, dtype=np.float64)
                if B.shape != (n, n):
                    raise RuntimeError("B' and B'' must be {} x {}".format(n, n))
                B = B.copy()
                B.sum_duplicates()
                B.sort_indices()
                Bs.append((nat.as_i32(B.indptr), nat.as_i32(B.indices), nat.as_f64(B.data)))
            self._fdpf_arrays = Bs
            (bpp_, bpi, bpx), (bppp, bppi, bppx) = Bs
            rc = self._lib.pf_fdpf_plan_create(
                n, nat.ptr(self.Yp, nat.i32p), nat.ptr(self.Yi, nat.i32p), nat.cptr(self.Yx),
                nat.ptr(bpp_, nat.i32p), nat.ptr(bpi, nat.i32p), nat.ptr(bpx, nat.f64p), nat.ptr(bppp, nat.i32p),
                nat.ptr(bppi, nat.i32p), nat.ptr(bppx, nat.f64p), nat.ptr(self.slack_ids, nat.i32p),
                self.slack_ids.size, nat.ptr(w, nat.f64p), nat.ptr(self.pv, nat.i32p), self.pv.size,
                nat.ptr(self.pq, nat.i32p), self.pq.size, nat.ctypes.byref(opt), nat.ctypes.byref(h))
            nat.check(rc, "pf_fdpf_plan_create", self._lib)
        elif self.dc:
            # DC power flow (BaseDCAlgo): Ybus is the DC admittance matrix, FP64
            self.precision = 0
            rc = self._lib.pf_dc_plan_create(
                n, nat.ptr(self.Yp, nat.i32p), nat.ptr(self.Yi, nat.i32p), nat.cptr(self.Yx),
                nat.ptr(self.slack_ids, nat.i32p), self.slack_ids.size, nat.ptr(self.pv, nat.i32p), self.pv.size,
                nat.ptr(self.pq, nat.i32p), self.pq.size, nat.ctypes.byref(opt), nat.ctypes.byref(h))
            nat.check(rc, "pf_dc_plan_create", self._lib)
        else:
            rc = self._lib.pf_plan_create(
                n, nat.ptr(self.Yp, nat.i32p), nat.ptr(self.Yi, nat.i32p), nat.cptr(self.Yx), nat.cptr(V0),
                nat.cptr(Sbus), nat.ptr(self.slack_ids, nat.i32p), self.slack_ids.size, nat.ptr(w, nat.f64p),
                nat.ptr(self.pv, nat.i32p), self.pv.size, nat.ptr(self.pq, nat.i32p), self.pq.size,
                1 if distributed else 0, nat.ctypes.byref(opt), nat.ctypes.byref(h))
            nat.check(rc, "pf_plan_create", self._lib)
        self._h = h

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                self._lib.pf_plan_destroy(self._h)
                self._h = None
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def same_structure(self, Y, slack_ids, pv, pq):
        return (Y.shape[0] == self.n and np.array_equal(nat.as_i32(Y.indptr), self.Yp)
                and np.array_equal(nat.as_i32(Y.indices), self.Yi)
                and np.array_equal(nat.as_i32(slack_ids), self.slack_ids)
                and np.array_equal(nat.as_i32(pv), self.pv) and np.array_equal(nat.as_i32(pq), self.pq))

    def set_ybus_values(self, data):
        data = nat.as_c128(data).ravel()
        if not np.array_equal(data, self.Yx):
            self.Yx = data.copy()
            nat.check(self._lib.pf_set_ybus_values(self._h, nat.cptr(self.Yx)), "pf_set_ybus_values", self._lib)

    def info(self):
        inf = nat.PfPlanInfo()
        nat.check(self._lib.pf_plan_info_get(self._h, nat.ctypes.byref(inf)), "pf_plan_info_get", self._lib)
        return inf.as_dict()

    def timers(self):
        out = np.zeros(6)
        nat.check(self._lib.pf_timers(self._h, nat.ptr(out, nat.f64p), 6), "pf_timers", self._lib)
        return out

    def solve(self, V0, Sbus, max_iter, tol):
        V0 = nat.as_c128(V0).ravel()
        Sbus = nat.as_c128(Sbus).ravel()
        if V0.size != self.n or Sbus.size != self.n:
            raise RuntimeError("Size of V (init voltages) and Sbus should be the same as the size of Ybus.")
        Vout = np.zeros(self.n, dtype=np.complex128)
        conv, it, err = (nat.ctypes.c_int(0) for _ in range(3))
        rc = self._lib.pf_solve(self._h, nat.cptr(V0), nat.cptr(Sbus), int(max_iter), float(tol), nat.cptr(Vout),
                                nat.ctypes.byref(conv), nat.ctypes.byref(it), nat.ctypes.byref(err))
        nat.check(rc, "pf_solve", self._lib)
        return Vout, bool(conv.value), it.value, err.value

    def get_J(self):
        m = nat.ctypes.c_int(0)
        nz = self._lib.pf_get_J(self._h, nat.ctypes.byref(m), None, None, None)
        if nz < 0:
            raise RuntimeError(nat.last_error(self._lib))
        Jp = np.zeros(m.value + 1, dtype=np.int32)
        Ji = np.zeros(nz, dtype=np.int32)
        Jx = np.zeros(nz)
        rc = self._lib.pf_get_J(self._h, None, nat.ptr(Jp, nat.i32p), nat.ptr(Ji, nat.i32p), nat.ptr(Jx, nat.f64p))
        if rc < 0:
            raise RuntimeError(nat.last_error(self._lib))
        return sparse.csc_matrix((Jx, Ji, Jp), shape=(m.value, m.value))

    def batch_n1(self, coeffs, V0, Sbus, max_iter, tol):
        """``coeffs``: list (one per case) of lists of ``(row, col, y)`` to remove from Ybus."""
        ncases = len(coeffs)
        cptr_ = np.zeros(ncases + 1, dtype=np.int32)
        rows, cols, vals = [], [], []
        for c, lst in enumerate(coeffs):
            cptr_[c + 1] = cptr_[c] + len(lst)
            for (r, cc, y) in lst:
                rows.append(r)
                cols.append(cc)
                vals.append(y)
        return self.batch_n1_arrays(cptr_, rows, cols, vals, V0, Sbus, max_iter, tol)

    def batch_n1_arrays(self, case_ptr, rows, cols, vals, V0, Sbus, max_iter, tol, out=None):
        """N-1 batch from flat coefficient arrays.  ``out``: optional ``(V[ncases, n] complex128,
        conv, iters, errs int32[ncases])`` arrays to write into (e.g. views of pinned host memory,
        which the device copies into at full bus speed); fresh arrays otherwise."""
        case_ptr = nat.as_i32(case_ptr)
        ncases = case_ptr.size - 1
        rows, cols = nat.as_i32(rows), nat.as_i32(cols)
        vals = nat.as_c128(vals).ravel()
        if rows.size == 0:
            rows, cols, vals = np.zeros(1, np.int32), np.zeros(1, np.int32), np.zeros(1, np.complex128)
        V0 = nat.as_c128(V0).ravel()
        Sbus = nat.as_c128(Sbus).ravel()
        if out is not None:
            Vout, conv, iters, errs = out
            ok = (Vout.dtype == np.complex128 and Vout.shape == (ncases, self.n) and Vout.flags.c_contiguous
                  and all(a.dtype == np.int32 and a.size >= max(ncases, 1) and a.flags.c_contiguous
                          for a in (conv, iters, errs)))
            if not ok:
                raise ValueError("out arrays must be V[ncases, n] complex128 and three int32[ncases], contiguous")
        else:
            Vout = np.empty((ncases, self.n), dtype=np.complex128)  # every row is written
            conv = np.zeros(max(ncases, 1), dtype=np.int32)
            iters = np.zeros(max(ncases, 1), dtype=np.int32)
            errs = np.zeros(max(ncases, 1), dtype=np.int32)
        rc = self._lib.pf_batch_n1(self._h, ncases, nat.ptr(case_ptr, nat.i32p), nat.ptr(rows, nat.i32p),
                                   nat.ptr(cols, nat.i32p), nat.cptr(vals), nat.cptr(V0), nat.cptr(Sbus),
                                   int(max_iter), float(tol), nat.cptr(Vout), nat.ptr(conv, nat.i32p),
                                   nat.ptr(iters, nat.i32p), nat.ptr(errs, nat.i32p))
        nat.check(rc, "pf_batch_n1", self._lib)
        return Vout, conv[:ncases].astype(bool), iters[:ncases], errs[:ncases]

    def batch_ts(self, Sbuses, V0, nchunks, max_iter, tol, out=None):
        """Time series.  ``out``: optional ``(V[nsteps, n] complex128, conv, iters, errs int32)``
        arrays to write into (pinned host memory takes the rows straight from the kernel)."""
        Sb = nat.as_c128(Sbuses)
        nsteps = Sb.shape[0]
        V0 = nat.as_c128(V0).ravel()
        if out is not None:
            Vout, conv, iters, errs = out
            ok = (Vout.dtype == np.complex128 and Vout.shape == (nsteps, self.n) and Vout.flags.c_contiguous
                  and all(a.dtype == np.int32 and a.size >= max(nsteps, 1) and a.flags.c_contiguous
                          for a in (conv, iters, errs)))
            if not ok:
                raise ValueError("out arrays must be V[nsteps, n] complex128 and three int32[nsteps], contiguous")
        else:
            Vout = np.zeros((nsteps, self.n), dtype=np.complex128)
            conv = np.zeros(max(nsteps, 1), dtype=np.int32)
            iters = np.zeros(max(nsteps, 1), dtype=np.int32)
            errs = np.zeros(max(nsteps, 1), dtype=np.int32)
        status = nat.ctypes.c_int(0)
        rc = self._lib.pf_batch_ts(self._h, nsteps, nat.cptr(Sb), nat.cptr(V0), int(nchunks), int(max_iter),
                                   float(tol), nat.cptr(Vout), nat.ptr(conv, nat.i32p), nat.ptr(iters, nat.i32p),
                                   nat.ptr(errs, nat.i32p), nat.ctypes.byref(status))
        nat.check(rc, "pf_batch_ts", self._lib)
        return status.value, Vout, conv[:nsteps].astype(bool), iters[:nsteps], errs[:nsteps]


class _GPUNRSolverBase:
    """Method set of KLUSolverSingleSlack / KLUSolver (src/main.cpp:228-254)."""

    _distributed = False
    _precision = 0
    _dc = False

    def __init__(self, **plan_options):
        self._plan = None
        self._plan_options = plan_options
        self.reset()

    def reset(self):
        """Forget the pattern, ordering and pivots (the next call re-analyses)."""
        self._plan = None
        self._V = np.zeros(0, dtype=np.complex128)
        self._err = ErrorType.NotInitError
        self._nb_iter = 0
        self._timer_total = 0.0

    def compute_pf(self, Ybus, V, Sbus, slack_ids, slack_weights, pv, pq, max_iter, tol):
        t0 = time.perf_counter()
        Y = canonical_csc(Ybus)
        n = Y.shape[0]
        V = nat.as_c128(V).ravel()
        Sbus = nat.as_c128(Sbus).ravel()
        if Sbus.size != n or Y.shape[1] != n:
            raise RuntimeError("compute_pf: Size of the Sbus should be the same as the size of Ybus. Currently: "
                               "Sbus  ({}) and Ybus ({}, {}).".format(Sbus.size, Y.shape[0], Y.shape[1]))
        if V.size != n:
            raise RuntimeError("compute_pf: Size of V (init voltages) should be the same as the size of Ybus. "
                               "Currently: V  ({}) and Ybus ({}, {}).".format(V.size, Y.shape[0], Y.shape[1]))
        w = nat.as_f64(slack_weights)
        if w.size != n:
            w = np.zeros(n)
            sl = nat.as_i32(slack_ids)
            w[sl] = 1.0 / max(sl.size, 1)
        if self._plan is None or not self._plan.same_structure(Y, slack_ids, pv, pq):
            self._plan = Plan(Y, V, Sbus, slack_ids, w, pv, pq, distributed=self._distributed,
                              precision=self._precision, dc=self._dc, **self._plan_options)
        else:
            self._plan.set_ybus_values(Y.data)
        Vout, conv, it, err = self._plan.solve(V, Sbus, max_iter, tol)
        self._V = Vout
        self._nb_iter = it
        self._err = ErrorType(err)
        self._timer_total = time.perf_counter() - t0
        return conv

    solve = compute_pf

    def get_V(self):
        return self._V.copy()

    def get_Va(self):
        return np.angle(self._V)

    def get_Vm(self):
        return np.abs(self._V)

    def get_J(self):
        if self._plan is None:
            raise RuntimeError("get_J: no power flow has been computed")
        return self._plan.get_J()

    def get_error(self):
        return self._err

    def get_nb_iter(self):
        return self._nb_iter

    def converged(self):
        return self._err == ErrorType.NoError

    def get_timers(self):
        """``(timer_Fx, timer_solve, timer_check, timer_total)`` as in BaseAlgo.hpp:91-97.

        The engine fuses the phases in one kernel: the kernel time is reported as the
        solve time and the mismatch / check timers are 0.
        """
        t = self._plan.timers() if self._plan is not None else np.zeros(6)
        return (0.0, float(t[3]), 0.0, self._timer_total)

    def get_plan(self):
        return self._plan


class GPUNRSolverSingleSlack(_GPUNRSolverBase):
    """Drop-in for KLUSolverSingleSlack (single slack, FP64)."""

    _distributed = False
    _precision = 0


class GPUNRSolver(_GPUNRSolverBase):
    """Drop-in for KLUSolver (distributed slack, FP64)."""

    _distributed = True
    _precision = 0


class GPUNRMixedSolverSingleSlack(_GPUNRSolverBase):
    """Single slack, FP32 LU and solves, FP64 mismatch, update and convergence test."""

    _distributed = False
    _precision = 1


class GPUDCSolver(_GPUNRSolverBase):
    """Drop-in for KLUDCSolver (BaseDCAlgo, src/powerflow_algorithm/BaseDCAlgo.tpp): one FP64
    linear solve of B theta = Re(Sbus) with B = Re(Ybus) of the DC Ybus, without the slack."""

    _dc = True

    def get_J(self):
        raise RuntimeError("get_J: a DC solver has no Jacobian")


def _fingerprint(B):
    B = sparse.csc_matrix(B, dtype=np.float64).copy()
    B.sum_duplicates()
    B.sort_indices()
    return B.shape, B.indptr.copy(), B.indices.copy(), B.data.copy()


def _same_fingerprint(a, b):
    return a[0] == b[0] and all(np.array_equal(x, y) for x, y in zip(a[1:], b[1:]))


class _GPUFDPFSolverBase(_GPUNRSolverBase):
    """Drop-in for the reference's FDPF solvers (BaseFDPFAlgo, src/powerflow_algorithm/
    BaseFDPFAlgo.tpp:11-214; bound as FDPF_XB_* / FDPF_BX_*).  The reference's solver takes B'
    and B'' from the grid model it is attached to (GridModel::fillBp_Bpp); here
    ``set_gridmodel(grid)`` (a ``lightsim2grid_b200.GridModel``) or ``set_Bp_Bpp(Bp, Bpp)``
    gives them.  The factors are kept while B', B'', the pattern, slacks, PV and PQ stay the same."""

    _method = FDPFMethod.XB

    def __init__(self, **plan_options):
        self._Bp = self._Bpp = None
        self._grid = None
        self._bfp = []
        super().__init__(**plan_options)

    def set_gridmodel(self, grid):
        self._grid = grid
        self._plan = None

    def set_Bp_Bpp(self, Bp, Bpp):
        self._Bp, self._Bpp = sparse.csc_matrix(Bp), sparse.csc_matrix(Bpp)
        self._grid = None
        self._plan = None

    def _matrices(self):
        if self._grid is not None:
            return self._grid.get_Bp_Bpp(self._method)
        if self._Bp is None:
            raise RuntimeError("compute_pf: no B' / B'' (call set_gridmodel or set_Bp_Bpp first)")
        return self._Bp, self._Bpp

    def compute_pf(self, Ybus, V, Sbus, slack_ids, slack_weights, pv, pq, max_iter, tol):
        t0 = time.perf_counter()
        Y = canonical_csc(Ybus)
        n = Y.shape[0]
        V = nat.as_c128(V).ravel()
        Sbus = nat.as_c128(Sbus).ravel()
        if Sbus.size != n or Y.shape[1] != n:
            raise RuntimeError("BaseFDPFAlgo::compute_pf: Size of the Sbus should be the same as the size of Ybus. "
                               "Currently: Sbus  ({}) and Ybus ({}, {}).".format(Sbus.size, Y.shape[0], Y.shape[1]))
        if V.size != n:
            raise RuntimeError("BaseFDPFAlgo::compute_pf: Size of V (init voltages) should be the same as the size "
                               "of Ybus. Currently: V  ({}) and Ybus ({}, {}).".format(V.size, Y.shape[0], Y.shape[1]))
        w = nat.as_f64(slack_weights)
        if w.size != n:
            w = np.zeros(n)
            sl = nat.as_i32(slack_ids)
            w[sl] = 1.0 / max(sl.size, 1)
        Bp, Bpp = self._matrices()
        fp = [_fingerprint(B) for B in (Bp, Bpp)]
        same = (self._plan is not None and self._plan.same_structure(Y, slack_ids, pv, pq)
                and all(_same_fingerprint(a, b) for a, b in zip(fp, self._bfp)))
        if not same:
            self._plan = Plan(Y, V, Sbus, slack_ids, w, pv, pq, fdpf=(Bp, Bpp), **self._plan_options)
            self._bfp = fp
        else:
            self._plan.set_ybus_values(Y.data)
        Vout, conv, it, err = self._plan.solve(V, Sbus, max_iter, tol)
        self._V = Vout
        self._nb_iter = it
        self._err = ErrorType(err)
        self._timer_total = time.perf_counter() - t0
        return conv

    solve = compute_pf

    def get_J(self):
        raise RuntimeError("get_J: a fast decoupled solver has no Jacobian")

    def _sub(self, which):
        if self._plan is None:
            raise RuntimeError("no power flow has been computed")
        p = self._plan
        Bp, Bpp = self._matrices()
        pvpq = np.r_[p.slack_ids[1:], p.pv, p.pq].astype(np.int64)
        ids = pvpq if which == 0 else p.pq.astype(np.int64)
        B = sparse.csc_matrix(Bp if which == 0 else Bpp)
        return B[ids][:, ids].tocsc()

    def debug_get_Bp_python(self):
        """B'[pvpq, pvpq] as the solver uses it (BaseFDPFAlgo.hpp:47)."""
        return self._sub(0)

    def debug_get_Bpp_python(self):
        """B''[pq, pq] as the solver uses it (BaseFDPFAlgo.hpp:48)."""
        return self._sub(1)


class GPUFDPFSolverXB(_GPUFDPFSolverBase):
    """Drop-in for FDPF_XB_KLUSolver: B' without resistances, B'' with them."""

    _method = FDPFMethod.XB


class GPUFDPFSolverBX(_GPUFDPFSolverBase):
    """Drop-in for FDPF_BX_KLUSolver: B' with resistances, B'' without them."""

    _method = FDPFMethod.BX


class GPUNRMixedSolver(_GPUNRSolverBase):
    """Distributed slack, FP32 LU and solves, FP64 mismatch, update and convergence test."""

    _distributed = True
    _precision = 1


SOLVER_CLASSES = {
    SolverType.GPUNR: GPUNRSolver,
    SolverType.GPUNRSingleSlack: GPUNRSolverSingleSlack,
    SolverType.GPUNRMixed: GPUNRMixedSolver,
    SolverType.GPUNRMixedSingleSlack: GPUNRMixedSolverSingleSlack,
    SolverType.GPUDC: GPUDCSolver,
    SolverType.GPUFDPF_XB: GPUFDPFSolverXB,
    SolverType.GPUFDPF_BX: GPUFDPFSolverBX,
}
