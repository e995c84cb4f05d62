"""Fast decoupled power flow restated on the CPU with scipy (oracle for the GPU FDPF plans).

TEST INFRASTRUCTURE ONLY: imported by tests/ (and nothing in the product package).

Follows BaseFDPFAlgo::compute_pf (src/powerflow_algorithm/BaseFDPFAlgo.tpp:11-173) and
has_converged (BaseFDPFAlgo.hpp:118-170):
* pvpq = [slacks after the first, pv, pq] (retrieve_pv_with_slack, BaseAlgo.hpp:201-216);
* B'_ = B'[pvpq, pvpq], B''_ = B''[pq, pq] (fill_sparse_matrices, BaseFDPFAlgo.tpp:175-214),
  factorised once;
* slack_absorbed = Re(sum Sbus), never updated (:62);
* mis = (V conj(Ybus V) - Sbus + slack_absorbed w) / |V|, P = Re(mis)[pvpq], Q = Im(mis)[pq];
  converged when ||P||_inf < tol and ||Q||_inf < tol (BaseAlgo.cpp:131-141);
* per iteration: Va[pvpq] -= B'_^-1 P; t = exp(j Va); V = Vm t; (Vm, Va) = (|V|, arg V);
  mismatch (stop if converged); Vm[pq] -= B''_^-1 Q; V = Vm t (the same t); (Vm, Va) again;
  mismatch.  A non-finite mismatch is InifiniteValue (3): after a P half-step the loop stops
  there, after a Q half-step it stops after the next iteration's B' solve (one more iteration
  counted when max_iter allows); no convergence after max_iter is TooManyIterations (2).

Also restates the grid-level B' / B'' of a line-only grid (GridModel::fillBp_Bpp,
src/GridModel.cpp:1037-1064; get_fdpf_coeffs, TwoSidesContainer_rxh_A.hpp:810-837).
"""
import numpy as np
from scipy import sparse
from scipy.sparse.linalg import splu


def make_Bp_Bpp(n, f, t, r, x, h, status, method):
    """B', B'' (n x n CSC) for lines (from, to, r, x, total shunt h), method 0 = XB, 1 = BX."""
    on = np.asarray(status, bool)
    f, t = np.asarray(f)[on], np.asarray(t)[on]
    r, x, h = np.asarray(r)[on], np.asarray(x)[on], np.asarray(h, np.complex128)[on]
    Bp_trip, Bpp_trip = [], []
    for k in range(f.size):
        if method == 0:
            ys_bp, ys_bpp = 1.0 / complex(0.0, x[k]), 1.0 / complex(r[k], x[k])
        else:
            ys_bp, ys_bpp = 1.0 / complex(r[k], x[k]), 1.0 / complex(0.0, x[k])
        yff_bp = ys_bp.imag
        yff_bpp = ys_bpp.imag + (0.5 * h[k]).imag
        ytt_bpp = ys_bpp.imag + (0.5 * h[k]).imag
        a, b = int(f[k]), int(t[k])
        Bp_trip += [(a, a, -yff_bp), (b, b, -yff_bp), (a, b, yff_bp), (b, a, yff_bp)]
        Bpp_trip += [(a, a, -yff_bpp), (b, b, -ytt_bpp), (a, b, ys_bpp.imag), (b, a, ys_bpp.imag)]
    out = []
    for trip in (Bp_trip, Bpp_trip):
        rr = np.array([e[0] for e in trip], np.int64)
        cc = np.array([e[1] for e in trip], np.int64)
        vv = np.array([e[2] for e in trip], np.float64)
        B = sparse.csc_matrix((vv, (rr, cc)), shape=(n, n))
        B.sum_duplicates()
        B.sort_indices()
        out.append(B)
    return out[0], out[1]


def _mismatch(Y, V, Vm, Sbus, sa, w, pvpq, pq):
    mis = (V * np.conj(Y @ V) - Sbus + sa * w) / Vm
    finite = bool(np.all(np.isfinite(mis)))
    return mis.real[pvpq], mis.imag[pq], finite


def fdpf(Ybus, V0, Sbus, slack_ids, slack_weights, pv, pq, Bp, Bpp, max_iter, tol):
    """Returns (V, converged, iterations, error ordinal)."""
    Y = sparse.csr_matrix(Ybus)
    n = Y.shape[0]
    slack_ids = np.asarray(slack_ids, np.int64)
    pvpq = np.r_[slack_ids[1:], np.asarray(pv, np.int64), np.asarray(pq, np.int64)].astype(np.int64)
    pq = np.asarray(pq, np.int64)
    w = np.asarray(slack_weights, np.float64)
    Sbus = np.asarray(Sbus, np.complex128)
    Bp_ = sparse.csc_matrix(Bp)[pvpq][:, pvpq].tocsc()
    Bpp_ = sparse.csc_matrix(Bpp)[pq][:, pq].tocsc()
    try:
        lp = splu(Bp_) if pvpq.size else None
        lpp = splu(Bpp_) if pq.size else None
    except RuntimeError:
        return np.asarray(V0, np.complex128).copy(), False, 0, 5  # SolverFactor
    sa = float(np.sum(Sbus).real)
    V = np.asarray(V0, np.complex128).copy()
    Vm, Va = np.abs(V), np.angle(V)
    P, Q, _ = _mismatch(Y, V, Vm, Sbus, sa, w, pvpq, pq)
    norm = lambda a: np.max(np.abs(a)) if a.size else 0.0
    conv = norm(P) < tol and norm(Q) < tol
    it, err = 0, 0
    while not conv and it < max_iter:
        it += 1
        if lp is not None:
            Va[pvpq] -= lp.solve(P)
        t = np.cos(Va) + 1j * np.sin(Va)
        V = Vm * t
        Vm, Va = np.abs(V), np.angle(V)
        P, Q, finite = _mismatch(Y, V, Vm, Sbus, sa, w, pvpq, pq)
        if not finite:
            err = 3
            break
        if norm(P) < tol and norm(Q) < tol:
            conv = True
            break
        if lpp is not None:
            Vm[pq] -= lpp.solve(Q)
        V = Vm * t
        Vm, Va = np.abs(V), np.angle(V)
        P, Q, finite = _mismatch(Y, V, Vm, Sbus, sa, w, pvpq, pq)
        if not finite:
            err = 3
            if it < max_iter:
                it += 1
            break
        conv = norm(P) < tol and norm(Q) < tol
    if not conv and err == 0:
        err = 2
    return V, bool(conv), it, err
