"""Minimal grid container with the reference's Ybus / Sbus / PV / PQ conventions.

The reference's ``GridModel`` (src/GridModel.cpp, 2.9k lines) converts pandapower or
IIDM networks; only its solver-facing conventions matter for the power-flow path and
they are restated here:

* branch pi-model (src/element_container/TwoSidesContainer_rxh_A.hpp:921-940):
  ``ys = 1/(r + jx)``, ``y_ff = ys + h_or``, ``y_tt = ys + h_ex``, ``y_ft = y_tf = -ys``;
  a line's total shunt ``h`` is split half / half (LineContainer.cpp:27-33);
* Ybus assembly (GridModel.cpp:676-699): triplets of every element, duplicates summed,
  compressed column storage;
* Sbus (GridModel.cpp:701-716): generators minus loads, divided by ``sn_mva`` when it
  differs from 1;
* PV buses (GridModel.cpp:718-760): buses of voltage-regulating generators in generator
  order, de-duplicated, slack excluded; PQ buses: every other non-slack bus, ascending;
* slack weights (GeneratorContainer.cpp:119-156): normalised to sum to one.

Element data are given in per-unit on ``sn_mva`` except powers, which are in MW / MVAr.
"""
import numpy as np
from scipy import sparse


class Coeff(tuple):
    """``(row_id, col_id, value)``: one Ybus coefficient (src/Utils.hpp:60-64)."""

    __slots__ = ()

    def __new__(cls, row_id, col_id, value):
        return tuple.__new__(cls, (int(row_id), int(col_id), complex(value)))

    row_id = property(lambda self: self[0])
    col_id = property(lambda self: self[1])
    value = property(lambda self: self[2])


class GridModel:
    """Buses, branches (lines), generators and loads of one transmission grid."""

    def __init__(self, n_bus, sn_mva=1.0, init_vm_pu=1.04):
        self.n_bus = int(n_bus)
        self.sn_mva = float(sn_mva)
        self.init_vm_pu = float(init_vm_pu)
        self.bus_vn_kv = np.full(self.n_bus, 138.0)
        self.line_from = np.zeros(0, dtype=np.int64)
        self.line_to = np.zeros(0, dtype=np.int64)
        self.line_r = np.zeros(0)
        self.line_x = np.zeros(0)
        self.line_h = np.zeros(0, dtype=np.complex128)
        self.line_status = np.zeros(0, dtype=bool)
        self.gen_bus = np.zeros(0, dtype=np.int64)
        self.gen_p_mw = np.zeros(0)
        self.gen_vm_pu = np.zeros(0)
        self.gen_slack_weight = np.zeros(0)
        self.load_bus = np.zeros(0, dtype=np.int64)
        self.load_p_mw = np.zeros(0)
        self.load_q_mvar = np.zeros(0)
        self.sgen_bus = np.zeros(0, dtype=np.int64)
        self.sgen_p_mw = np.zeros(0)
        self._solver = None

    # ------------------------------------------------------------------ elements
    def init_powerlines(self, r, x, h, from_bus, to_bus):
        self.line_r = np.asarray(r, dtype=np.float64).copy()
        self.line_x = np.asarray(x, dtype=np.float64).copy()
        self.line_h = np.asarray(h, dtype=np.complex128).copy()
        self.line_from = np.asarray(from_bus, dtype=np.int64).copy()
        self.line_to = np.asarray(to_bus, dtype=np.int64).copy()
        self.line_status = np.ones(self.line_r.size, dtype=bool)

    def init_generators(self, p_mw, vm_pu, bus, slack_weight):
        self.gen_p_mw = np.asarray(p_mw, dtype=np.float64).copy()
        self.gen_vm_pu = np.asarray(vm_pu, dtype=np.float64).copy()
        self.gen_bus = np.asarray(bus, dtype=np.int64).copy()
        self.gen_slack_weight = np.asarray(slack_weight, dtype=np.float64).copy()

    def init_loads(self, p_mw, q_mvar, bus):
        self.load_p_mw = np.asarray(p_mw, dtype=np.float64).copy()
        self.load_q_mvar = np.asarray(q_mvar, dtype=np.float64).copy()
        self.load_bus = np.asarray(bus, dtype=np.int64).copy()

    def init_sgens(self, p_mw, bus):
        self.sgen_p_mw = np.asarray(p_mw, dtype=np.float64).copy()
        self.sgen_bus = np.asarray(bus, dtype=np.int64).copy()

    def deactivate_powerline(self, line_id):
        self.line_status[line_id] = False

    def reactivate_powerline(self, line_id):
        self.line_status[line_id] = True

    def nb_powerline(self):
        return int(self.line_r.size)

    def nb_trafo(self):
        return 0

    def total_bus(self):
        return self.n_bus

    def get_sn_mva(self):
        return self.sn_mva

    # ------------------------------------------------------------------ branch coefficients
    def branch_admittances(self):
        """``(y_ff, y_ft, y_tf, y_tt)`` per line (zero when the line is out of service)."""
        ys = 1.0 / (self.line_r + 1j * self.line_x)
        h_half = 0.5 * self.line_h
        on = self.line_status.astype(np.float64)
        y_ff = (ys + h_half) * on
        y_tt = (ys + h_half) * on
        y_ft = -ys * on
        y_tf = -ys * on
        return y_ff, y_ft, y_tf, y_tt

    def branch_coeffs(self, branch_ids):
        """Ybus coefficients of the given branches, in the reference's order.

        ContingencyAnalysis.cpp:97-105: ``(b1,b1,y_ff), (b2,b2,y_tt), (b1,b2,y_ft), (b2,b1,y_tf)``
        for every connected branch.
        """
        y_ff, y_ft, y_tf, y_tt = self.branch_admittances()
        out = []
        for br in branch_ids:
            if not self.line_status[br]:
                continue
            b1, b2 = int(self.line_from[br]), int(self.line_to[br])
            out.append(Coeff(b1, b1, y_ff[br]))
            out.append(Coeff(b2, b2, y_tt[br]))
            out.append(Coeff(b1, b2, y_ft[br]))
            out.append(Coeff(b2, b1, y_tf[br]))
        return out

    # ------------------------------------------------------------------ solver inputs
    def get_Ybus(self):
        """Ybus in canonical CSC form (duplicates summed, sorted indices)."""
        y_ff, y_ft, y_tf, y_tt = self.branch_admittances()
        on = self.line_status
        f, t = self.line_from[on], self.line_to[on]
        rows = np.concatenate([f, t, f, t])
        cols = np.concatenate([f, t, t, f])
        vals = np.concatenate([y_ff[on], y_tt[on], y_ft[on], y_tf[on]])
        Y = sparse.csc_matrix((vals, (rows, cols)), shape=(self.n_bus, self.n_bus), dtype=np.complex128)
        Y.sum_duplicates()
        Y.sort_indices()
        return Y

    def get_dcYbus(self):
        """DC Ybus (fillYbus with ac = false, GridModel.cpp:676-699): per branch in service
        y_ff = y_tt = 1/x, y_ft = y_tf = -1/x (TwoSidesContainer_rxh_A.hpp:933-939)."""
        on = self.line_status
        f, t = self.line_from[on], self.line_to[on]
        yd = (1.0 / (self.line_x[on] + 0j))
        rows = np.concatenate([f, t, f, t])
        cols = np.concatenate([f, t, t, f])
        vals = np.concatenate([yd, yd, -yd, -yd])
        Y = sparse.csc_matrix((vals, (rows, cols)), shape=(self.n_bus, self.n_bus), dtype=np.complex128)
        Y.sum_duplicates()
        Y.sort_indices()
        return Y

    def get_Bp_Bpp(self, method=0):
        """Grid-level B' and B'' of the fast decoupled power flow, ``method`` 0 = XB, 1 = BX
        (GridModel::fillBp_Bpp, GridModel.cpp:1037-1064; line terms TwoSidesContainer_rxh_A.hpp:
        503-580 with get_fdpf_coeffs :810-837).  Per line in service, with ys' = 1/(j x) and
        ys'' = 1/(r + j x) for XB (swapped for BX): B' gets -Im(ys') at (f,f) and (t,t) and
        +Im(ys') at (f,t) and (t,f); B'' gets -(Im(ys'') + Im(h)/2) at (f,f) and (t,t) and
        +Im(ys'') off the diagonal.  Canonical CSC, duplicates summed."""
        on = self.line_status
        f, t = self.line_from[on], self.line_to[on]
        r, x, h = self.line_r[on], self.line_x[on], self.line_h[on]
        ys_x = 1.0 / (1j * x)
        ys_rx = 1.0 / (r + 1j * x)
        ys_p, ys_pp = (ys_x, ys_rx) if int(method) == 0 else (ys_rx, ys_x)
        bp, bpp = np.imag(ys_p), np.imag(ys_pp)
        hh = np.imag(0.5 * h)
        rows = np.concatenate([f, t, f, t])
        cols = np.concatenate([f, t, t, f])
        out = []
        for vals in (np.concatenate([-bp, -bp, bp, bp]),
                     np.concatenate([-(bpp + hh), -(bpp + hh), bpp, bpp])):
            B = sparse.csc_matrix((vals, (rows, cols)), shape=(self.n_bus, self.n_bus), dtype=np.float64)
            B.sum_duplicates()
            B.sort_indices()
            out.append(B)
        return out[0], out[1]

    def debug_get_Bp_python(self, method=0):
        """Grid-level B' (the reference binds GridModel.debug_get_Bp_python(FDPFMethod))."""
        return self.get_Bp_Bpp(method)[0]

    def debug_get_Bpp_python(self, method=0):
        """Grid-level B''."""
        return self.get_Bp_Bpp(method)[1]

    def dc_branch_coeffs(self, branch_ids):
        """DC Ybus coefficients of the given branches, in the reference's order."""
        out = []
        for br in branch_ids:
            if not self.line_status[br]:
                continue
            b1, b2 = int(self.line_from[br]), int(self.line_to[br])
            yd = 1.0 / (self.line_x[br] + 0j)
            out.extend([Coeff(b1, b1, yd), Coeff(b2, b2, yd), Coeff(b1, b2, -yd), Coeff(b2, b1, -yd)])
        return out

    def _sbus_from(self, gen_p, sgen_p, load_p, load_q):
        S = np.zeros(self.n_bus, dtype=np.complex128)
        np.add.at(S, self.gen_bus, gen_p)
        if self.sgen_bus.size:
            np.add.at(S, self.sgen_bus, sgen_p)
        np.add.at(S, self.load_bus, -(load_p + 1j * load_q))
        if abs(self.sn_mva - 1.0) > 1e-7:
            S = S / self.sn_mva
        return S

    def get_Sbus(self):
        return self._sbus_from(self.gen_p_mw, self.sgen_p_mw, self.load_p_mw, self.load_q_mvar)

    def get_slack_ids(self):
        sl = []
        for g in range(self.gen_bus.size):
            if self.gen_slack_weight[g] > 0 and self.gen_bus[g] not in sl:
                sl.append(int(self.gen_bus[g]))
        return np.asarray(sl, dtype=np.int64)

    def get_slack_weights(self):
        w = np.zeros(self.n_bus)
        np.add.at(w, self.gen_bus, self.gen_slack_weight)
        tot = w.sum()
        if tot > 0:
            w = w / tot
        return w

    def get_pv(self):
        slack = set(self.get_slack_ids().tolist())
        pv, seen = [], set()
        for b in self.gen_bus.tolist():
            if b in slack or b in seen:
                continue
            seen.add(b)
            pv.append(int(b))
        return np.asarray(pv, dtype=np.int64)

    def get_pq(self):
        slack = set(self.get_slack_ids().tolist())
        pv = set(self.get_pv().tolist())
        return np.asarray([b for b in range(self.n_bus) if b not in slack and b not in pv], dtype=np.int64)

    def flat_start(self):
        """|V| at the generator set-point (init_vm_pu elsewhere), angle 0."""
        V = np.full(self.n_bus, self.init_vm_pu, dtype=np.complex128)
        V[self.gen_bus] = self.gen_vm_pu
        return V

    def sbuses_from_injections(self, gen_p, sgen_p, load_p, load_q):
        """Per-step Sbus matrix (TimeSeries.hpp:79-151 restated): ``(nb_steps, n_bus)``."""
        gen_p = np.atleast_2d(np.asarray(gen_p, dtype=np.float64))
        nb = gen_p.shape[0]
        load_p = np.atleast_2d(np.asarray(load_p, dtype=np.float64))
        load_q = np.atleast_2d(np.asarray(load_q, dtype=np.float64))
        S = np.zeros((nb, self.n_bus), dtype=np.complex128)
        for g in range(self.gen_bus.size):
            S[:, self.gen_bus[g]] += gen_p[:, g]
        if self.sgen_bus.size and sgen_p is not None and np.size(sgen_p):
            sgen_p = np.atleast_2d(np.asarray(sgen_p, dtype=np.float64))
            for g in range(self.sgen_bus.size):
                S[:, self.sgen_bus[g]] += sgen_p[:, g]
        for ld in range(self.load_bus.size):
            S[:, self.load_bus[ld]] -= load_p[:, ld] + 1j * load_q[:, ld]
        if abs(self.sn_mva - 1.0) > 1e-7:
            S /= self.sn_mva
        return S

    # ------------------------------------------------------------------ power flow
    def ac_pf(self, Vinit, max_iter=10, tol=1e-8, solver_type=None):
        """One AC power flow (GridModel::ac_pf, GridModel.cpp:301-349) on the GPU engine."""
        from .solver import GPUNRSolverSingleSlack, GPUNRSolver, SolverType

        if solver_type is None or solver_type == SolverType.GPUNRSingleSlack:
            cls = GPUNRSolverSingleSlack
        elif solver_type == SolverType.GPUNR:
            cls = GPUNRSolver
        else:
            raise RuntimeError("GridModel.ac_pf: unsupported solver type {}".format(solver_type))
        if self._solver is None or not isinstance(self._solver, cls):
            self._solver = cls()
        ok = self._solver.compute_pf(self.get_Ybus(), np.asarray(Vinit, dtype=np.complex128), self.get_Sbus(),
                                     self.get_slack_ids(), self.get_slack_weights(), self.get_pv(), self.get_pq(),
                                     max_iter, tol / self.sn_mva)
        if not ok:
            return np.zeros(0, dtype=np.complex128)
        return self._solver.get_V()
