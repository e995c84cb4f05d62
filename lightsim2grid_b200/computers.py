"""Batch computers: ContingencyAnalysisCPP and TimeSeriesCPP on the GPU engine.

Method sets follow the reference's bindings (src/main.cpp:1158-1251); semantics follow
src/batch_algorithm/ContingencyAnalysis.cpp, TimeSeries.cpp and BaseBatchSolverSynch.{hpp,cpp}:

* a base ("N") power flow runs first and fixes the sparsity pattern and the pivots
  (BaseBatchSolverSynch.hpp:277-321); if it diverges nothing else is computed;
* ContingencyAnalysis: every contingency removes its branches' Ybus coefficients (pattern
  kept), islanded cases are skipped, every case starts from the same Vinit
  (ContingencyAnalysis.cpp:166-233); tolerance ``tol / sn_mva``;
* TimeSeries: Sbus per step from the injections; step i starts from step i-1's solution
  and the series stops at the first divergence (TimeSeries.cpp:14-109).  The engine cuts
  the series into contiguous chunks solved in parallel (``nb_chunks``; 1 reproduces the
  reference's single chain).
"""
import time

import numpy as np

from .solver import SolverType, GPU_SOLVERS, FDPF_SOLVERS, Plan, solver_flags


class _BatchBase:
    def __init__(self, grid_model):
        self._grid = grid_model
        self.init_from_n_powerflow = False
        self._solver_type = SolverType.GPUNRSingleSlack
        self._plan_options = {}
        self.clear()

    # solver control (src/main.cpp:1168-1171)
    def change_solver(self, solver_type):
        solver_flags(solver_type)
        self._solver_type = SolverType(solver_type)
        self.clear()

    def available_solvers(self):
        return list(GPU_SOLVERS)

    def get_solver_type(self):
        return self._solver_type

    def set_plan_options(self, **kwargs):
        """Engine options (threads, lu_placement, fuse_forward, fp64_fallback, max_ctas_per_sm, refine)."""
        self._plan_options = dict(kwargs)
        self._plan = None

    def clear(self):
        self._plan = None
        self._voltages = np.zeros((0, 0), dtype=np.complex128)
        self._amps_flows = np.zeros((0, 0))
        self._active_power_flows = np.zeros((0, 0))
        self._nb_solved = 0
        self._timer_total = 0.0
        self._timer_solver = 0.0
        self._timer_pre_proc = 0.0
        self._timer_compute_A = 0.0
        self._timer_compute_P = 0.0
        self._conv = np.zeros(0, dtype=bool)
        self._iters = np.zeros(0, dtype=np.int32)
        self._errs = np.zeros(0, dtype=np.int32)

    # timers (src/main.cpp:1174-1178)
    def total_time(self):
        return self._timer_total

    def solver_time(self):
        return self._timer_solver

    def preprocessing_time(self):
        return self._timer_pre_proc

    def amps_computation_time(self):
        return self._timer_compute_A

    def nb_solved(self):
        return self._nb_solved

    # results
    def get_voltages(self):
        return self._voltages

    def get_flows(self):
        return self._amps_flows

    def get_power_flows(self):
        return self._active_power_flows

    def get_convergence(self):
        """Per-case convergence flags (engine extension)."""
        return self._conv

    def get_iterations(self):
        return self._iters

    def get_errors(self):
        return self._errs

    def get_plan(self):
        return self._plan

    # ------------------------------------------------------------------ shared machinery
    def _prepare(self, Vinit, max_iter, tol):
        """Base power flow (BaseBatchSolverSynch::_finish_preprocessing)."""
        g = self._grid
        Vinit = np.asarray(Vinit, dtype=np.complex128).ravel()
        if Vinit.size != g.total_bus():
            raise RuntimeError("Size of the Vinit should be the same as the total number of buses. Currently: "
                               "Vinit: {} and there are {} buses.".format(Vinit.size, g.total_bus()))
        Y = g.get_Ybus()
        S = g.get_Sbus()
        sl, w, pv, pq = g.get_slack_ids(), g.get_slack_weights(), g.get_pv(), g.get_pq()
        distributed, precision = solver_flags(self._solver_type)
        V0 = Vinit.copy()
        V0[g.gen_bus] = np.abs(g.gen_vm_pu) * np.exp(1j * np.angle(V0[g.gen_bus]))
        fdpf = None
        if self._solver_type in FDPF_SOLVERS:
            # fast decoupled: B' and B'' of the base grid, kept for every case and step
            fdpf = g.get_Bp_Bpp(FDPF_SOLVERS[self._solver_type])
        self._plan = Plan(Y, V0, S, sl, w, pv, pq, distributed=distributed, precision=precision, fdpf=fdpf,
                          **self._plan_options)
        Vn, conv, it, err = self._plan.solve(V0, S, max_iter, tol)
        Vstart = Vn if (self.init_from_n_powerflow and conv) else V0
        return Y, S, Vstart, conv

    # flows (BaseBatchSolverSynch.hpp:87-192): the GPU kernel of lightsim2grid_b200.flows on the
    # stored voltages (rows of failed or skipped cases are zero: NaN amps, 0 MW, as in the
    # reference); `removed`: per row, branches zeroed where finite (clean_flows)
    def _branch_flows(self, amps, removed=None):
        from .flows import BranchSet, flows_host

        a, p = flows_host(BranchSet(self._grid), self._voltages, removed=removed, amps=amps, power=not amps)
        return a if amps else p


class ContingencyAnalysisCPP(_BatchBase):
    """N-1 / N-k security analysis (src/batch_algorithm/ContingencyAnalysis.{hpp,cpp})."""

    def __init__(self, grid_model):
        self._li_defaults = []
        super().__init__(grid_model)

    # contingency list (ContingencyAnalysis.hpp:36-62); kept sorted and unique like the
    # reference's std::set<std::set<int>>
    def _norm(self):
        self._li_defaults = sorted(set(self._li_defaults))

    def add_all_n1(self):
        for br in range(self._grid.nb_powerline() + self._grid.nb_trafo()):
            self._li_defaults.append((br,))
        self._norm()

    def add_n1(self, branch_id):
        self._li_defaults.append((int(branch_id),))
        self._norm()

    def add_nk(self, branch_ids):
        self._li_defaults.append(tuple(sorted(set(int(b) for b in branch_ids))))
        self._norm()

    def add_multiple_n1(self, branch_ids):
        for b in branch_ids:
            self._li_defaults.append((int(b),))
        self._norm()

    def remove_n1(self, branch_id):
        key = (int(branch_id),)
        had = key in self._li_defaults
        self._li_defaults = [c for c in self._li_defaults if c != key]
        return had

    def remove_nk(self, branch_ids):
        key = tuple(sorted(set(int(b) for b in branch_ids)))
        had = key in self._li_defaults
        self._li_defaults = [c for c in self._li_defaults if c != key]
        return had

    def remove_multiple_n1(self, branch_ids):
        return sum(self.remove_n1(b) for b in branch_ids)

    def my_defaults(self):
        return [list(c) for c in self._li_defaults]

    my_defaults_vect = my_defaults

    def clear(self):
        super().clear()

    def reset(self):
        self._li_defaults = []
        self.clear()

    def clear_results_only(self):
        super().clear()

    def _coeffs(self):
        return [self._grid.branch_coeffs(list(c)) for c in self._li_defaults]

    def is_grid_connected_after_contingency(self):
        """1 / 0 per contingency (ContingencyAnalysis.cpp:134-146)."""
        g = self._grid
        from . import _native as nat

        S = g.get_Sbus()
        plan = Plan(g.get_Ybus(), g.flat_start(), S, g.get_slack_ids(), g.get_slack_weights(), g.get_pv(),
                    g.get_pq(), distributed=False, precision=0)
        coeffs = self._coeffs()
        cp = np.zeros(len(coeffs) + 1, dtype=np.int32)
        rows, cols, vals = [], [], []
        for c, lst in enumerate(coeffs):
            cp[c + 1] = cp[c] + len(lst)
            for (r, cc, y) in lst:
                rows.append(r)
                cols.append(cc)
                vals.append(y)
        rows = nat.as_i32(rows if rows else [0])
        cols = nat.as_i32(cols if cols else [0])
        vals = nat.as_c128(vals if vals else [0j]).ravel()
        solv = np.zeros(max(len(coeffs), 1), dtype=np.int32)
        optr = np.zeros(len(coeffs) + 1, dtype=np.int32)
        cap = max(int(cp[-1]), 1)
        opos = np.zeros(cap, dtype=np.int32)
        oval = np.zeros(cap, dtype=np.complex128)
        rc = plan._lib.pf_n1_prepare(plan.handle, len(coeffs), nat.ptr(cp, nat.i32p), nat.ptr(rows, nat.i32p),
                                     nat.ptr(cols, nat.i32p), nat.cptr(vals), nat.ptr(solv, nat.i32p),
                                     nat.ptr(optr, nat.i32p), nat.ptr(opos, nat.i32p), nat.cptr(oval), cap)
        if rc < 0:
            raise RuntimeError(nat.last_error(plan._lib))
        return solv[:len(coeffs)].astype(np.int32)

    def compute(self, Vinit, max_iter, tol):
        """ContingencyAnalysis::compute (ContingencyAnalysis.cpp:166-233)."""
        t0 = time.perf_counter()
        g = self._grid
        nb = len(self._li_defaults)
        self._voltages = np.zeros((nb, g.total_bus()), dtype=np.complex128)
        self._conv = np.zeros(nb, dtype=bool)
        self._iters = np.zeros(nb, dtype=np.int32)
        self._errs = np.full(nb, 8, dtype=np.int32)
        Y, S, Vstart, n_conv = self._prepare(Vinit, max_iter, tol)
        t1 = time.perf_counter()
        self._timer_pre_proc = t1 - t0
        if not n_conv:
            self._timer_total = time.perf_counter() - t0
            return
        Vout, conv, iters, errs = self._plan.batch_n1(self._coeffs(), Vstart, S, max_iter, tol / g.sn_mva)
        self._voltages = Vout
        self._conv, self._iters, self._errs = conv, iters, errs
        self._nb_solved = int(np.sum(errs != 1))
        self._timer_solver = float(self._plan.timers()[0])
        self._timer_total = time.perf_counter() - t0

    def compute_flows(self):
        """Amps per branch and case (ContingencyAnalysis.hpp:110-114): removed branches 0,
        failed or skipped cases NaN (their voltages are zero), ContingencyAnalysis.cpp:237-250."""
        t0 = time.perf_counter()
        self._amps_flows = self._branch_flows(True, removed=[list(c) for c in self._li_defaults])
        self._timer_compute_A = time.perf_counter() - t0
        return self._amps_flows

    def compute_power_flows(self):
        """Active power (MW) per branch and case (ContingencyAnalysis.hpp:116-120)."""
        t0 = time.perf_counter()
        self._active_power_flows = self._branch_flows(False, removed=[list(c) for c in self._li_defaults])
        self._timer_compute_P = time.perf_counter() - t0
        return self._active_power_flows

    def modif_Ybus_time(self):
        return self._timer_pre_proc


class TimeSeriesCPP(_BatchBase):
    """Time series of power flows (src/batch_algorithm/TimeSeries.{hpp,cpp})."""

    def __init__(self, grid_model):
        super().__init__(grid_model)
        self._status = 0
        self._Sbuses = np.zeros((0, 0), dtype=np.complex128)
        self.nb_chunks = 0

    def get_status(self):
        return self._status

    def get_sbuses(self):
        return self._Sbuses

    def compute_Sbuses(self, gen_p, sgen_p, load_p, load_q):
        self._Sbuses = self._grid.sbuses_from_injections(gen_p, sgen_p, load_p, load_q)
        return self._Sbuses

    def compute_Vs(self, gen_p, sgen_p, load_p, load_q, Vinit, max_iter, tol):
        """TimeSeries::compute_Vs (TimeSeries.cpp:14-109); returns the status (1 success)."""
        t0 = time.perf_counter()
        g = self._grid
        Sb = self.compute_Sbuses(gen_p, sgen_p, load_p, load_q)
        nsteps = Sb.shape[0]
        self._voltages = np.zeros((nsteps, g.total_bus()), dtype=np.complex128)
        self._status = 0
        Y, S, Vstart, n_conv = self._prepare(Vinit, max_iter, tol)
        self._timer_pre_proc = time.perf_counter() - t0
        if not n_conv:
            self._timer_total = time.perf_counter() - t0
            return -1
        status, Vout, conv, iters, errs = self._plan.batch_ts(Sb, Vstart, self.nb_chunks, max_iter,
                                                              tol / g.sn_mva)
        self._voltages = Vout
        self._conv, self._iters, self._errs = conv, iters, errs
        self._nb_solved = int(np.sum(errs != 8))
        self._status = status
        self._timer_solver = float(self._plan.timers()[0])
        self._timer_total = time.perf_counter() - t0
        return self._status

    def compute_flows(self):
        """Amps per branch and snapshot (TimeSeries.hpp:69-72)."""
        t0 = time.perf_counter()
        self._amps_flows = self._branch_flows(True)
        self._timer_compute_A = time.perf_counter() - t0
        return self._amps_flows

    def compute_power_flows(self):
        t0 = time.perf_counter()
        self._active_power_flows = self._branch_flows(False)
        self._timer_compute_P = time.perf_counter() - t0
        return self._active_power_flows

    def close(self):
        self.clear()


# the reference's Python names (lightsim2grid/contingencyAnalysis.py, timeSerie.py)
ContingencyAnalysis = ContingencyAnalysisCPP
SecurityAnalysis = ContingencyAnalysisCPP
TimeSerie = TimeSeriesCPP
