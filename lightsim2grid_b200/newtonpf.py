"""pandapower-compatible ``newtonpf`` on the GPU engine.

Mirrors lightsim2grid/pandapower_compat/newtonpf/_newtonpf.py:30-351: ``newtonpf_new``
(with ``ref``) and ``newtonpf_old`` (without), same return tuple
``(V, converged, iterations, J, Vm_it, Va_it)``.
"""
import numpy as np

from .solver import GPUNRSolver, GPUNRSolverSingleSlack, GPUNRMixedSolver, GPUNRMixedSolverSingleSlack


def _isolate_slack_ids(Sbus, pv, pq):
    """_newtonpf.py:30-37: slack = every bus neither PV nor PQ, equal weights."""
    ref = np.array(sorted(set(np.arange(Sbus.shape[0])) - set(np.asarray(pv).tolist()) -
                          set(np.asarray(pq).tolist())), dtype=np.int64)
    slack_weights = np.zeros(Sbus.shape[0])
    slack_weights[ref] = 1.0 / ref.shape[0]
    return ref, slack_weights


def _get_valid_solver(options):
    """_newtonpf.py:40-57, with the GPU solvers; ``options["gpu_mixed_precision"]`` picks FP32 LU."""
    mixed = bool(options.get("gpu_mixed_precision", False))
    if options.get("distributed_slack", False):
        return GPUNRMixedSolver() if mixed else GPUNRSolver()
    return GPUNRMixedSolverSingleSlack() if mixed else GPUNRSolverSingleSlack()


def _run(solver, Ybus, Sbus, V0, ref, slack_weights, pv, pq, options):
    max_iteration = options["max_iteration"]
    tolerance_pu = options["tolerance_mva"]
    solver.solve(Ybus, V0, Sbus, ref, slack_weights, pv, pq, max_iteration, tolerance_pu)
    Va = solver.get_Va()
    Vm = solver.get_Vm()
    V = Vm * np.exp(1j * Va)
    J = solver.get_J()
    return V, solver.converged(), solver.get_nb_iter(), J, None, None


def newtonpf_new(Ybus, Sbus, V0, ref, pv, pq, ppci, options):
    """_newtonpf.py:234-351 (pandapower > 2.7 signature)."""
    slack_weights = None
    if isinstance(ppci, dict) and "bus" in ppci:
        try:
            from pandapower.pypower.idx_bus import SL_FAC  # noqa: F401  (optional dependency)
            slack_weights = np.asarray(ppci["bus"][:, SL_FAC], dtype=np.float64)
        except Exception:
            slack_weights = None
    if slack_weights is None:
        ref, slack_weights = _isolate_slack_ids(np.asarray(Sbus), pv, pq) if ref is None else (
            np.asarray(ref), _weights_for(ref, np.asarray(Sbus).shape[0]))
    solver = _get_valid_solver(options)
    return _run(solver, Ybus, Sbus, V0, ref, slack_weights, pv, pq, options)


def newtonpf_old(Ybus, Sbus, V0, pv, pq, ppci, options):
    """_newtonpf.py:122-231 (pandapower <= 2.7 signature)."""
    ref, slack_weights = _isolate_slack_ids(np.asarray(Sbus), pv, pq)
    solver = _get_valid_solver(options)
    return _run(solver, Ybus, Sbus, V0, ref, slack_weights, pv, pq, options)


def _weights_for(ref, n):
    w = np.zeros(n)
    ref = np.atleast_1d(np.asarray(ref))
    w[ref] = 1.0 / max(ref.size, 1)
    return w


def newtonpf(*args, **kwargs):
    """Dispatches between the two signatures by argument count (_newtonpf.py:60-120)."""
    nargs = len(args) + len(kwargs)
    if nargs == 8 or "ref" in kwargs:
        return newtonpf_new(*args, **kwargs)
    return newtonpf_old(*args, **kwargs)
