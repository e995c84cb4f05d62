"""DC power flow restated on the CPU with scipy (oracle for the GPU DC plans).

TEST INFRASTRUCTURE ONLY: imported by tests/ (and nothing in the product package).

Follows BaseDCAlgo::compute_pf (src/powerflow_algorithm/BaseDCAlgo.tpp:5-175):
* the slacks after the first count as PV (retrieve_pv_with_slack, BaseAlgo.hpp:201-216); the
  slack buses are those neither PV nor PQ (extract_slack_bus_id, BaseAlgo.cpp:143-181);
* B = Re(Ybus) without the slack rows and columns, RHS = Re(Sbus) at the other buses
  (remove_slack_buses :208-232, :86-93);
* solve; a non-finite solution or one with |theta| >= 1e6 fails (SolverSolve, :115-123);
* Va = theta (0 at the slack) + arg(V[slack]); Vm = |V|; V = Vm e^{j Va} (:124-140).
"""
import numpy as np
from scipy import sparse
from scipy.sparse.linalg import splu


def dc_pf(Ybus, V, Sbus, slack_ids, pv, pq):
    """Returns (V, ok)."""
    Y = sparse.csc_matrix(Ybus)
    n = Y.shape[0]
    V = np.asarray(V, dtype=np.complex128)
    tagged = np.zeros(n, bool)
    tagged[np.asarray(slack_ids)[1:]] = True
    tagged[np.asarray(pv, dtype=np.int64)] = True
    tagged[np.asarray(pq, dtype=np.int64)] = True
    ids = np.flatnonzero(tagged)
    slack = np.flatnonzero(~tagged)
    B = sparse.csc_matrix(Y.real)[ids][:, ids]
    P = np.asarray(Sbus).real[ids]
    try:
        theta = splu(sparse.csc_matrix(B)).solve(P)
    except RuntimeError:
        return np.zeros(n, np.complex128), False
    if not np.all(np.isfinite(theta)) or np.abs(theta).max() >= 1e6:
        return np.zeros(n, np.complex128), False
    Va = np.zeros(n)
    Va[ids] = theta
    Va += np.angle(V[slack[0]])
    return np.abs(V) * np.exp(1j * Va), True
