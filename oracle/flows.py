"""Branch flows of batch results, restated on the CPU with numpy (oracle for the GPU kernel).

TEST INFRASTRUCTURE ONLY: imported by tests/ (and nothing in the product package).

Follows, element by element:
* ``BaseBatchSolverSynch::compute_amps_flows`` (src/batch_algorithm/BaseBatchSolverSynch.hpp:87-139),
  AC branch: ``I_ft = conj(y_ff E_f + y_ft E_t)``, ``S_ft = E_f I_ft``,
  ``amps = |S_ft| sn_mva / (sqrt(3) |E_f| vn_kv(from))``;
* ``compute_active_power_flows`` (:140-192): ``p = Re(S_ft) sn_mva``;
* both start from zero matrices and skip out-of-service branches (:63-64, :108);
* ``ContingencyAnalysis::clean_flows`` (src/batch_algorithm/ContingencyAnalysis.cpp:237-250):
  each case's removed branches are set to 0 where the value is finite.
"""
import numpy as np


def branch_flows(V, from_, to, y_ff, y_ft, vn_kv_from, status, sn_mva, removed=None):
    """Returns (amps[rows, nbr], p_mw[rows, nbr]) for result rows ``V[rows, n]``."""
    V = np.asarray(V, dtype=np.complex128)
    rows, nbr = V.shape[0], len(from_)
    amps = np.zeros((rows, nbr))
    pmw = np.zeros((rows, nbr))
    on = np.asarray(status, dtype=bool)
    f, t = np.asarray(from_)[on], np.asarray(to)[on]
    Ef, Et = V[:, f], V[:, t]
    I_ft = np.conj(np.asarray(y_ff)[on][None, :] * Ef + np.asarray(y_ft)[on][None, :] * Et)
    S_ft = Ef * I_ft
    with np.errstate(divide="ignore", invalid="ignore"):
        amps[:, on] = np.abs(S_ft) * sn_mva / (np.sqrt(3.0) * (np.abs(Ef) * np.asarray(vn_kv_from)[on][None, :]))
    pmw[:, on] = S_ft.real * sn_mva
    if removed is not None:
        for r, lst in enumerate(removed):
            for b in lst:
                if np.isfinite(amps[r, b]):
                    amps[r, b] = 0.0
                if np.isfinite(pmw[r, b]):
                    pmw[r, b] = 0.0
    return amps, pmw
