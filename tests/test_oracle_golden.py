"""The oracle against the reference's golden NR vectors (lightsim2grid/tests/test_KLUSolver.py:76-127).

Same tolerances as the reference test: J blocks and Va / Vm by L1 sum <= 1e-4, the same
iteration count (the golden file name J_<k>, V_<k>), and the same five cases.
"""
import numpy as np
import pytest
from scipy import sparse
import scipy.sparse.linalg as spla

from oracle.oracle import OracleNR

TOL_TEST = 1e-4


def test_five_golden_cases(golden):
    assert len(golden) == 5


@pytest.mark.parametrize("distributed", [True, False])
def test_oracle_matches_golden(golden, distributed):
    for c in golden:
        s = OracleNR(distributed)
        ok = s.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
        assert ok, c["name"]
        assert s.get_nb_iter() == c["n_iter"], c["name"]
        J = s.get_J().toarray()
        if distributed:
            J = J[1:, 1:]
        Jg = c["J_ref"].toarray()
        npvpq = len(c["pv"]) + len(c["pq"])
        d = np.abs(J - Jg)
        assert d[:npvpq, :npvpq].sum() <= TOL_TEST
        assert d[npvpq:, :npvpq].sum() <= TOL_TEST
        assert d[:npvpq, npvpq:].sum() <= TOL_TEST
        assert d[npvpq:, npvpq:].sum() <= TOL_TEST
        assert np.abs(s.get_Va() - np.angle(c["V_ref"])).sum() <= TOL_TEST
        assert np.abs(s.get_Vm() - np.abs(c["V_ref"])).sum() <= TOL_TEST


def test_oracle_lu_against_scipy(golden):
    """The oracle's Newton steps agree with a scipy (SuperLU) Newton iteration."""
    c = [g for g in golden if g["name"] == "case300"][0]
    Y, S, V = c["Ybus"], c["Sbus"], c["V0"].copy()
    pv, pq = c["pv"], c["pq"]
    pvpq = np.r_[pv, pq]
    for _ in range(10):
        mis = V * np.conj(Y @ V) - S
        F = np.r_[mis[pv].real, mis[pq].real, mis[pq].imag]
        if np.abs(F).max() < 1e-8:
            break
        Ib = Y @ V
        diagV = sparse.diags(V)
        Vn = sparse.diags(V / np.abs(V))
        dVm = diagV @ np.conj(Y @ Vn) + sparse.diags(np.conj(Ib)) @ Vn
        dVa = 1j * diagV @ np.conj(sparse.diags(Ib) - Y @ diagV)
        dVm, dVa = sparse.csr_matrix(dVm), sparse.csr_matrix(dVa)
        J = sparse.bmat([[dVa[pvpq][:, pvpq].real, dVm[pvpq][:, pq].real],
                         [dVa[pq][:, pvpq].imag, dVm[pq][:, pq].imag]]).tocsc()
        dx = spla.spsolve(J, F)
        Va, Vm = np.angle(V), np.abs(V)
        Va[pv] -= dx[:len(pv)]
        Va[pq] -= dx[len(pv):len(pvpq)]
        Vm[pq] -= dx[len(pvpq):]
        V = Vm * np.exp(1j * Va)
    s = OracleNR(False)
    assert s.compute_pf(Y, c["V0"], S, c["ref"], c["weights"], pv, pq, 10, 1e-8)
    assert np.abs(s.get_V() - V).max() < 1e-10


def test_oracle_pinned_tightly_on_converged_golden_states(golden):
    """Beyond the reference test's L1 bar: on the fixtures that store a converged state (118, 300
    and 1888 buses; the 14- and 30-bus fixtures store the state after 3 iterations, 2e-3 pu of
    mismatch from convergence), the oracle's solution is the stored one to 1e-9 pu per bus, and its
    Jacobian is within 1e-6 per entry.  Measured: 1.9e-10, 1.7e-11 and 5.8e-10 pu."""
    for c in golden:
        if c["name"] not in ("case118", "case300", "case1888"):
            continue
        s = OracleNR(False)
        assert s.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
        V = s.get_V()
        assert np.abs(np.abs(V) - np.abs(c["V_ref"])).max() <= 1e-9, c["name"]
        assert np.abs(np.angle(V) - np.angle(c["V_ref"])).max() <= 1e-9, c["name"]
        assert np.abs(s.get_J().toarray() - c["J_ref"].toarray()).max() <= 1e-6, c["name"]
