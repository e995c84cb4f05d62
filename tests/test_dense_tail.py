"""Dense tail of high-fill plans.  On grids with long-range branches the LU fill gathers in a
dense trailing block; the plan factorises it as one dense matrix (pf_plan_info.tail_k) and the
phase programs keep only the sparse part.  CPU: the host emulation of the device schedule
(sparse programs + dense block) solves J x = b, and plans of the geometric grids have no tail.
GPU: N-1 batches of the chord grid through the dense tail against the oracle (the bars of the
other parity tests: FP64 flags and iterations equal, |dV| <= 1e-10 pu; mixed |dV| <= 1e-8 pu)."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

from conftest import grid_problem
from oracle.oracle import OracleNR, contingency_analysis
from test_host_plan import host_schedule_solve

TOL_FP64 = 1e-10
TOL_MIXED = 1e-8


def _solution_and_J(c):
    o = OracleNR(False)
    assert o.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
    V = o.get_V()
    # the Jacobian at the solution: one iteration from V towards other injections
    o2 = OracleNR(False)
    o2.compute_pf(c["Ybus"], V, c["Sbus"] * 1.01, c["ref"], c["weights"], c["pv"], c["pq"], 1, 1e-8)
    return V, o2.get_J().tocsc()


@pytest.mark.parametrize("name", ["grid2848c300"])
def test_host_schedule_with_dense_tail_solves_J(name):
    c = grid_problem(name)
    V, J = _solution_and_J(c)
    b = np.random.default_rng(1).standard_normal(J.shape[0])
    x, info = host_schedule_solve(c, V, b, False)
    assert info.tail_k >= 256
    # the block's columns left the programs: far fewer phases than elimination levels
    assert info.groups_refactor < info.levels_refactor and info.groups_backward < 64
    xr = spla.spsolve(J, b)
    assert np.abs(x - xr).max() <= 1e-10 * np.abs(xr).max()


@pytest.mark.parametrize("name", ["grid118", "grid2848", "grid2848c100"])
def test_small_or_sparse_tails_stay_in_the_programs(name):
    """Geometric grids have no dense trailing block; the 100-chord grid's (185 steps) is below the
    size from which the dense factorisation pays."""
    c = grid_problem(name)
    V, J = _solution_and_J(c)
    b = np.ones(J.shape[0])
    _, info = host_schedule_solve(c, V, b, False)
    assert info.tail_k == 0


def _vdiff(a, b):
    return max(np.abs(np.abs(a) - np.abs(b)).max(), np.abs(np.angle(a) - np.angle(b)).max())


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_dense_tail_n1_matches_oracle(precision):
    from lightsim2grid_b200 import Plan

    c = grid_problem("grid2848c300")
    o = OracleNR(False)
    assert o.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
    Vn = o.get_V()
    coeffs = [c["grid"].branch_coeffs([b]) for b in range(300)]
    ok, Vo, conv_o, it_o, err_o = contingency_analysis(c["Ybus"], c["Sbus"], Vn, c["ref"], c["weights"], c["pv"],
                                                       c["pq"], coeffs)
    plan = Plan(c["Ybus"], Vn, c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], precision=precision)
    inf = plan.info()
    assert inf["tail_k"] >= 256 and not inf["lu_in_shared"]
    V, conv, iters, errs = plan.batch_n1(coeffs, Vn, c["Sbus"], 10, 1e-8)
    assert np.array_equal(errs == 1, err_o == 8)
    assert np.array_equal(conv, conv_o)
    assert conv.sum() > 200
    if precision == 0:
        assert np.array_equal(iters[conv], it_o[conv_o])
    tol = TOL_FP64 if precision == 0 else TOL_MIXED
    for k in np.nonzero(conv)[0]:
        assert _vdiff(V[k], Vo[k]) <= tol, k


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_dense_tail_single_pf_matches_oracle(precision):
    from lightsim2grid_b200 import GPUNRSolverSingleSlack, GPUNRMixedSolverSingleSlack

    for name in ("grid2848c300", "grid2848c929"):
        c = grid_problem(name)
        o = OracleNR(False)
        ok_o = o.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
        s = (GPUNRSolverSingleSlack if precision == 0 else GPUNRMixedSolverSingleSlack)()
        ok = s.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
        assert ok == ok_o, name
        if precision == 0:
            assert s.get_nb_iter() == o.get_nb_iter(), name
        assert _vdiff(s.get_V(), o.get_V()) <= (TOL_FP64 if precision == 0 else TOL_MIXED), name
