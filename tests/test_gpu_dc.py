"""DC power flow on the GPU against the oracle's restatement of BaseDCAlgo::compute_pf
(src/powerflow_algorithm/BaseDCAlgo.tpp:5-175), single solves and N-1 batches."""
import numpy as np
import pytest

from conftest import grid_problem
from oracle.dc import dc_pf

pytestmark = pytest.mark.gpu

TOL = 1e-10  # pu: two FP64 sparse LU solves with different orderings and pivots


@pytest.mark.parametrize("name", ["grid14", "grid118", "grid2848"])
def test_dc_solver_matches_oracle(name):
    from lightsim2grid_b200 import ErrorType, GPUDCSolver

    c = grid_problem(name)
    g = c["grid"]
    Yd = g.get_dcYbus()
    S, sl, w, pv, pq = g.get_Sbus(), g.get_slack_ids(), g.get_slack_weights(), g.get_pv(), g.get_pq()
    V0 = c["V0"]
    s = GPUDCSolver()
    assert s.compute_pf(Yd, V0, S, sl, w, pv, pq, 10, 1e-8)
    assert s.get_nb_iter() == 1 and s.get_error() == ErrorType.NoError
    Vo, ok = dc_pf(Yd, V0, S, sl, pv, pq)
    assert ok
    assert np.abs(s.get_V() - Vo).max() <= TOL
    # a second call on new injections reuses the plan
    S2 = S * 1.1
    assert s.compute_pf(Yd, V0, S2, sl, w, pv, pq, 10, 1e-8)
    assert np.abs(s.get_V() - dc_pf(Yd, V0, S2, sl, pv, pq)[0]).max() <= TOL


def test_dc_n1_batch_matches_oracle():
    from lightsim2grid_b200 import Plan

    c = grid_problem("grid118")
    g = c["grid"]
    Yd = g.get_dcYbus()
    S, sl, w, pv, pq = g.get_Sbus(), g.get_slack_ids(), g.get_slack_weights(), g.get_pv(), g.get_pq()
    plan = Plan(Yd, c["V0"], S, sl, w, pv, pq, dc=True)
    coeffs = [g.dc_branch_coeffs([b]) for b in range(g.nb_powerline())]
    V, conv, iters, errs = plan.batch_n1(coeffs, c["V0"], S, 10, 1e-8)
    n_ok = 0
    for k, lst in enumerate(coeffs):
        Yk = Yd.tolil(copy=True)
        for (r, cc, y) in lst:
            Yk[r, cc] -= y
        Yk = Yk.tocsc()
        if errs[k] == 1:  # islanded: skipped, as the reference's check_invertible does
            assert not conv[k] and np.all(V[k] == 0)
            continue
        Vo, ok = dc_pf(Yk, c["V0"], S, sl, pv, pq)
        assert ok and conv[k]
        assert np.abs(V[k] - Vo).max() <= TOL
        n_ok += 1
    assert n_ok > 100
