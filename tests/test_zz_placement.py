"""The two placements of the packed phase programs (pf_options.placement 1, the default, and 2):
within a phase every written value has one thread and its operations keep their order, so an N-1
batch gives the same bits with either (voltages, iterations, error codes).  Mixed form on the
1354-bus grid and FP64 on the 118-bus grid, whose LUs sit in shared memory."""
import numpy as np
import pytest

from conftest import grid_problem
from oracle.oracle import OracleNR

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,precision,ncases", [("grid1354", 1, 400), ("grid118", 0, None)])
def test_placements_give_the_same_bits(name, precision, ncases):
    from lightsim2grid_b200 import Plan

    c = grid_problem(name)
    g = c["grid"]
    o = OracleNR(False)
    assert o.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
    Vn = o.get_V()
    nb = g.nb_powerline() if ncases is None else ncases
    coeffs = [g.branch_coeffs([b]) for b in range(nb)]
    out = []
    for placement in (1, 2):
        plan = Plan(c["Ybus"], Vn, c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], precision=precision,
                    placement=placement)
        assert plan.info()["lu_in_shared"] == 1
        out.append(plan.batch_n1(coeffs, Vn, c["Sbus"], 10, 1e-8))
    (V0, c0, i0, e0), (V1, c1, i1, e1) = out
    assert np.array_equal(e0, e1) and np.array_equal(c0, c1) and np.array_equal(i0, i1)
    assert np.array_equal(V0, V1)
