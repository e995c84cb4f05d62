"""The fast-decoupled oracle (oracle/fdpf.py) on the CPU, and the host-side checks of the
FDPF plan that need no GPU.

Pins: the fixed point of the FDPF iteration is the power-flow solution, so on the reference's
golden NR cases (lightsim2grid/tests/case*.zip, via tests/golden) the oracle must land on the
golden V within the reference test's tolerance (test_KLUSolver.py:76-127: L1 sums <= 1e-4).  The
golden files hold Ybus only, not the element data the reference builds B' / B'' from, so these
cases use B' = the off-diagonal part of -Im(Ybus) with zero row sums and B'' = -Im(Ybus); case300
(phase shifters, negative reactances) diverges with that B' and is left out.
"""
import numpy as np
import pytest
from scipy import sparse

from conftest import golden_cases
from oracle.fdpf import fdpf, make_Bp_Bpp
from oracle.oracle import OracleNR

TOL_TEST = 1e-4


def _b_from_ybus(Y):
    Y = sparse.csc_matrix(Y)
    off = Y - sparse.diags(Y.diagonal())
    Bp = sparse.csc_matrix(-off.imag + sparse.diags(np.asarray(off.imag.sum(axis=1)).ravel()))
    return Bp, sparse.csc_matrix(-Y.imag)


@pytest.mark.parametrize("name", ["case14", "case30", "case118", "case1888"])
def test_oracle_fixed_point_is_golden_solution(name):
    c = [g for g in golden_cases() if g["name"] == name][0]
    Y = c["Ybus"]
    n = Y.shape[0]
    Bp, Bpp = _b_from_ybus(Y)
    w = np.zeros(n)
    w[c["ref"][0]] = 1.0
    pv = np.r_[c["ref"][1:], c["pv"]].astype(np.int64)
    V, conv, it, err = fdpf(Y, c["V0"], c["Sbus"], c["ref"][:1], w, pv, c["pq"], Bp, Bpp, 100, 1e-8)
    assert conv and err == 0
    assert np.abs(np.angle(V) - np.angle(c["V_ref"])).sum() <= TOL_TEST
    assert np.abs(np.abs(V) - np.abs(c["V_ref"])).sum() <= TOL_TEST


@pytest.mark.parametrize("name", ["grid14", "grid118", "grid300"])
@pytest.mark.parametrize("method", [0, 1])
def test_grid_b_matrices_match_oracle_restatement(name, method):
    """GridModel.get_Bp_Bpp (product side) against the oracle's element-by-element triplets."""
    from lightsim2grid_b200 import synthetic

    g, _ = synthetic.make_named_grid(name)
    Bp, Bpp = g.get_Bp_Bpp(method)
    Bp2, Bpp2 = make_Bp_Bpp(g.n_bus, g.line_from, g.line_to, g.line_r, g.line_x, g.line_h, g.line_status, method)
    for a, b in ((Bp, Bp2), (Bpp, Bpp2)):
        assert a.shape == b.shape
        assert abs(a - b).max() <= 1e-12 * max(1.0, abs(b).max())


@pytest.mark.parametrize("name", ["grid14", "grid118", "grid300"])
@pytest.mark.parametrize("method", [0, 1])
def test_oracle_agrees_with_newton(name, method):
    """Same fixed point as the NR oracle on the synthetic grids."""
    from lightsim2grid_b200 import synthetic

    g, _ = synthetic.make_named_grid(name)
    Bp, Bpp = g.get_Bp_Bpp(method)
    args = (g.get_Ybus(), g.flat_start(), g.get_Sbus(), g.get_slack_ids(), g.get_slack_weights(), g.get_pv(),
            g.get_pq())
    V, conv, it, err = fdpf(*args, Bp, Bpp, 60, 1e-10)
    assert conv and err == 0 and it > 1
    nr = OracleNR(False)
    assert nr.compute_pf(args[0], args[1], args[2], args[3], args[4], args[5], args[6], 20, 1e-10)
    assert np.abs(V - nr.get_V()).max() <= 1e-8


def test_oracle_error_codes():
    from lightsim2grid_b200 import synthetic

    g, _ = synthetic.make_named_grid("grid118")
    Bp, Bpp = g.get_Bp_Bpp(0)
    args = (g.get_Ybus(), g.flat_start(), g.get_Sbus(), g.get_slack_ids(), g.get_slack_weights(), g.get_pv(),
            g.get_pq())
    V, conv, it, err = fdpf(*args, Bp, Bpp, 3, 1e-8)
    assert not conv and it == 3 and err == 2  # TooManyIterations
    V, conv, it, err = fdpf(*args, Bp, Bpp, 0, 1e-8)
    assert not conv and it == 0 and err == 2


def test_singular_b_prime_fails_at_plan_creation():
    """A singular B' is SolverFactor when the plan is built (before any device work)."""
    from lightsim2grid_b200 import Plan, synthetic

    g, _ = synthetic.make_named_grid("grid14")
    Bp, Bpp = g.get_Bp_Bpp(0)
    Bp = sparse.csc_matrix(Bp.shape)  # all zero
    with pytest.raises(RuntimeError, match=r"status 5"):
        Plan(g.get_Ybus(), g.flat_start(), g.get_Sbus(), g.get_slack_ids(), g.get_slack_weights(), g.get_pv(),
             g.get_pq(), fdpf=(Bp, Bpp))
