"""Batch semantics of the oracle, restating the reference's integration-test invariants on
synthetic grids (test_SecurityAnlysis_cpp.py:192-259, test_TimeSerie.py:287-300)."""
import numpy as np
from scipy import sparse

from conftest import grid_problem
from oracle.oracle import OracleNR, contingency_analysis, time_series
from lightsim2grid_b200 import synthetic


def test_contingency_equals_single_nr_on_modified_ybus():
    c = grid_problem("grid118")
    g = c["grid"]
    coeffs = [g.branch_coeffs([b]) for b in range(40)]
    ok, V, conv, iters, errs = contingency_analysis(c["Ybus"], c["Sbus"], c["V0"], c["ref"], c["weights"], c["pv"],
                                                    c["pq"], coeffs)
    assert ok == 1
    for k in range(40):
        Y = c["Ybus"].tolil()
        for (r, col, y) in coeffs[k]:
            Y[r, col] -= y
        Y = sparse.csc_matrix(Y)
        s = OracleNR(False)
        if errs[k] == 8:  # islanded: skipped, V row zero
            assert np.all(V[k] == 0)
            continue
        r1 = s.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
        assert r1
        s.compute_pf(Y, c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
        if conv[k]:
            assert np.abs(s.get_V() - V[k]).max() < 1e-9


def test_islanding_bridges_are_skipped():
    c = grid_problem("grid118")
    g = c["grid"]
    coeffs = [g.branch_coeffs([b]) for b in range(g.nb_powerline())]
    ok, V, conv, iters, errs = contingency_analysis(c["Ybus"], c["Sbus"], c["V0"], c["ref"], c["weights"], c["pv"],
                                                    c["pq"], coeffs)
    isl = errs == 8
    assert 0 < isl.sum() < len(coeffs)
    assert np.all(V[isl] == 0)
    # a leaf bus's only branch is a bridge
    deg = np.bincount(np.r_[g.line_from, g.line_to], minlength=g.n_bus)
    leaf_br = [b for b in range(g.nb_powerline()) if deg[g.line_from[b]] == 1 or deg[g.line_to[b]] == 1]
    assert all(isl[b] for b in leaf_br)


def test_time_series_step_equals_warm_started_nr():
    c = grid_problem("grid118")
    g = c["grid"]
    gen_p, sgen_p, load_p, load_q = synthetic.time_series_injections(g, 12, seed=5)
    Sb = g.sbuses_from_injections(gen_p, sgen_p, load_p, load_q)
    st, V, conv, iters, errs = time_series(c["Ybus"], c["Sbus"], Sb, c["V0"], c["ref"], c["weights"], c["pv"],
                                           c["pq"])
    assert st == 1 and conv.all()
    s = OracleNR(False)
    for k in range(1, 12):
        assert s.compute_pf(c["Ybus"], V[k - 1], Sb[k], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
        assert np.abs(s.get_V() - V[k]).max() < 1e-9
