"""Fast decoupled power flow on the GPU against the CPU restatement (oracle/fdpf.py) of
BaseFDPFAlgo::compute_pf (src/powerflow_algorithm/BaseFDPFAlgo.tpp:11-173).

Both factorise B'_ and B''_ once and iterate in FP64; they differ only in rounding (orderings,
pivots, operation order), so the iteration counts and error codes are equal and the voltages
agree to TOL_V.  N-1 and time-series batches keep the base-case B' / B'' for every case and step
(the reference's batch computers do the same: the solver is told nothing changed after the base
power flow) and change only Ybus (outage) or Sbus (step).
"""
import numpy as np
import pytest

from conftest import grid_problem
from oracle.fdpf import fdpf

pytestmark = pytest.mark.gpu

TOL_V = 1e-9


def _plan(c, Bp, Bpp, **kw):
    from lightsim2grid_b200 import Plan

    return Plan(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], fdpf=(Bp, Bpp), **kw)


@pytest.mark.parametrize("name", ["grid14", "grid118", "grid1354", "grid2848"])
@pytest.mark.parametrize("method", [0, 1])
def test_single_pf_matches_oracle(name, method):
    c = grid_problem(name)
    g = c["grid"]
    Bp, Bpp = g.get_Bp_Bpp(method)
    Vo, conv_o, it_o, err_o = fdpf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], Bp, Bpp,
                                   40, 1e-8)
    plan = _plan(c, Bp, Bpp)
    V, conv, it, err = plan.solve(c["V0"], c["Sbus"], 40, 1e-8)
    assert (conv, it, err) == (conv_o, it_o, err_o), name
    assert np.abs(V - Vo).max() <= TOL_V
    info = plan.info()
    assert info["precision"] == 0 and info["nnz_lu"] > 0


def test_factor_placements_agree():
    """Factors in shared memory (packed operations v[x] -= l * (v[z] / d)) or read from global
    memory (v[x] -= (l * v[z]) / d): the same iterations, voltages equal up to rounding."""
    c = grid_problem("grid118")
    Bp, Bpp = c["grid"].get_Bp_Bpp(0)
    p1, p2 = _plan(c, Bp, Bpp, lu_placement=1), _plan(c, Bp, Bpp, lu_placement=2)
    assert p1.info()["lu_in_shared"] == 1 and p2.info()["lu_in_shared"] == 0
    ref = p1.solve(c["V0"], c["Sbus"], 40, 1e-8)
    got = p2.solve(c["V0"], c["Sbus"], 40, 1e-8)
    assert ref[1:] == got[1:]
    assert np.abs(ref[0] - got[0]).max() <= TOL_V


def test_distributed_slack_and_iteration_limit():
    """Two slacks (the second joins pvpq with its weight in the mismatch), and a run cut by
    max_iter (TooManyIterations at the same count)."""
    c = dict(grid_problem("grid118"))
    g = c["grid"]
    pv = np.asarray(c["pv"])
    ref = np.r_[np.asarray(c["ref"])[:1], pv[:1]]
    w = np.zeros(g.n_bus)
    w[ref] = [0.6, 0.4]
    c.update(ref=ref, weights=w, pv=pv[1:])
    Bp, Bpp = g.get_Bp_Bpp(1)
    plan = _plan(c, Bp, Bpp)
    for max_iter in (40, 3):
        Vo, conv_o, it_o, err_o = fdpf(c["Ybus"], c["V0"], c["Sbus"], ref, w, c["pv"], c["pq"], Bp, Bpp, max_iter,
                                       1e-8)
        V, conv, it, err = plan.solve(c["V0"], c["Sbus"], max_iter, 1e-8)
        assert (conv, it, err) == (conv_o, it_o, err_o), max_iter
        assert np.abs(V - Vo).max() <= TOL_V


def test_n1_batch_keeps_base_factors():
    from scipy import sparse

    c = grid_problem("grid118")
    g = c["grid"]
    Bp, Bpp = g.get_Bp_Bpp(0)
    plan = _plan(c, Bp, Bpp)
    cases = list(range(0, g.nb_powerline(), 3))
    coeffs = [g.branch_coeffs([b]) for b in cases]
    V, conv, iters, errs = plan.batch_n1(coeffs, c["V0"], c["Sbus"], 40, 1e-8)
    n = g.n_bus
    for k, lst in enumerate(coeffs):
        if errs[k] == 1:  # islanded: skipped like ContingencyAnalysis
            assert np.all(V[k] == 0)
            continue
        r = [e[0] for e in lst]
        cc = [e[1] for e in lst]
        y = [e[2] for e in lst]
        Yk = sparse.csc_matrix(c["Ybus"] - sparse.csc_matrix((y, (r, cc)), shape=(n, n)))
        Vo, conv_o, it_o, err_o = fdpf(Yk, c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], Bp, Bpp, 40,
                                       1e-8)
        assert (bool(conv[k]), int(iters[k]), int(errs[k])) == (conv_o, it_o, err_o), cases[k]
        if conv_o:
            assert np.abs(V[k] - Vo).max() <= TOL_V
        else:
            assert np.all(V[k] == 0)


def test_time_series_chain_matches_oracle():
    from lightsim2grid_b200 import synthetic

    c = grid_problem("grid118")
    g = c["grid"]
    Bp, Bpp = g.get_Bp_Bpp(1)
    gen_p, sgen_p, load_p, load_q = synthetic.time_series_injections(g, 24, seed=5)
    Sb = g.sbuses_from_injections(gen_p, sgen_p, load_p, load_q)
    plan = _plan(c, Bp, Bpp)
    st, V, conv, iters, errs = plan.batch_ts(Sb, c["V0"], 1, 40, 1e-8)
    Vprev = np.asarray(c["V0"], np.complex128)
    for k in range(Sb.shape[0]):
        Vo, conv_o, it_o, err_o = fdpf(c["Ybus"], Vprev, Sb[k], c["ref"], c["weights"], c["pv"], c["pq"], Bp, Bpp, 40,
                                       1e-8)
        assert (bool(conv[k]), int(iters[k])) == (conv_o, it_o), k
        assert np.abs(V[k] - Vo).max() <= TOL_V
        Vprev = Vo


def test_solver_class_and_computer():
    from lightsim2grid_b200 import (ContingencyAnalysisCPP, GPUFDPFSolverXB, GPUFDPFSolverBX, SolverType,
                                    SOLVER_CLASSES)

    c = grid_problem("grid118")
    g = c["grid"]
    for st, cls, meth in ((SolverType.GPUFDPF_XB, GPUFDPFSolverXB, 0), (SolverType.GPUFDPF_BX, GPUFDPFSolverBX, 1)):
        assert SOLVER_CLASSES[st] is cls
        s = cls()
        s.set_gridmodel(g)
        ok = s.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 40, 1e-8)
        Bp, Bpp = g.get_Bp_Bpp(meth)
        Vo, conv_o, it_o, _ = fdpf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], Bp, Bpp,
                                   40, 1e-8)
        assert ok == conv_o and s.get_nb_iter() == it_o
        assert np.abs(s.get_V() - Vo).max() <= TOL_V
        pvpq = np.r_[np.asarray(c["ref"])[1:], c["pv"], c["pq"]].astype(np.int64)
        assert abs(s.debug_get_Bp_python() - Bp[pvpq][:, pvpq]).max() == 0
        with pytest.raises(RuntimeError):
            s.get_J()
    # ContingencyAnalysisCPP with the fast decoupled solver: start = V0 with the generators'
    # set points (BaseBatchSolverSynch::_finish_preprocessing), base B' / B'' for every case
    from scipy import sparse

    ca = ContingencyAnalysisCPP(g)
    ca.change_solver(SolverType.GPUFDPF_XB)
    branches = list(range(12))
    ca.add_multiple_n1(branches)
    ca.compute(c["V0"], 100, 1e-8)
    V = ca.get_voltages()
    errs = ca.get_errors()
    V0 = np.asarray(c["V0"], np.complex128).copy()
    V0[g.gen_bus] = np.abs(g.gen_vm_pu) * np.exp(1j * np.angle(V0[g.gen_bus]))
    Bp, Bpp = g.get_Bp_Bpp(0)
    n = g.n_bus
    for k, b in enumerate(branches):
        if errs[k] == 1:
            continue
        lst = g.branch_coeffs([b])
        Yk = sparse.csc_matrix(c["Ybus"] - sparse.csc_matrix(([e[2] for e in lst], ([e[0] for e in lst],
                                                                                   [e[1] for e in lst])), shape=(n, n)))
        Vo, conv_o, it_o, err_o = fdpf(Yk, V0, c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], Bp, Bpp, 100,
                                       1e-8 / g.sn_mva)
        assert int(errs[k]) == err_o, b
        if conv_o:
            assert np.abs(V[k] - Vo).max() <= TOL_V
