"""Branch flows on the GPU against the oracle's restatement of the reference
(BaseBatchSolverSynch.hpp:87-192 flows, ContingencyAnalysis.cpp:237-250 clean_flows)."""
import numpy as np
import pytest

from conftest import grid_problem
from oracle.flows import branch_flows

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # relative, per value (the kernel and numpy order the complex products alike)


def _same(a, b):
    fa, fb = np.isfinite(a), np.isfinite(b)
    assert np.array_equal(fa, fb)
    assert np.all(np.abs(a[fa] - b[fb]) <= RTOL * np.maximum(1.0, np.abs(b[fb])))


def _oracle(bs, V, removed=None):
    return branch_flows(V, bs.from_, bs.to, bs.yff, bs.yft, bs.vn_kv_from, bs.status, bs.sn_mva, removed)


def test_host_entry_point_matches_oracle():
    from lightsim2grid_b200.flows import BranchSet, flows_host

    c = grid_problem("grid118")
    g = c["grid"]
    g.line_status[5] = False  # one branch out of service: 0 everywhere
    try:
        bs = BranchSet(g)
    finally:
        g.line_status[5] = True
    rng = np.random.default_rng(0)
    V = (1.0 + 0.05 * rng.standard_normal((20, g.n_bus))) * np.exp(1j * 0.1 * rng.standard_normal((20, g.n_bus)))
    V[3] = 0.0  # a failed case: NaN amps, 0 MW
    removed = [[int(rng.integers(bs.nbr))] for _ in range(20)]
    a, p = flows_host(bs, V, removed=removed)
    ao, po = _oracle(bs, V, removed)
    _same(a, ao)
    _same(p, po)
    assert np.all(a[:, 5] == 0) and np.all(p[:, 5] == 0)
    assert np.all(np.isnan(np.delete(a[3], [5, removed[3][0]]))) and np.all(p[3] == 0)


def test_contingency_analysis_flows_match_oracle():
    from lightsim2grid_b200 import ContingencyAnalysisCPP, SolverType
    from lightsim2grid_b200.flows import BranchSet

    c = grid_problem("grid118")
    g = c["grid"]
    ca = ContingencyAnalysisCPP(g)
    ca.change_solver(SolverType.GPUNRSingleSlack)
    ca.add_all_n1()
    ca.compute(c["V0"], 10, 1e-8)
    A = ca.compute_flows()
    P = ca.compute_power_flows()
    removed = [list(x) for x in ca.my_defaults()]
    ao, po = _oracle(BranchSet(g), ca.get_voltages(), removed)
    _same(A, ao)
    _same(P, po)


def test_device_entry_point_with_case_map():
    """Rows in case order from compact device results: islanded cases (map -1) and failed
    instances (errs != 0) read as zero voltages."""
    import torch

    from lightsim2grid_b200.flows import BranchSet, flows_device, outage_lists

    c = grid_problem("grid118")
    g = c["grid"]
    bs = BranchSet(g)
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(1)
    k, rows = 12, 16
    Vc = (1.0 + 0.05 * rng.standard_normal((k, g.n_bus))) * np.exp(1j * 0.1 * rng.standard_normal((k, g.n_bus)))
    errs = np.zeros(k, np.int32)
    errs[4] = 2  # a failed instance
    cmap = np.array([0, 1, -1, 2, 3, 4, 5, -1, 6, 7, 8, 9, 10, 11, -1, 0], np.int32)
    removed = [[int(x)] for x in rng.integers(bs.nbr, size=rows)]
    ptr, ids = outage_lists(removed)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    dV, dE, dM, dP, dI = t(Vc.view(np.float64)), t(errs), t(cmap), t(ptr), t(ids)
    A = torch.full((rows * bs.nbr,), -1.0, dtype=torch.float64, device=dev)
    P = torch.full((rows * bs.nbr,), -1.0, dtype=torch.float64, device=dev)
    bst, keep = bs.device(dev)
    for _ in range(2):
        flows_device(bst, bs.n, dV.data_ptr(), rows, torch.cuda.current_stream().cuda_stream,
                     map_ptr=dM.data_ptr(), errs_ptr=dE.data_ptr(), out_ptr=dP.data_ptr(), out_ids=dI.data_ptr(),
                     amps_ptr=A.data_ptr(), p_ptr=P.data_ptr())
    torch.cuda.synchronize()
    Vrows = np.zeros((rows, g.n_bus), np.complex128)
    for r, i in enumerate(cmap):
        if i >= 0 and errs[i] == 0:
            Vrows[r] = Vc[i]
    ao, po = _oracle(bs, Vrows, removed)
    _same(A.cpu().numpy().reshape(rows, bs.nbr), ao)
    _same(P.cpu().numpy().reshape(rows, bs.nbr), po)
