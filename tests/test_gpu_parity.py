"""GPU engine against the CPU oracle, through the C ABI (pf_* entry points).

Bars: FP64 form -- the same convergence flag and iteration count
as the oracle and |dVm|, |dVa| <= 1e-10 pu; mixed form (FP32 LU) -- the same convergence
flag and |dV| <= 1e-8 pu against the FP64 oracle.
"""
import numpy as np
import pytest

from conftest import grid_problem
from oracle.oracle import OracleNR, contingency_analysis, time_series

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10
TOL_MIXED = 1e-8


def _solvers():
    from lightsim2grid_b200 import (GPUNRSolverSingleSlack, GPUNRSolver, GPUNRMixedSolverSingleSlack,
                                    GPUNRMixedSolver)

    return {(False, 0): GPUNRSolverSingleSlack, (True, 0): GPUNRSolver, (False, 1): GPUNRMixedSolverSingleSlack,
            (True, 1): GPUNRMixedSolver}


def _vdiff(a, b):
    return max(np.abs(np.abs(a) - np.abs(b)).max(), np.abs(np.angle(a) - np.angle(b)).max())


def _problems(golden):
    return list(golden) + [grid_problem(n) for n in ("grid14", "grid118", "grid1354", "grid2848")]


@pytest.mark.parametrize("distributed", [False, True])
def test_single_pf_fp64_matches_oracle(golden, distributed):
    for c in _problems(golden):
        o = OracleNR(distributed)
        ok_o = o.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
        s = _solvers()[(distributed, 0)]()
        ok = s.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
        assert ok == ok_o, c["name"]
        assert s.get_nb_iter() == o.get_nb_iter(), c["name"]
        assert int(s.get_error()) == o.get_error(), c["name"]
        assert _vdiff(s.get_V(), o.get_V()) <= TOL_FP64, c["name"]
        Jg, Jo = s.get_J(), o.get_J()
        assert np.array_equal(Jg.indptr, Jo.indptr) and np.array_equal(Jg.indices, Jo.indices)
        assert np.abs(Jg.data - Jo.data).max() <= 1e-9 * max(1.0, np.abs(Jo.data).max()), c["name"]


@pytest.mark.parametrize("distributed", [False, True])
def test_single_pf_mixed_matches_oracle(golden, distributed):
    for c in _problems(golden):
        o = OracleNR(distributed)
        ok_o = o.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
        s = _solvers()[(distributed, 1)]()
        ok = s.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
        assert ok == ok_o, c["name"]
        assert _vdiff(s.get_V(), o.get_V()) <= TOL_MIXED, c["name"]


def test_golden_vectors_directly(golden):
    """The reference's own test (test_KLUSolver.py:94-114) against the GPU solver."""
    from lightsim2grid_b200 import GPUNRSolver

    for c in golden:
        s = GPUNRSolver()
        assert s.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
        assert s.get_nb_iter() == c["n_iter"]
        J = s.get_J().toarray()[1:, 1:]
        assert np.abs(J - c["J_ref"].toarray()).sum() <= 1e-4 * 4
        assert np.abs(s.get_Va() - np.angle(c["V_ref"])).sum() <= 1e-4
        assert np.abs(s.get_Vm() - np.abs(c["V_ref"])).sum() <= 1e-4


def test_newtonpf_signatures():
    from lightsim2grid_b200 import newtonpf

    c = grid_problem("grid118")
    opts = {"max_iteration": 10, "tolerance_mva": 1e-8}
    V, conv, it, J, _, _ = newtonpf(c["Ybus"], c["Sbus"], c["V0"], c["ref"], c["pv"], c["pq"], None, opts)
    V2, conv2, it2, J2, _, _ = newtonpf(c["Ybus"], c["Sbus"], c["V0"], c["pv"], c["pq"], None, opts)
    o = OracleNR(False)
    o.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
    assert conv and conv2 and it == it2 == o.get_nb_iter()
    assert _vdiff(V, o.get_V()) <= TOL_FP64 and _vdiff(V2, o.get_V()) <= TOL_FP64


def test_recycling_is_deterministic():
    """test_solver_control.py:55-120: repeated calls give the same V (1e-10); here bit-equal."""
    from lightsim2grid_b200 import GPUNRSolverSingleSlack

    c = grid_problem("grid1354")
    s = GPUNRSolverSingleSlack()
    args = (c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
    s.compute_pf(*args)
    V1 = s.get_V()
    s.compute_pf(*args)
    assert np.array_equal(V1, s.get_V())
    s.reset()
    s.compute_pf(*args)
    assert np.array_equal(V1, s.get_V())


def test_edge_cases_match_oracle():
    from lightsim2grid_b200 import GPUNRSolverSingleSlack

    c = grid_problem("grid118")
    base = (c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"])
    o = OracleNR(False)
    o.compute_pf(*base, 10, 1e-8)
    Vsol = o.get_V()
    cases = [
        ("max_iter 0", (c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 0, 1e-8)),
        ("already solved", (c["Ybus"], Vsol, c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)),
        ("too few iterations", (c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 2, 1e-8)),
        ("nan injection", (c["Ybus"], c["V0"], np.where(np.arange(len(c["Sbus"])) == 5, np.nan, c["Sbus"]),
                           c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)),
        ("overload", (c["Ybus"], c["V0"], 8.0 * c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)),
    ]
    for name, args in cases:
        o = OracleNR(False)
        ok_o = o.compute_pf(*args)
        s = GPUNRSolverSingleSlack()
        ok = s.compute_pf(*args)
        assert ok == ok_o, name
        assert int(s.get_error()) == o.get_error(), name
        assert s.get_nb_iter() == o.get_nb_iter(), name
        if ok:
            assert _vdiff(s.get_V(), o.get_V()) <= TOL_FP64, name


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("distributed", [False, True])
def test_angles_across_pi_match_oracle(precision, distributed):
    """Start voltages turned by 3.1 rad: the angles of many buses cross pi during the iterations,
    where the reference's re-derivation of Va = arg(V) wraps them (BaseNRSingleSlackAlgo.tpp:
    131-132); the engine must give the oracle's flags, iterations and voltages."""
    c = grid_problem("grid118")
    V0 = c["V0"] * np.exp(1j * 3.1)
    for scale in (1.0, 1.5):
        args = (c["Ybus"], V0, scale * c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
        o = OracleNR(distributed)
        ok_o = o.compute_pf(*args)
        s = _solvers()[(distributed, precision)]()
        ok = s.compute_pf(*args)
        assert ok == ok_o
        if precision == 0:
            assert s.get_nb_iter() == o.get_nb_iter()
        if ok:
            V = s.get_V()
            assert np.abs(np.angle(V)).max() > 3.0  # the solution sits across the wrap
            assert np.abs(V - o.get_V()).max() <= (TOL_FP64 if precision == 0 else TOL_MIXED)


def _n1(c, ncases=None):
    g = c["grid"]
    nb = g.nb_powerline() if ncases is None else min(ncases, g.nb_powerline())
    return [g.branch_coeffs([b]) for b in range(nb)]


@pytest.mark.parametrize("precision", [0, 1])
def test_n1_batch_matches_oracle(precision):
    from lightsim2grid_b200 import Plan

    for name, ncases in (("grid118", None), ("grid2848", 300)):
        c = grid_problem(name)
        o_n = OracleNR(False)
        assert o_n.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
        Vn = o_n.get_V()
        coeffs = _n1(c, ncases)
        ok, Vo, conv_o, it_o, err_o = contingency_analysis(c["Ybus"], c["Sbus"], Vn, c["ref"], c["weights"],
                                                           c["pv"], c["pq"], coeffs)
        plan = Plan(c["Ybus"], Vn, c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], precision=precision)
        V, conv, iters, errs = plan.batch_n1(coeffs, Vn, c["Sbus"], 10, 1e-8)
        islanded_o = err_o == 8
        assert np.array_equal(errs == 1, islanded_o), name
        assert np.array_equal(conv, conv_o), name
        if precision == 0:
            assert np.array_equal(iters[conv], it_o[conv_o]), name
        tol = TOL_FP64 if precision == 0 else TOL_MIXED
        for k in np.nonzero(conv)[0]:
            assert _vdiff(V[k], Vo[k]) <= tol, (name, k)
        assert np.all(V[~conv] == 0)


@pytest.mark.parametrize("precision", [0, 1])
def test_n1_batch_ordering_options_agree(precision):
    """The default elimination order (minimum degree, then its least-depth equivalent) and
    minimum degree alone: the same flags and iteration counts on the N-1 batch of the 1354-bus
    grid, and voltages within the precision's bar of each other."""
    from lightsim2grid_b200 import Plan

    c = grid_problem("grid1354")
    o_n = OracleNR(False)
    assert o_n.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
    Vn = o_n.get_V()
    coeffs = _n1(c, 400)
    out = []
    for ordering in (0, 1):
        plan = Plan(c["Ybus"], Vn, c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], precision=precision,
                    ordering=ordering)
        out.append((plan.info()["levels_refactor"],) + tuple(plan.batch_n1(coeffs, Vn, c["Sbus"], 10, 1e-8)))
    (l0, V0, c0, i0, e0), (l1, V1, c1, i1, e1) = out
    assert l0 < l1
    assert np.array_equal(e0, e1) and np.array_equal(c0, c1)
    if precision == 0:
        assert np.array_equal(i0, i1)
    tol = TOL_FP64 if precision == 0 else TOL_MIXED
    for k in np.nonzero(c0)[0]:
        assert _vdiff(V0[k], V1[k]) <= tol, k


def test_n1_computer_api():
    from lightsim2grid_b200 import ContingencyAnalysisCPP, SolverType

    c = grid_problem("grid118")
    g = c["grid"]
    ca = ContingencyAnalysisCPP(g)
    ca.change_solver(SolverType.GPUNRSingleSlack)
    ca.add_all_n1()
    assert len(ca.my_defaults()) == g.nb_powerline()
    ca.compute(c["V0"], 10, 1e-8)
    V = ca.get_voltages()
    assert V.shape == (g.nb_powerline(), g.n_bus)
    ca.compute_flows()
    A = ca.get_flows()
    conv = ca.get_convergence()
    assert np.all(np.isnan(A[~conv])) and np.all(A[conv, np.nonzero(conv)[0]] == 0.0)
    connected = ca.is_grid_connected_after_contingency()
    assert np.array_equal(connected == 0, ca.get_errors() == 1)


def test_time_series_matches_oracle():
    from lightsim2grid_b200 import Plan, synthetic

    c = grid_problem("grid118")
    g = c["grid"]
    gen_p, sgen_p, load_p, load_q = synthetic.time_series_injections(g, 48, seed=7)
    Sb = g.sbuses_from_injections(gen_p, sgen_p, load_p, load_q)
    st_o, Vo, conv_o, it_o, err_o = time_series(c["Ybus"], c["Sbus"], Sb, c["V0"], c["ref"], c["weights"], c["pv"],
                                                c["pq"])
    assert st_o == 1
    plan = Plan(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], precision=0)
    # one chunk: the reference's exact warm-start chain
    st, V, conv, iters, errs = plan.batch_ts(Sb, c["V0"], 1, 10, 1e-8)
    assert st == 1 and conv.all()
    assert np.array_equal(iters, it_o)
    assert max(_vdiff(V[k], Vo[k]) for k in range(48)) <= TOL_FP64
    # 8 chunks: each chunk restarts from V0; the answers agree within the solver tolerance
    st, V8, conv8, _, _ = plan.batch_ts(Sb, c["V0"], 8, 10, 1e-8)
    assert st == 1 and conv8.all()
    assert max(_vdiff(V8[k], Vo[k]) for k in range(48)) <= 1e-7


def test_time_series_stops_at_first_divergence():
    from lightsim2grid_b200 import Plan

    c = grid_problem("grid118")
    Sb = np.tile(c["Sbus"], (10, 1))
    Sb[6] *= 40.0  # step 6 cannot be solved
    st_o, Vo, conv_o, it_o, err_o = time_series(c["Ybus"], c["Sbus"], Sb, c["V0"], c["ref"], c["weights"], c["pv"],
                                                c["pq"])
    plan = Plan(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], precision=0)
    st, V, conv, iters, errs = plan.batch_ts(Sb, c["V0"], 1, 10, 1e-8)
    assert st == st_o == 0
    assert np.array_equal(conv, conv_o)
    assert np.all(V[6:] == 0)


def test_device_batch_matches_host_batch():
    import torch
    from lightsim2grid_b200 import Plan, _native as nat

    c = grid_problem("grid118")
    coeffs = _n1(c)
    plan = Plan(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], precision=0)
    V, conv, iters, errs = plan.batch_n1(coeffs, c["V0"], c["Sbus"], 10, 1e-8)
    lib = plan._lib
    cp = np.zeros(len(coeffs) + 1, np.int32)
    rows, cols, vals = [], [], []
    for k, lst in enumerate(coeffs):
        cp[k + 1] = cp[k] + len(lst)
        for (r, cc, y) in lst:
            rows.append(r)
            cols.append(cc)
            vals.append(y)
    rows, cols, vals = nat.as_i32(rows), nat.as_i32(cols), nat.as_c128(vals).ravel()
    solv = np.zeros(len(coeffs), np.int32)
    optr = np.zeros(len(coeffs) + 1, np.int32)
    opos = np.zeros(cp[-1], np.int32)
    oval = np.zeros(cp[-1], np.complex128)
    w = lib.pf_n1_prepare(plan.handle, len(coeffs), nat.ptr(cp, nat.i32p), nat.ptr(rows, nat.i32p),
                          nat.ptr(cols, nat.i32p), nat.cptr(vals), nat.ptr(solv, nat.i32p), nat.ptr(optr, nat.i32p),
                          nat.ptr(opos, nat.i32p), nat.cptr(oval), int(cp[-1]))
    assert w >= 0
    ns = int(solv.sum())
    dev = torch.device("cuda:0")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    dV0 = t(nat.as_c128(c["V0"]).ravel().view(np.float64))
    dS = t(nat.as_c128(c["Sbus"]).ravel().view(np.float64))
    dptr, dpos, dval = t(optr[:ns + 1]), t(opos[:w]), t(oval[:w].view(np.float64))
    jf = t(np.arange(ns, dtype=np.int32))
    jc = t(np.ones(ns, dtype=np.int32))
    dVout = torch.zeros(ns * c["Ybus"].shape[0] * 2, dtype=torch.float64, device=dev)
    dit = torch.zeros(ns, dtype=torch.int32, device=dev)
    der = torch.zeros(ns, dtype=torch.int32, device=dev)
    b = nat.PfDeviceBatch(n_inst=ns, V0=dV0.data_ptr(), v0_stride=0, Sbus=dS.data_ptr(), sbus_stride=0,
                          ovr_ptr=dptr.data_ptr(), ovr_pos=dpos.data_ptr(), ovr_val=dval.data_ptr(), max_iter=10,
                          tol=1e-8, chain=0, job_first=jf.data_ptr(), job_count=jc.data_ptr(), njobs=ns,
                          Vout=dVout.data_ptr(), iters=dit.data_ptr(), errs=der.data_ptr())
    stream = torch.cuda.current_stream().cuda_stream
    assert lib.pf_batch_device(plan.handle, nat.ctypes.byref(b), stream) == 0, nat.last_error(lib)
    torch.cuda.synchronize()
    Vd = dVout.cpu().numpy().view(np.complex128).reshape(ns, -1)
    idx = np.nonzero(solv)[0]
    ok = conv[idx]
    assert np.array_equal(der.cpu().numpy() == 0, ok)
    assert np.array_equal(Vd[ok], V[idx[ok]])


def test_n1_order_is_hardest_first():
    """pf_n1_order: a permutation of the solvable instances by decreasing power mismatch of the
    outage at V0 (restated here with numpy); device batches in that order give the same results."""
    from lightsim2grid_b200 import Plan, _native as nat

    c = grid_problem("grid118")
    g = c["grid"]
    coeffs = _n1(c)
    plan = Plan(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], precision=0)
    lib = plan._lib
    cp = np.zeros(len(coeffs) + 1, np.int32)
    rows, cols, vals = [], [], []
    for k, lst in enumerate(coeffs):
        cp[k + 1] = cp[k] + len(lst)
        for (r, cc, y) in lst:
            rows.append(r)
            cols.append(cc)
            vals.append(y)
    rows, cols, vals = nat.as_i32(rows), nat.as_i32(cols), nat.as_c128(vals).ravel()
    solv = np.zeros(len(coeffs), np.int32)
    optr = np.zeros(len(coeffs) + 1, np.int32)
    opos = np.zeros(cp[-1], np.int32)
    oval = np.zeros(cp[-1], np.complex128)
    w = lib.pf_n1_prepare(plan.handle, len(coeffs), nat.ptr(cp, nat.i32p), nat.ptr(rows, nat.i32p),
                          nat.ptr(cols, nat.i32p), nat.cptr(vals), nat.ptr(solv, nat.i32p), nat.ptr(optr, nat.i32p),
                          nat.ptr(opos, nat.i32p), nat.cptr(oval), int(cp[-1]))
    ns = int(solv.sum())
    V0 = nat.as_c128(c["V0"]).ravel()
    order = np.zeros(ns, np.int32)
    assert lib.pf_n1_order(plan.handle, ns, nat.ptr(optr, nat.i32p), nat.ptr(opos, nat.i32p), nat.cptr(oval),
                           nat.cptr(V0), nat.ptr(order, nat.i32p)) == 0
    assert np.array_equal(np.sort(order), np.arange(ns))
    # the score restated: dS_r = V_r conj(sum dY_rc V_c) over the instance's changed entries
    Yc = c["Ybus"].tocsr()
    Yc.sort_indices()
    r_of = np.repeat(np.arange(Yc.shape[0]), np.diff(Yc.indptr))
    score = np.zeros(ns)
    for i in range(ns):
        acc = {}
        for k in range(optr[i], optr[i + 1]):
            p = opos[k]
            r, cc = r_of[p], Yc.indices[p]
            acc[r] = acc.get(r, 0) + (oval[k] - Yc.data[p]) * V0[cc]
        score[i] = max(abs(V0[r] * np.conj(v)) for r, v in acc.items())
    assert np.all(np.diff(score[order]) <= 1e-12 * max(1.0, score.max()))


def test_n1_rows_into_pinned_output_match_pageable():
    """pf_batch_n1 writes the rows straight into a pinned, device-mapped output array (zero rows
    for islanded and failed cases, FP64 re-run rows included): the same arrays as through the
    device buffer and copy used for pageable outputs."""
    import torch
    from lightsim2grid_b200 import Plan

    c = grid_problem("grid2848")
    o_n = OracleNR(False)
    assert o_n.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
    Vn = o_n.get_V()
    g = c["grid"]
    coeffs = [g.branch_coeffs([b]) for b in range(g.nb_powerline())]
    plan = Plan(c["Ybus"], Vn, c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], precision=1)
    Vp, convp, itp, errp = plan.batch_n1(coeffs, Vn, c["Sbus"], 10, 1e-8)
    nc, n = len(coeffs), g.n_bus
    pinned = torch.empty(nc * n * 2, dtype=torch.float64, pin_memory=True).numpy().view(np.complex128)
    pinned = pinned.reshape(nc, n)
    pinned[:] = 7.0  # every row must be written
    ints = [torch.full((nc,), -5, dtype=torch.int32, pin_memory=True).numpy() for _ in range(3)]
    cp = np.zeros(nc + 1, np.int32)
    rows, cols, vals = [], [], []
    for k, lst in enumerate(coeffs):
        cp[k + 1] = cp[k] + len(lst)
        for (r, cc, y) in lst:
            rows.append(r)
            cols.append(cc)
            vals.append(y)
    for _ in range(2):
        V, conv, it, err = plan.batch_n1_arrays(cp, rows, cols, vals, Vn, c["Sbus"], 10, 1e-8,
                                                out=(pinned, *ints))
        assert np.array_equal(err, errp) and np.array_equal(it, itp) and np.array_equal(conv, convp)
        assert np.array_equal(V, Vp)
    assert (errp == 1).any() and (errp > 1).any()  # islanded and failed cases are exercised


@pytest.mark.parametrize("diverge", [False, True])
def test_time_series_rows_into_pinned_output_match_pageable(diverge):
    """pf_batch_ts with a pinned, device-mapped output (rows written by the kernel, zero rows
    after the first divergence) gives the same arrays as the copy path of pageable outputs."""
    import torch
    from lightsim2grid_b200 import Plan, synthetic

    c = grid_problem("grid118")
    g = c["grid"]
    gen_p, sgen_p, load_p, load_q = synthetic.time_series_injections(g, 40, seed=11)
    Sb = g.sbuses_from_injections(gen_p, sgen_p, load_p, load_q)
    if diverge:
        Sb[25] *= 40.0
    plan = Plan(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], precision=1)
    ref = plan.batch_ts(Sb, c["V0"], 4, 10, 1e-8)
    n = g.n_bus
    Vp = torch.empty(40 * n * 2, dtype=torch.float64, pin_memory=True).numpy().view(np.complex128).reshape(40, n)
    Vp[:] = 7.0
    ints = [torch.full((40,), -5, dtype=torch.int32, pin_memory=True).numpy() for _ in range(3)]
    for _ in range(2):
        st, V, conv, it, er = plan.batch_ts(Sb, c["V0"], 4, 10, 1e-8, out=(Vp, *ints))
        assert st == ref[0]
        assert np.array_equal(conv, ref[2]) and np.array_equal(it, ref[3]) and np.array_equal(er, ref[4])
        assert np.array_equal(V, ref[1])
    if diverge:
        assert st == 0 and np.all(V[25:] == 0)
