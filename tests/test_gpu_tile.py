"""The batch-interleaved Newton kernel (pf_tile.cu: 32 instances per CTA, one per lane) against
the CPU oracle and against the one-CTA-per-instance kernel, through the C ABI.

Same bars as the other Newton parity tests: FP64 -- the oracle's convergence flags and
iteration counts, |dVm|, |dVa| <= 1e-10 pu; mixed -- the oracle's flags, |dV| <= 1e-8 pu.
"""
import numpy as np
import pytest

from conftest import grid_problem
from oracle.oracle import OracleNR, contingency_analysis

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10
TOL_MIXED = 1e-8


def _vdiff(a, b):
    return max(np.abs(np.abs(a) - np.abs(b)).max(), np.abs(np.angle(a) - np.angle(b)).max())


def _base(c, distributed=False):
    o = OracleNR(distributed)
    assert o.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
    return o.get_V()


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name,ncases", [("grid118", None), ("grid1354", 400), ("grid2848", 300)])
def test_tile_n1_matches_oracle(precision, name, ncases):
    from lightsim2grid_b200 import Plan

    c = grid_problem(name)
    g = c["grid"]
    Vn = _base(c)
    nb = g.nb_powerline() if ncases is None else ncases
    coeffs = [g.branch_coeffs([b]) for b in range(nb)]
    ok, Vo, conv_o, it_o, err_o = contingency_analysis(c["Ybus"], c["Sbus"], Vn, c["ref"], c["weights"], c["pv"],
                                                       c["pq"], coeffs)
    plan = Plan(c["Ybus"], Vn, c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], precision=precision,
                batch_layout=2)
    V, conv, iters, errs = plan.batch_n1(coeffs, Vn, c["Sbus"], 10, 1e-8)
    assert np.array_equal(errs == 1, err_o == 8), name
    assert np.array_equal(conv, conv_o), name
    if precision == 0:
        assert np.array_equal(iters[conv], it_o[conv_o]), name
    tol = TOL_FP64 if precision == 0 else TOL_MIXED
    for k in np.nonzero(conv)[0]:
        assert _vdiff(V[k], Vo[k]) <= tol, (name, k)
    assert np.all(V[~conv] == 0)


@pytest.mark.parametrize("precision", [0, 1])
def test_tile_distributed_slack_matches_one_cta_kernel(precision):
    """Two slacks with weights: the interleaved and the one-CTA kernels agree."""
    from lightsim2grid_b200 import Plan

    c = dict(grid_problem("grid118"))
    g = c["grid"]
    pv = np.asarray(c["pv"])
    ref = np.r_[np.asarray(c["ref"])[:1], pv[:1]]
    w = np.zeros(g.n_bus)
    w[ref] = [0.7, 0.3]
    c.update(ref=ref, weights=w, pv=pv[1:])
    Vn = _base(c, distributed=True)
    coeffs = [g.branch_coeffs([b]) for b in range(g.nb_powerline())]
    out = []
    for layout in (1, 2):
        plan = Plan(c["Ybus"], Vn, c["Sbus"], ref, w, c["pv"], c["pq"], distributed=True, precision=precision,
                    batch_layout=layout)
        out.append(plan.batch_n1(coeffs, Vn, c["Sbus"], 10, 1e-8))
    (V1, c1, i1, e1), (V2, c2, i2, e2) = out
    assert np.array_equal(e1, e2) and np.array_equal(c1, c2)
    if precision == 0:
        assert np.array_equal(i1, i2)
    tol = TOL_FP64 if precision == 0 else TOL_MIXED
    for k in np.nonzero(c1)[0]:
        assert _vdiff(V1[k], V2[k]) <= tol, k


def test_tile_device_batch_with_multi_instance_jobs():
    """Device batch whose jobs hold several independent instances (chain 0) and more jobs than
    lanes: every instance as in the one-CTA kernel."""
    import torch
    from lightsim2grid_b200 import Plan, _native as nat

    c = grid_problem("grid118")
    g = c["grid"]
    Vn = _base(c)
    coeffs = [g.branch_coeffs([b]) for b in range(g.nb_powerline())]
    res = []
    for layout in (1, 2):
        plan = Plan(c["Ybus"], Vn, c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], precision=0,
                    batch_layout=layout)
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
                              nat.ptr(cols, nat.i32p), nat.cptr(vals), nat.ptr(solv, nat.i32p),
                              nat.ptr(optr, nat.i32p), nat.ptr(opos, nat.i32p), nat.cptr(oval), int(cp[-1]))
        assert w >= 0
        ns = int(solv.sum())
        # jobs of 1 to 3 instances
        jf, jc, i = [], [], 0
        while i < ns:
            k = min(1 + (i % 3), ns - i)
            jf.append(i)
            jc.append(k)
            i += k
        dev = torch.device("cuda:0")
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        bufs = [t(nat.as_c128(Vn).ravel().view(np.float64)), t(nat.as_c128(c["Sbus"]).ravel().view(np.float64)),
                t(optr[:ns + 1]), t(opos[:w]), t(oval[:w].view(np.float64)), t(np.array(jf, np.int32)),
                t(np.array(jc, np.int32))]
        dV = torch.zeros(ns * g.n_bus * 2, dtype=torch.float64, device=dev)
        dit = torch.zeros(ns, dtype=torch.int32, device=dev)
        der = torch.zeros(ns, dtype=torch.int32, device=dev)
        b = nat.PfDeviceBatch(n_inst=ns, V0=bufs[0].data_ptr(), v0_stride=0, Sbus=bufs[1].data_ptr(),
                              sbus_stride=0, ovr_ptr=bufs[2].data_ptr(), ovr_pos=bufs[3].data_ptr(),
                              ovr_val=bufs[4].data_ptr(), max_iter=10, tol=1e-8, chain=0,
                              job_first=bufs[5].data_ptr(), job_count=bufs[6].data_ptr(), njobs=len(jf),
                              Vout=dV.data_ptr(), iters=dit.data_ptr(), errs=der.data_ptr())
        assert lib.pf_batch_device(plan.handle, nat.ctypes.byref(b), torch.cuda.current_stream().cuda_stream) == 0
        torch.cuda.synchronize()
        res.append((dV.cpu().numpy().view(np.complex128).reshape(ns, -1), dit.cpu().numpy(), der.cpu().numpy()))
    (V1, i1, e1), (V2, i2, e2) = res
    assert np.array_equal(e1, e2) and np.array_equal(i1, i2)
    ok = e1 == 0
    assert max(_vdiff(V1[k], V2[k]) for k in np.nonzero(ok)[0]) <= TOL_FP64


def _threads():
    import os

    try:
        return max(1, len(os.sched_getaffinity(0)))
    except Exception:
        return 1


@pytest.mark.parametrize("precision", [0, 1])
def test_tile_headline_batch_with_hand_off_matches_oracle(precision):
    """Every outage of the 2,848-bus grid through the batch-interleaved layout: the CTAs hand their
    last running instances to the one-CTA kernel (continued from their state) and, in the mixed
    form, the 11 instances that fail in FP32 are solved again in FP64 -- all in one stream, and
    the results are the oracle's (FP64: flags, error codes and iteration counts)."""
    from lightsim2grid_b200 import Plan
    from oracle.oracle import ContingencyBatch

    c = grid_problem("grid2848")
    g = c["grid"]
    Vn = _base(c)
    coeffs = [g.branch_coeffs([b]) for b in range(g.nb_powerline())]
    ob = ContingencyBatch(c["Ybus"], c["Sbus"], Vn, c["ref"], c["weights"], c["pv"], c["pq"], coeffs)
    ok, Vo, conv_o, it_o, err_o, _ = ob.run(_threads())
    plan = Plan(c["Ybus"], Vn, c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], precision=precision,
                batch_layout=2)
    V, conv, iters, errs = plan.batch_n1(coeffs, Vn, c["Sbus"], 10, 1e-8)
    isl = err_o == 8
    assert np.array_equal(errs == 1, isl)
    assert np.array_equal(conv, conv_o)
    assert np.array_equal(errs[~isl], err_o[~isl])
    failed = ~isl & ~conv_o
    if precision == 0:
        assert np.array_equal(iters[~isl], it_o[~isl])
    else:
        assert plan.timers()[5] >= failed.sum()
        assert np.array_equal(iters[failed], it_o[failed])
    tol = TOL_FP64 if precision == 0 else TOL_MIXED
    assert max(_vdiff(V[k], Vo[k]) for k in np.nonzero(conv)[0]) <= tol
    assert np.all(V[~conv] == 0)


@pytest.mark.parametrize("precision", [0, 1])
def test_auto_layout_on_the_largest_grid_matches_oracle(precision):
    """The 6,515-bus plans keep their LU in global memory; with enough jobs per SM the default
    layout is the batch-interleaved one.  1,200 outages against the oracle."""
    from lightsim2grid_b200 import Plan
    from oracle.oracle import ContingencyBatch

    c = grid_problem("grid6515")
    g = c["grid"]
    Vn = _base(c)
    coeffs = [g.branch_coeffs([b]) for b in range(1200)]
    ob = ContingencyBatch(c["Ybus"], c["Sbus"], Vn, c["ref"], c["weights"], c["pv"], c["pq"], coeffs)
    ok, Vo, conv_o, it_o, err_o, _ = ob.run(_threads())
    plan = Plan(c["Ybus"], Vn, c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], precision=precision)
    assert plan.info()["lu_in_shared"] == 0 and plan.info()["nnz_lu"] >= 60000
    V, conv, iters, errs = plan.batch_n1(coeffs, Vn, c["Sbus"], 10, 1e-8)
    isl = err_o == 8
    assert np.array_equal(errs == 1, isl)
    assert np.array_equal(conv, conv_o)
    if precision == 0:
        assert np.array_equal(iters[~isl], it_o[~isl])
    tol = TOL_FP64 if precision == 0 else TOL_MIXED
    assert max(_vdiff(V[k], Vo[k]) for k in np.nonzero(conv)[0]) <= tol
