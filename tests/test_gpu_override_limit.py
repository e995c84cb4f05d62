"""Device batches whose instances carry more Ybus overrides than the kernels stage (32): such an
instance is reported as not computed (NotInitError, 0 iterations, start voltages out) instead of
being solved with a truncated override list; the other instances are unaffected."""
import numpy as np
import pytest

from conftest import grid_problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["newton", "dc", "fdpf"])
def test_too_many_overrides_is_not_computed(kind):
    import torch
    from lightsim2grid_b200 import Plan, _native as nat

    c = grid_problem("grid118")
    g = c["grid"]
    Y = g.get_dcYbus() if kind == "dc" else c["Ybus"]
    kw = {"dc": True} if kind == "dc" else ({"fdpf": g.get_Bp_Bpp(0)} if kind == "fdpf" else {})
    plan = Plan(Y, c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], precision=0, **kw)
    lib = plan._lib
    coeffs = g.dc_branch_coeffs([5]) if kind == "dc" else g.branch_coeffs([5])
    rows = nat.as_i32([e[0] for e in coeffs])
    cols = nat.as_i32([e[1] for e in coeffs])
    pos = np.zeros(rows.size, np.int32)
    assert lib.pf_ybus_positions(plan.handle, int(rows.size), rows.ctypes.data, cols.ctypes.data,
                                 pos.ctypes.data) == 0
    assert np.all(pos >= 0)
    Yc = Y.tocsr()
    vals = np.array([Yc[r, cc] - e[2] for (r, cc), e in zip(zip(rows, cols), coeffs)], np.complex128)
    # instance 0: 33 overrides (the outage's entries repeated), instance 1: the plain outage
    reps = -(-33 // pos.size)
    p0, v0 = np.tile(pos, reps)[:33], np.tile(vals, reps)[:33]
    optr = np.array([0, 33, 33 + pos.size], np.int32)
    opos = np.r_[p0, pos].astype(np.int32)
    oval = np.r_[v0, vals]
    dev = torch.device("cuda:0")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    n = g.n_bus
    V0 = nat.as_c128(c["V0"]).ravel()
    bufs = [t(V0.view(np.float64)), t(nat.as_c128(c["Sbus"]).ravel().view(np.float64)), t(optr), t(opos),
            t(oval.view(np.float64)), t(np.arange(2, dtype=np.int32)), t(np.ones(2, np.int32))]
    dV = torch.full((2 * n * 2,), 7.0, dtype=torch.float64, device=dev)
    dit = torch.full((2,), -1, dtype=torch.int32, device=dev)
    der = torch.full((2,), -1, dtype=torch.int32, device=dev)
    b = nat.PfDeviceBatch(n_inst=2, V0=bufs[0].data_ptr(), v0_stride=0, Sbus=bufs[1].data_ptr(), sbus_stride=0,
                          ovr_ptr=bufs[2].data_ptr(), ovr_pos=bufs[3].data_ptr(), ovr_val=bufs[4].data_ptr(),
                          max_iter=40, tol=1e-8, chain=0, job_first=bufs[5].data_ptr(), job_count=bufs[6].data_ptr(),
                          njobs=2, Vout=dV.data_ptr(), iters=dit.data_ptr(), errs=der.data_ptr())
    assert lib.pf_batch_device(plan.handle, nat.ctypes.byref(b), torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    V = dV.cpu().numpy().view(np.complex128).reshape(2, n)
    it, er = dit.cpu().numpy(), der.cpu().numpy()
    assert er[0] == 8 and it[0] == 0
    assert np.array_equal(V[0], V0)
    # the second instance is the ordinary outage: the host N-1 path gives the same answer
    Vh, conv, iters, errs = plan.batch_n1([coeffs], c["V0"], c["Sbus"], 40, 1e-8)
    assert er[1] == errs[0] and it[1] == iters[0]
    if errs[0] == 0:
        assert np.abs(V[1] - Vh[0]).max() <= 1e-12
