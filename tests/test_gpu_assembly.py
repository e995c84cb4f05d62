"""Ybus and Sbus assembled on the GPU against the host restatement of the reference's
GridModel::fillYbus / fillSbus_me (GridModel.cpp:676-716) and TimeSeries::compute_Sbuses
(TimeSeries.hpp:79-151), and a power flow on device-assembled Ybus values."""
import numpy as np
import pytest

from conftest import grid_problem

pytestmark = pytest.mark.gpu

RTOL = 1e-15  # the reference sums in branch order, the host restatement in scipy's order


def _close(a, b):
    assert np.all(np.abs(a - b) <= RTOL * np.maximum(1.0, np.abs(b))), np.abs(a - b).max()


@pytest.fixture(scope="module")
def setup():
    import torch

    from lightsim2grid_b200 import Plan
    from lightsim2grid_b200.assembly import DeviceAssembly

    c = grid_problem("grid118")
    g = c["grid"]
    plan = Plan(g.get_Ybus(), c["V0"], g.get_Sbus(), g.get_slack_ids(), g.get_slack_weights(), g.get_pv(),
                g.get_pq(), precision=0)
    return c, g, plan, DeviceAssembly(plan, g, torch.device("cuda:0"))


def test_ybus_matches_host_assembly(setup):
    import torch

    c, g, plan, asm = setup
    yv = asm.ybus(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    dev = yv.cpu().numpy().view(np.complex128)
    _close(dev, asm.host_ybus_in_storage_order(g.get_Ybus()))


def test_changed_branches_and_solve(setup):
    import torch

    from lightsim2grid_b200 import Plan

    c, g, plan, asm = setup
    st = torch.cuda.current_stream().cuda_stream
    r, x, h, on = g.line_r.copy(), g.line_x.copy(), g.line_h.copy(), g.line_status.copy()
    r2, x2, on2 = r.copy(), x.copy(), on.copy()
    r2[3] *= 1.5
    x2[7] *= 0.8
    on2[11] = False
    g.line_r, g.line_x, g.line_status = r2, x2, on2
    try:
        Yh = g.get_Ybus()
        asm.set_branches(r2, x2, h, on2)
        yv = asm.ybus(st)
        torch.cuda.synchronize()
        _close(yv.cpu().numpy().view(np.complex128), asm.host_ybus_in_storage_order(Yh))
        # the plan solves on the device-assembled values like a plan built from the host Ybus
        asm.apply(yv, st)
        torch.cuda.synchronize()
        S = g.get_Sbus()
        V, conv, it, err = plan.solve(c["V0"], S, 10, 1e-8)
        ref = Plan(Yh, c["V0"], S, g.get_slack_ids(), g.get_slack_weights(), g.get_pv(), g.get_pq(), precision=0)
        Vr, convr, itr, _ = ref.solve(c["V0"], S, 10, 1e-8)
        assert conv and convr and it == itr
        assert np.abs(V - Vr).max() <= 1e-10
    finally:
        g.line_r, g.line_x, g.line_status = r, x, on
        asm.set_branches(r, x, h, on)
        asm.apply(asm.ybus(st), st)
        torch.cuda.synchronize()


def test_sbus_rows_match_host(setup):
    import torch

    from lightsim2grid_b200 import synthetic

    c, g, plan, asm = setup
    gp, _, lp, lq = synthetic.time_series_injections(g, 50, seed=3)
    dev = torch.device("cuda:0")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    out = asm.sbus(t(gp), t(lp), t(lq), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    S = out.cpu().numpy().view(np.complex128).reshape(50, g.n_bus)
    Sh = g.sbuses_from_injections(gp, np.zeros((50, 0)), lp, lq)
    assert np.array_equal(S, Sh)  # same element order per bus, same operations
