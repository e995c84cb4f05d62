"""Serving loop on the GPU: requests that overlap on the device (continuous batching over
several grids) give the same results as each request run alone, and the results match the
oracle (power flow from the base-case state with scaled injections; N-1 batch as the
reference's ContingencyAnalysis, ContingencyAnalysis.cpp:166-233)."""
import numpy as np
import pytest

from oracle.oracle import OracleNR, contingency_analysis

pytestmark = pytest.mark.gpu

TOL_ORACLE = 1e-8  # |V - V_oracle| (pu) for the mixed form converged at 1e-8 pu


@pytest.fixture(scope="module", params=["launch per request", "device loop"])
def server(request):
    from lightsim2grid_b200 import synthetic
    from lightsim2grid_b200.serving import PowerFlowServer

    # the six grids of the serving workload (14 to 6,515 buses): the large grids' CTAs are the
    # ones that stay resident longest beside other requests
    grids = {name: synthetic.make_named_grid(name)[0]
             for name in ("grid14", "grid118", "grid300", "grid1354", "grid2848", "grid6515")}
    srv = PowerFlowServer(grids, hbm_budget=2 << 30, slots=16, precision=1, large_request_ctas=16,
                          device_loop=request.param == "device loop")
    srv.grids = grids
    return srv


def _requests(srv, seed, duration=0.04, rate=3000):
    from lightsim2grid_b200.serving import make_requests

    g = srv.grids
    return make_requests({k: v.n_bus for k, v in g.items()}, rate=rate, duration=duration, seed=seed,
                         branches_of={k: v.nb_powerline() for k, v in g.items()}, n1_min=8, n1_max=24)


def test_mix_equals_alone(server):
    reqs = _requests(server, seed=11)
    assert len(reqs) >= 40
    done = server.serve(reqs, realtime=True)
    assert len(done) == len(reqs)
    assert server.last.peak_inflight >= 2  # work did overlap
    by_id = {r.rid: r for r in done}
    # every fifth request, and every request on the three largest grids
    picked = set(sorted(by_id)[::5]) | {rid for rid, r in by_id.items() if r.grid in ("grid1354", "grid2848",
                                                                                     "grid6515")}
    assert {by_id[rid].grid for rid in picked} >= {"grid1354", "grid2848", "grid6515"}
    for rid in sorted(picked):
        mix = by_id[rid]
        alone = server.solve_alone(mix)
        assert np.array_equal(alone.errs, mix.errs) and np.array_equal(alone.iters, mix.iters)
        assert np.array_equal(alone.V, mix.V)  # bit for bit: one CTA per instance, same inputs


def test_results_match_oracle(server):
    from lightsim2grid_b200.serving import PF

    reqs = _requests(server, seed=5, duration=0.02)
    done = server.serve(reqs, realtime=True)
    checked = {"pf": 0, "n1": 0}
    for r in done:
        s = server.services[r.grid]
        g = server.grids[r.grid]
        Y, sl, w, pv, pq = g.get_Ybus(), g.get_slack_ids(), g.get_slack_weights(), g.get_pv(), g.get_pq()
        if r.kind == PF and checked["pf"] < 6:
            o = OracleNR(False)
            ok = o.compute_pf(Y, s.Vbase, s.Sbase * r.scale, sl, w, pv, pq, 10, 1e-8)
            assert bool(r.converged[0]) == ok
            if ok:
                assert np.abs(r.V[0] - o.get_V()).max() <= TOL_ORACLE
            checked["pf"] += 1
        elif r.kind != PF and checked["n1"] < 4:
            coeffs = [g.branch_coeffs([int(b)]) for b in r.branches]
            _, Vo, conv_o, _, _ = contingency_analysis(Y, s.Sbase, s.Vbase, sl, w, pv, pq, coeffs, 10, 1e-8)
            # results in case order: islanded outages skipped (zero row), as the reference does
            assert np.array_equal(r.converged, conv_o.astype(bool))
            ok = r.converged
            assert np.all(r.V[~ok] == 0)
            if ok.any():
                assert np.abs(r.V[ok] - Vo[ok]).max() <= TOL_ORACLE
            checked["n1"] += 1
    assert checked["pf"] >= 3 and checked["n1"] >= 2


def test_device_loop_equals_launch_per_request(server):
    """The same requests through the persistent device loop and through one launch per request:
    the same bits (the same solver code per instance, inputs read through L2 in both)."""
    reqs = _requests(server, seed=23, duration=0.03)
    done = {r.rid: r for r in server.serve(reqs, realtime=True)}
    other = not server.native.device_loop
    server.native.set_device_loop(other)
    try:
        again = {r.rid: r for r in server.serve(_requests(server, seed=23, duration=0.03), realtime=True)}
    finally:
        server.native.set_device_loop(not other)
    assert set(done) == set(again) and len(done) >= 20
    for rid, r in done.items():
        a = again[rid]
        assert np.array_equal(r.errs, a.errs) and np.array_equal(r.iters, a.iters), rid
        assert np.array_equal(r.V, a.V), rid


def test_latency_split_counts_every_request(server):
    """pf_server_latency_split: per grid and kind, every finished request is counted once, with
    non-negative admission wait and device time, and reset clears the counts."""
    g = server.grids
    for name in g:
        for kind in ("pf", "n1"):
            server.native.latency_split(name, kind, reset=True)
    reqs = _requests(server, seed=31, duration=0.03)
    done = server.serve(reqs, realtime=True)
    assert len(done) == len(reqs)
    total = 0
    for name in g:
        for kind in ("pf", "n1"):
            n = sum(1 for r in done if r.grid == name and r.kind == kind)
            sp = server.native.latency_split(name, kind, reset=True)
            assert sp["count"] == n, (name, kind)
            if n:
                assert 0.0 <= sp["wait_p50_ms"] <= sp["wait_p99_ms"]
                assert 0.0 <= sp["device_p50_ms"] <= sp["device_p99_ms"]
            assert server.native.latency_split(name, kind)["count"] == 0
            total += n
    assert total == len(reqs)
