"""World-size-2 gloo run of the multi-GPU plumbing on CPU: contiguous shards cover every
case once, the gathered per-shard results equal the single-process result, and timings are
reduced as the max over ranks.  The per-rank compute here is the CPU oracle (no GPU)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from lightsim2grid_b200.replicas import shard_bounds, aggregate_rate


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_q):
    import sys
    import datetime
    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from lightsim2grid_b200 import synthetic
        from lightsim2grid_b200.replicas import shard_bounds, max_over_ranks, gather_rows
        from oracle.oracle import contingency_analysis

        g, _ = synthetic.make_named_grid("grid118")
        coeffs = [g.branch_coeffs([b]) for b in range(g.nb_powerline())]
        a, b = shard_bounds(len(coeffs), rank, world)
        ok, V, conv, iters, errs = contingency_analysis(g.get_Ybus(), g.get_Sbus(), g.flat_start(),
                                                        g.get_slack_ids(), g.get_slack_weights(), g.get_pv(),
                                                        g.get_pq(), coeffs[a:b])
        full_V = gather_rows(V, len(coeffs))
        full_conv = gather_rows(conv, len(coeffs))
        tmax = max_over_ranks(1.0 + rank)
        if rank == 0:
            out_q.put((full_V, full_conv, tmax))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_shards_cover_all_cases():
    for n in (0, 1, 7, 186):
        for w in (1, 2, 3, 8):
            seen = []
            for r in range(w):
                a, b = shard_bounds(n, r, w)
                seen.extend(range(a, b))
            assert seen == list(range(n))
    assert aggregate_rate(100, 2.0, 4) == 200.0


def test_two_rank_gloo_gather_and_max():
    from lightsim2grid_b200 import synthetic
    from oracle.oracle import contingency_analysis

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    full_V, full_conv, tmax = q.get(timeout=240)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    g, _ = synthetic.make_named_grid("grid118")
    coeffs = [g.branch_coeffs([b]) for b in range(g.nb_powerline())]
    ok, V, conv, iters, errs = contingency_analysis(g.get_Ybus(), g.get_Sbus(), g.flat_start(), g.get_slack_ids(),
                                                    g.get_slack_weights(), g.get_pv(), g.get_pq(), coeffs)
    assert np.array_equal(full_conv, conv)
    # the reference's loop subtracts and re-adds each case's coefficients in place, so Ybus
    # carries round-off from earlier cases (ContingencyAnalysis.cpp:204-231): a shard that
    # starts mid-list sees a Ybus differing in the last bits
    assert np.abs(full_V - V).max() <= 1e-12
    assert tmax == 2.0
