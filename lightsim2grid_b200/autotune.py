"""Autotuner for the engine's schedules.

A plan's level-group schedules (the phase programs) are laid out for a thread count: the
operations of every elimination level are packed onto that many threads, so the thread count
sets the width of every phase and, with the shared-memory layout, how many CTAs stay resident
per SM.  Which setting is fastest depends on the grid (its levels' sizes) and on the batch, so
it is measured: ``tune`` builds the candidate plans, runs a sample batch of the real workload
on the device with each, and keeps the fastest (CUDA-event time per converged power flow).
"""
import json

import numpy as np

from . import _native as nat
from .solver import Plan

DEFAULT_CANDIDATES = ({"threads": 128}, {"threads": 256}, {"threads": 512})


def _time_launches(launch, repeat, stream):
    import torch

    launch()
    torch.cuda.synchronize()
    ts = []
    for _ in range(repeat):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        launch()
        e1.record(stream)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1) * 1e-3)
    return float(np.median(ts))


def tune_n1(grid, branches, precision=1, candidates=DEFAULT_CANDIDATES, repeat=3, device=None, max_iter=10,
            tol=1e-8):
    """Picks plan options for N-1 batches of ``grid``: each candidate solves the outages of
    ``branches`` from the base-case state.  Returns (best options, table of measurements)."""
    import torch

    from .multi import GridCases

    dev = torch.device("cuda:0") if device is None else torch.device(device)
    st = torch.cuda.current_stream(dev)
    table = []
    for opt in candidates:
        try:
            c = GridCases("tune", grid, branches, dev, precision=precision, max_iter=max_iter, tol=tol, **opt)
        except RuntimeError as e:  # a candidate that cannot be built or launched
            table.append({"options": dict(opt), "error": str(e)})
            continue
        k = c.ninst
        jf = torch.arange(k, dtype=torch.int32, device=dev)
        jc = torch.ones(k, dtype=torch.int32, device=dev)
        b = c.batch
        b2 = nat.PfDeviceBatch(n_inst=k, V0=b.V0, v0_stride=0, Sbus=b.Sbus, sbus_stride=0, ovr_ptr=b.ovr_ptr,
                               ovr_pos=b.ovr_pos, ovr_val=b.ovr_val, max_iter=max_iter, tol=tol, chain=0,
                               job_first=jf.data_ptr(), job_count=jc.data_ptr(), njobs=k, Vout=b.Vout,
                               iters=b.iters, errs=b.errs)
        lib = c.plan._lib

        def launch():
            nat.check(lib.pf_batch_device(c.plan.handle, nat.ctypes.byref(b2), st.cuda_stream), "pf_batch_device", lib)

        sec = _time_launches(launch, repeat, st)
        nconv = int((c.dev["er"][:k] == 0).sum().item()) if k else 0
        info = c.plan.info()
        table.append({"options": dict(opt), "seconds": sec, "converged": nconv,
                      "pf_per_s": nconv / sec if sec > 0 else None,
                      "ctas_per_sm": info["ctas_per_sm"], "lu_in_shared": info["lu_in_shared"],
                      "phases": info["groups_refactor"] + info["groups_backward"]})
    ok = [r for r in table if r.get("pf_per_s")]
    if not ok:
        raise RuntimeError("no candidate could run: " + json.dumps(table))
    best = max(ok, key=lambda r: r["pf_per_s"])
    return dict(best["options"]), table


def tune_uneven(parts, precision=1, candidates=({"threads": 256}, {"threads": 512}), repeat=3, device=None):
    """Picks the thread count of a launch over several grids (``parts``: (name, grid,
    branches)); every plan of the launch is built for it.  Returns (best options, table)."""
    import torch

    from .multi import build_uneven

    dev = torch.device("cuda:0") if device is None else torch.device(device)
    st = torch.cuda.current_stream(dev)
    table = []
    for opt in candidates:
        mb, cases = build_uneven(parts, dev, precision=precision, **opt)
        sec = _time_launches(lambda: mb.launch(st.cuda_stream), repeat, st)
        nconv = sum(int(c.results()[1].sum()) for c in cases)
        table.append({"options": dict(opt), "seconds": sec, "converged": nconv, "pf_per_s": nconv / sec,
                      "launch": mb.info()})
        mb.close()
    best = max(table, key=lambda r: r["pf_per_s"])
    return dict(best["options"]), table
