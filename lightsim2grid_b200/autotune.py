"""Autotuner for the engine's level-group and tile schedules.

A plan's schedules are fixed on the host when the plan is built, and which ones run fastest
depends on the grid and on the batch, so they are measured on the device:

* the elimination order sets the level groups (phases) of every program: minimum degree with a
  preference for low elimination levels among the vertices of degree up to the minimum +
  ``level_slack`` (``ordering`` 0; slack 2 by default, larger slacks give fewer, wider phases
  for a little more fill), or without that preference (``ordering`` 3);
* ``placement`` spreads the packed programs' clusters of operations over the phase (1, the
  default) or puts them in the first slots of their threads (2), trading shared-memory bank
  conflicts;
* ``threads`` is the width every phase is packed for and, with the shared-memory layout, sets
  the CTAs resident per SM;
* ``batch_layout`` picks one CTA per instance (1) or the batch-interleaved tile kernel (2: 32
  instances per CTA, every value interleaved over them) for N-1 batches.

``tune_n1`` times every candidate plan on a sample of the real workload (CUDA events, median
of ``repeat`` launches after one warm-up) and keeps the most converged power flows per second;
``tune_uneven`` does the same for a launch over several grids (config 3): each grid's schedule
options first, then the launch's thread count with those.  The reference analyses its matrix
once with KLU (src/linear_solvers/KLUSolver.cpp:24-45) and has nothing to tune; these choices
exist because the device schedules do.

Choices are cached per plan fingerprint (the grid's Ybus pattern and values, PV/PQ sets,
precision and the sample) in memory, and in the JSON file named by the environment variable
``LIGHTSIM2GRID_B200_TUNE_CACHE`` when it is set.
"""
import hashlib
import json
import os

import numpy as np

from . import _native as nat

_CACHE = {}


def _fingerprint(grid, precision, branches, extra=""):
    h = hashlib.sha1()
    Y = grid.get_Ybus().tocsc()
    Y.sort_indices()
    for a in (Y.indptr, Y.indices, Y.data, grid.get_pv(), grid.get_pq(), np.asarray(branches)):
        h.update(np.ascontiguousarray(a).tobytes())
    h.update("{}|{}".format(precision, extra).encode())
    return h.hexdigest()


def _cache_get(key):
    if key in _CACHE:
        return _CACHE[key]
    path = os.environ.get("LIGHTSIM2GRID_B200_TUNE_CACHE")
    if path and os.path.exists(path):
        try:
            with open(path) as fh:
                d = json.load(fh)
            if key in d:
                _CACHE[key] = d[key]
                return d[key]
        except (OSError, ValueError):
            pass
    return None


def _cache_put(key, value):
    _CACHE[key] = value
    path = os.environ.get("LIGHTSIM2GRID_B200_TUNE_CACHE")
    if path:
        try:
            d = {}
            if os.path.exists(path):
                with open(path) as fh:
                    d = json.load(fh)
            d[key] = value
            with open(path, "w") as fh:
                json.dump(d, fh)
        except (OSError, ValueError):
            pass


def schedule_candidates(m):
    """Elimination-order and placement candidates (threads left to the plan's default)."""
    out = []
    for order in ({"ordering": 0}, {"ordering": 0, "level_slack": 4}, {"ordering": 3}):
        for placement in (1, 2):
            out.append(dict(order, placement=placement))
    return out


def n1_candidates(m, n):
    """Candidates for N-1 batches of a grid with m unknowns and n buses."""
    threads = (128, 256) if m < 600 else ((256, 512) if m < 4000 else (512, 640, 768))
    out = []
    for t in threads:
        for c in schedule_candidates(m):
            out.append(dict(c, threads=t, batch_layout=1))
    if n >= 1000:
        out.append({"batch_layout": 2})
    return out


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


def tune_n1(grid, branches, precision=1, candidates=None, repeat=3, device=None, max_iter=10, tol=1e-8):
    """Picks plan options for N-1 batches of ``grid``: each candidate solves the outages of
    ``branches`` from the base-case state.  Returns (best options, table of measurements)."""
    import torch

    from .multi import GridCases

    dev = torch.device("cuda:0") if device is None else torch.device(device)
    st = torch.cuda.current_stream(dev)
    m = int(grid.get_pv().size + 2 * grid.get_pq().size)
    if candidates is None:
        candidates = n1_candidates(m, grid.n_bus)
    key = _fingerprint(grid, precision, branches, json.dumps(candidates, sort_keys=True) + "|n1")
    hit = _cache_get(key)
    if hit is not None:
        return dict(hit["best"]), hit["table"]
    table = []
    base_state = None
    for opt in candidates:
        try:
            c = GridCases("tune", grid, branches, dev, precision=precision, max_iter=max_iter, tol=tol,
                          base_state=base_state, **opt)
        except RuntimeError as e:  # a candidate that cannot be built or launched
            table.append({"options": dict(opt), "error": str(e)})
            continue
        base_state = (c.Vbase, c.Sbase)
        k = c.ninst
        jf = torch.from_numpy(np.ascontiguousarray(c.order)).to(dev)
        jc = torch.ones(max(k, 1), dtype=torch.int32, device=dev)
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
                      "pf_per_s": nconv / sec if sec > 0 else None, "threads": info["threads"],
                      "ctas_per_sm": info["ctas_per_sm"], "lu_in_shared": info["lu_in_shared"],
                      "levels": info["levels_refactor"],
                      "phases": info["groups_refactor"] + info["groups_backward"]})
        del c
    ok = [r for r in table if r.get("pf_per_s")]
    if not ok:
        raise RuntimeError("no candidate could run: " + json.dumps(table))
    best = max(ok, key=lambda r: r["pf_per_s"])
    _cache_put(key, {"best": best["options"], "table": table})
    return dict(best["options"]), table


def tune_uneven(parts, precision=1, repeat=3, device=None, threads=(256, 512, 640, 768), schedules=True):
    """Picks the options of a launch over several grids (``parts``: (name, grid, branches)):
    for each grid the schedule options (elimination order and level slack, placement) that run
    its own sample fastest, then the launch's thread count with those.  Returns (options for
    ``build_uneven``, table of measurements)."""
    import torch

    from .multi import build_uneven

    dev = torch.device("cuda:0") if device is None else torch.device(device)
    st = torch.cuda.current_stream(dev)
    per_grid, table = {}, {"per_grid": {}, "threads": []}
    if schedules:
        for name, g, br in parts:
            m = int(g.get_pv().size + 2 * g.get_pq().size)
            cands = [dict(c, threads=max(threads), batch_layout=1) for c in schedule_candidates(m)]
            best, tab = tune_n1(g, br, precision=precision, candidates=cands, repeat=repeat, device=dev)
            best = {k: v for k, v in best.items() if k in ("ordering", "level_slack", "placement")}
            per_grid[name] = best
            table["per_grid"][name] = tab
    rows = []
    for t in threads:
        mb, cases = build_uneven(parts, dev, precision=precision, threads=t, per_grid=per_grid)
        sec = _time_launches(lambda: mb.launch(st.cuda_stream), repeat, st)
        nconv = sum(int(c.results()[1].sum()) for c in cases)
        rows.append({"threads": t, "seconds": sec, "converged": nconv, "pf_per_s": nconv / sec,
                     "launch": mb.info()})
        mb.close()
    table["threads"] = rows
    best = max(rows, key=lambda r: r["pf_per_s"])
    return {"threads": best["threads"], "per_grid": per_grid}, table
