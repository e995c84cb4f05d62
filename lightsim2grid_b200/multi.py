"""Uneven-size batched N-1: contingencies of grids of different sizes in one persistent launch.

The reference runs one ``ContingencyAnalysis`` per grid, one case after the other
(``src/batch_algorithm/ContingencyAnalysis.cpp:166-233``).  Here the cases of several grids
form one job list: a CTA takes the next job, loads that job's plan (its segment) into shared
memory when it differs from the previous one, and solves the instance.  The launch allocates
nothing and is captured once in a CUDA graph (``MultiBatch.graph``); the jobs are ordered
costliest grid first so that the small grids' jobs fill the tail.

``python -m lightsim2grid_b200.multi`` measures the 4,096-outage mix over the 118-, 1,354- and
2,848-bus synthetic grids (proportion 1:2:5, mixed precision).
"""
import argparse
import json
import sys
import time

import numpy as np

from . import _native as nat
from .solver import Plan


class MultiBatch:
    """One launch over several (plan, device batch) segments and a job list (device arrays)."""

    def __init__(self, plans, batches, job_seg, job_first, job_count, keep=()):
        self._lib = nat.load()
        self.plans = list(plans)
        self.keep = list(keep)  # device tensors the batches and jobs point to
        self._job = (job_seg, job_first, job_count)
        arr = (nat.ctypes.c_void_p * len(plans))(*[p.handle for p in plans])
        barr = (nat.PfDeviceBatch * len(batches))(*batches)
        h = nat.ctypes.c_void_p()
        rc = self._lib.pf_multi_create(arr, barr, len(plans), job_seg.data_ptr(), job_first.data_ptr(),
                                       job_count.data_ptr(), int(job_seg.numel()), nat.ctypes.byref(h))
        nat.check(rc, "pf_multi_create", self._lib)
        self._h = h
        self.graph = None

    def launch(self, stream):
        nat.check(self._lib.pf_multi_launch(self._h, stream), "pf_multi_launch", self._lib)

    def info(self):
        t, g = nat.ctypes.c_int(0), nat.ctypes.c_int(0)
        sm, sc = nat.ctypes.c_longlong(0), nat.ctypes.c_longlong(0)
        nat.check(self._lib.pf_multi_info(self._h, nat.ctypes.byref(t), nat.ctypes.byref(g), nat.ctypes.byref(sm),
                                          nat.ctypes.byref(sc)), "pf_multi_info", self._lib)
        return {"threads": t.value, "grid": g.value, "shared_bytes": sm.value, "scratch_bytes": sc.value}

    def capture(self):
        """Captures one launch in a CUDA graph (after a launch outside capture has set the
        kernel's attributes); replay with ``self.graph.replay()``."""
        import torch

        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.launch(s.cuda_stream)
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            self.launch(s.cuda_stream)
        torch.cuda.synchronize()
        self.graph = g
        return g

    def close(self):
        self.graph = None
        if getattr(self, "_h", None):
            self._lib.pf_multi_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GridCases:
    """One grid's part of an uneven batch: its plan, base state and the compacted, solvable
    N-1 instances for the drawn branches (islanded outages are skipped, as the reference's
    check_invertible does, ContingencyAnalysis.cpp:14-45)."""

    def __init__(self, name, grid, branches, device, precision=1, max_iter=10, tol=1e-8, base_state=None,
                 **plan_options):
        import torch

        self.name, self.grid, self.branches = name, grid, np.asarray(branches, np.int64)
        Y, S = grid.get_Ybus(), grid.get_Sbus()
        sl, w, pv, pq = grid.get_slack_ids(), grid.get_slack_weights(), grid.get_pv(), grid.get_pq()
        if base_state is None:
            base = Plan(Y, grid.flat_start(), S, sl, w, pv, pq, precision=0)
            V, conv, _, _ = base.solve(grid.flat_start(), S, max_iter, tol)
            if not conv:
                raise RuntimeError("base case of {} did not converge".format(name))
            del base
        else:  # (base-case voltages, injections) of an earlier GridCases of the same grid
            V, S = base_state
        self.Vbase, self.Sbase = nat.as_c128(V).ravel().copy(), nat.as_c128(S).ravel().copy()
        self.plan = Plan(Y, V, S, sl, w, pv, pq, precision=precision, **plan_options)
        self.n = int(Y.shape[0])
        coeffs = [grid.branch_coeffs([int(b)]) for b in self.branches]
        cp = np.zeros(len(coeffs) + 1, np.int32)
        rows, cols, vals = [], [], []
        for k, lst in enumerate(coeffs):
            cp[k + 1] = cp[k] + len(lst)
            for (r, c, y) in lst:
                rows.append(r)
                cols.append(c)
                vals.append(y)
        rows, cols, vals = nat.as_i32(rows), nat.as_i32(cols), nat.as_c128(vals).ravel()
        cap = max(int(cp[-1]), 1)
        solv = np.zeros(len(coeffs), np.int32)
        optr = np.zeros(len(coeffs) + 1, np.int32)
        opos, oval = np.zeros(cap, np.int32), np.zeros(cap, np.complex128)
        lib = self.plan._lib
        nw = lib.pf_n1_prepare(self.plan.handle, len(coeffs), nat.ptr(cp, nat.i32p), nat.ptr(rows, nat.i32p),
                               nat.ptr(cols, nat.i32p), nat.cptr(vals), nat.ptr(solv, nat.i32p),
                               nat.ptr(optr, nat.i32p), nat.ptr(opos, nat.i32p), nat.cptr(oval), cap)
        if nw < 0:
            raise RuntimeError(nat.last_error(lib))
        self.solvable = solv.astype(bool)
        ns = self.ninst = int(solv.sum())
        # the instances hardest first (power mismatch of the outage at the start voltages)
        self.order = np.zeros(max(ns, 1), np.int32)
        rc = lib.pf_n1_order(self.plan.handle, ns, nat.ptr(optr, nat.i32p), nat.ptr(opos, nat.i32p), nat.cptr(oval),
                             nat.cptr(self.Vbase), nat.ptr(self.order, nat.i32p))
        if rc != 0:
            raise RuntimeError(nat.last_error(lib))
        self.order = self.order[:ns]
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
        self.dev = dict(V0=t(self.Vbase.view(np.float64)), S=t(self.Sbase.view(np.float64)), optr=t(optr[:ns + 1]),
                        opos=t(opos[:max(nw, 1)]), oval=t(oval[:max(nw, 1)].view(np.float64)),
                        V=torch.zeros(max(ns, 1) * self.n * 2, dtype=torch.float64, device=device),
                        it=torch.zeros(max(ns, 1), dtype=torch.int32, device=device),
                        er=torch.full((max(ns, 1),), -1, dtype=torch.int32, device=device))
        d = self.dev
        self.batch = nat.PfDeviceBatch(n_inst=ns, V0=d["V0"].data_ptr(), v0_stride=0, Sbus=d["S"].data_ptr(),
                                       sbus_stride=0, ovr_ptr=d["optr"].data_ptr(), ovr_pos=d["opos"].data_ptr(),
                                       ovr_val=d["oval"].data_ptr(), max_iter=max_iter, tol=tol, chain=0,
                                       job_first=0, job_count=0, njobs=0, Vout=d["V"].data_ptr(),
                                       iters=d["it"].data_ptr(), errs=d["er"].data_ptr())

    def results(self):
        """(V[ncases, n], converged[ncases], iters, errs) in drawn-branch order; islanded and
        diverged cases have V = 0 and converged = False."""
        k = len(self.branches)
        V = np.zeros((k, self.n), np.complex128)
        conv = np.zeros(k, bool)
        it = np.zeros(k, np.int32)
        er = np.full(k, -1, np.int32)
        if self.ninst:
            Vd = self.dev["V"].cpu().numpy().view(np.complex128).reshape(-1, self.n)[:self.ninst]
            itd, erd = self.dev["it"].cpu().numpy()[:self.ninst], self.dev["er"].cpu().numpy()[:self.ninst]
            idx = np.flatnonzero(self.solvable)
            V[idx] = np.where((erd == 0)[:, None], Vd, 0.0)
            conv[idx] = erd == 0
            it[idx], er[idx] = itd, erd
        return V, conv, it, er


def build_uneven(parts, device, precision=1, max_iter=10, tol=1e-8, per_grid=None, **plan_options):
    """``parts``: list of (name, GridModel, drawn branches).  Returns (MultiBatch, [GridCases]).
    Jobs: one per solvable instance, grids ordered by decreasing size (costliest first), each
    grid's instances hardest first (pf_n1_order).  ``per_grid``: name -> plan options of that
    grid (its schedule: elimination order, level slack, placement), over ``plan_options``."""
    import torch

    per_grid = per_grid or {}
    cases = [GridCases(nm, g, br, device, precision, max_iter, tol, **dict(plan_options, **per_grid.get(nm, {})))
             for nm, g, br in parts]
    order = sorted(range(len(cases)), key=lambda i: -cases[i].plan.info()["nnz_lu"])
    seg, first = [], []
    for i in order:
        seg.extend([i] * cases[i].ninst)
        first.extend(cases[i].order.tolist())
    t = lambda a: torch.from_numpy(np.asarray(a, np.int32)).to(device)
    js, jf, jc = t(seg if seg else [0]), t(first if first else [0]), t(np.ones(max(len(seg), 1), np.int32))
    mb = MultiBatch([c.plan for c in cases], [c.batch for c in cases], js[:len(seg)], jf[:len(seg)],
                    jc[:len(seg)], keep=[js, jf, jc])
    return mb, cases


def draw_outages(grids_counts, seed=0):
    """Draws outages per grid: ``grids_counts`` = list of (name, GridModel, count); without
    replacement while the grid has enough branches, with replacement beyond."""
    rng = np.random.default_rng(seed)
    out = []
    for name, g, k in grids_counts:
        nb = g.nb_powerline()
        br = rng.choice(nb, size=k, replace=k > nb)
        out.append((name, g, np.sort(br)))
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description="uneven-size batched N-1 in one graph-captured launch")
    ap.add_argument("--total", type=int, default=4096)
    ap.add_argument("--repeat", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--threads", type=int, default=0,
                    help="0: thread count and per-grid schedules autotuned on a sample of the mix")
    ap.add_argument("--seed", type=int, default=4096)
    args = ap.parse_args(argv)
    import torch

    from . import synthetic

    dev = torch.device("cuda:0")
    names, weights = ("grid118", "grid1354", "grid2848"), (1, 2, 5)
    counts = [args.total * w // sum(weights) for w in weights]
    counts[-1] += args.total - sum(counts)
    grids = [(nm, synthetic.make_named_grid(nm)[0], k) for nm, k in zip(names, counts)]
    tuning = None
    best = {"threads": args.threads}
    if args.threads <= 0:
        from .autotune import tune_uneven

        sample = draw_outages([(nm, g, max(8, k // 8)) for nm, g, k in grids], args.seed + 1)
        best, tuning = tune_uneven(sample, precision=1)
    mb, cases = build_uneven(draw_outages(grids, args.seed), dev, precision=1, **best)
    st = torch.cuda.current_stream()
    for _ in range(args.warmup):
        mb.launch(st.cuda_stream)
    torch.cuda.synchronize()
    g = mb.capture()
    for _ in range(2):
        g.replay()
    torch.cuda.synchronize()
    flush = torch.empty(256 << 20 >> 2, dtype=torch.float32, device=dev)
    times = []
    for _ in range(args.repeat):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g.replay()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) * 1e-3)
    conv = {c.name: int(c.results()[1].sum()) for c in cases}
    tot = sum(conv.values())
    out = {"workload": "uneven N-1: {} outages over {} in proportion 1:2:5, mixed precision, one graph-captured "
                       "launch".format(args.total, "/".join(names)),
           "cases": {c.name: len(c.branches) for c in cases}, "solvable": {c.name: c.ninst for c in cases},
           "converged": conv, "ms": [1e3 * t for t in times], "converged_pf_per_s": tot / float(np.mean(times)),
           "launch": mb.info(), "autotune": tuning}
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
