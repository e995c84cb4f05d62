"""Serving loop: power-flow and N-1 requests over several grids on one GPU, continuously
batched.

The reference solves one grid at a time from Python (``ContingencyAnalysisCPP.compute``,
``TimeSeriesCPP.compute_Vs``; ``src/main.cpp:1158-1251``); it has no request loop.  This
module serves both request kinds for many grids at once through the native serving core of
the library (``pf_server_*``, ``csrc/pf_server.cpp``):

* every grid keeps its plan (pattern, ordering, pivots, phase programs), its base-case
  voltages and injections and its branch-removal coefficients across requests
  (``GridService``);
* a request is admitted as soon as it has been submitted, a stream slot is free and its device
  memory (inputs, outputs and the kernel's per-CTA working memory) fits the HBM budget, which is
  one arena allocated at start-up; admitted requests run as their own launches on their own
  streams, so work that arrives while other requests are on the GPU overlaps with them
  (continuous batching);
* each instance is solved by one CTA from its own inputs, so a request's result does not
  depend on what else is in flight.

Python only generates the arrivals, submits requests and collects finished ones.

CUDA maps streams onto ``CUDA_DEVICE_MAX_CONNECTIONS`` hardware queues (8 unless set), and
launches that share a queue wait for one another; a serving process sets it to 32 before
CUDA starts (``configure_process``) so that a short request is not queued behind a long one.
"""
import gc
import time

import numpy as np

from . import _native as nat
from .solver import Plan

PF, N1 = "pf", "n1"


def configure_process():
    """Call before the process first uses CUDA: 32 hardware queues for the streams."""
    import os

    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")


class Request:
    """One request: a power flow with scaled injections (``scale``, one factor per bus) or an
    N-1 batch (``branches``).  Results are filled in when it completes."""

    __slots__ = ("rid", "grid", "kind", "arrival", "scale", "branches", "V", "converged", "iters", "errs",
                 "t_admit", "t_done", "nbytes", "ninst")

    def __init__(self, rid, grid, kind, arrival, scale=None, branches=None):
        self.rid, self.grid, self.kind, self.arrival = rid, grid, kind, float(arrival)
        self.scale, self.branches = scale, branches
        self.V = self.converged = self.iters = self.errs = None
        self.t_admit = self.t_done = None
        self.nbytes = 0
        self.ninst = 0

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.arrival


def make_requests(grids, rate, duration, seed=0, pf_fraction=0.5, n1_min=8, n1_max=64, branches_of=None,
                  perturb=0.10):
    """Poisson arrivals at ``rate`` requests/s over ``duration`` s; each request picks a grid
    uniformly, is a power flow with injections scaled by U[1 - perturb, 1 + perturb] per bus
    (probability ``pf_fraction``) or an N-1 batch of U{n1_min..n1_max} distinct branches.
    ``grids``: name -> number of buses; ``branches_of``: name -> number of branches."""
    rng = np.random.default_rng(seed)
    names = sorted(grids)
    out, t, rid = [], 0.0, 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        g = names[rng.integers(len(names))]
        if rng.random() < pf_fraction:
            out.append(Request(rid, g, PF, t, scale=rng.uniform(1 - perturb, 1 + perturb, grids[g])))
        else:
            nb = branches_of[g]
            k = int(rng.integers(n1_min, n1_max + 1))
            out.append(Request(rid, g, N1, t, branches=np.sort(rng.choice(nb, size=min(k, nb), replace=False))))
        rid += 1
    return out


def latency_stats(done):
    lat = np.array([r.latency for r in done if r.latency is not None])
    if lat.size == 0:
        return {}
    span = max(r.t_done for r in done) - min(r.arrival for r in done)
    inst = sum(r.ninst for r in done)
    conv = sum(int(np.sum(r.converged)) for r in done if r.converged is not None)
    return {"requests": int(lat.size), "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3), "mean_ms": float(lat.mean() * 1e3),
            "max_ms": float(lat.max() * 1e3), "requests_per_s": float(lat.size / span) if span > 0 else None,
            "instances": int(inst), "converged_pf": int(conv),
            "converged_pf_per_s": float(conv / span) if span > 0 else None}


class GridService:
    """State of one served grid: its plan, base-case voltages and injections, and its N-1
    removal coefficients (reference conventions: ``ContingencyAnalysis.cpp:14-45``)."""

    def __init__(self, name, grid, precision=1, max_iter=10, tol=1e-8, **plan_options):
        self.name, self.max_iter, self.tol = name, int(max_iter), float(tol)
        Y, S = grid.get_Ybus(), grid.get_Sbus()
        sl, w, pv, pq = grid.get_slack_ids(), grid.get_slack_weights(), grid.get_pv(), grid.get_pq()
        base = Plan(Y, grid.flat_start(), S, sl, w, pv, pq, precision=0)
        V, conv, _, _ = base.solve(grid.flat_start(), S, max_iter, tol)
        if not conv:
            raise RuntimeError("base case of {} did not converge".format(name))
        del base
        self.n = int(Y.shape[0])
        self.plan = Plan(Y, V, S, sl, w, pv, pq, precision=precision, **plan_options)
        info = self.plan.info()
        self.slab, self.grid_ctas = int(info["slab_bytes"]), int(info["grid"])
        self.Vbase = nat.as_c128(V).ravel().copy()
        self.Sbase = nat.as_c128(S).ravel().copy()
        coeffs = [grid.branch_coeffs([b]) for b in range(grid.nb_powerline())]
        self.nbranch = len(coeffs)
        self.cptr = np.zeros(self.nbranch + 1, np.int32)
        rows, cols, vals = [], [], []
        for k, lst in enumerate(coeffs):
            self.cptr[k + 1] = self.cptr[k] + len(lst)
            for (r, c, y) in lst:
                rows.append(r)
                cols.append(c)
                vals.append(y)
        self.rows, self.cols = nat.as_i32(rows), nat.as_i32(cols)
        self.vals = nat.as_c128(vals).ravel()

    def n1_overrides(self, branches):
        """(solvable mask, ovr_ptr, ovr_pos, ovr_val) for the given branches, compacted."""
        branches = np.asarray(branches, np.int64)
        lens = (self.cptr[branches + 1] - self.cptr[branches]).astype(np.int64)
        cp = np.zeros(branches.size + 1, np.int32)
        np.cumsum(lens, out=cp[1:])
        starts = np.repeat(self.cptr[branches].astype(np.int64) - cp[:-1], lens)
        idx = starts + np.arange(int(cp[-1]), dtype=np.int64)
        rows, cols = np.ascontiguousarray(self.rows[idx]), np.ascontiguousarray(self.cols[idx])
        vals = np.ascontiguousarray(self.vals[idx]) if idx.size else np.zeros(1, np.complex128)
        if idx.size == 0:
            rows, cols = np.zeros(1, np.int32), np.zeros(1, np.int32)
        cap = max(int(cp[-1]), 1)
        solv = np.zeros(branches.size, np.int32)
        optr = np.zeros(branches.size + 1, np.int32)
        opos = np.zeros(cap, np.int32)
        oval = np.zeros(cap, np.complex128)
        lib = self.plan._lib
        nw = lib.pf_n1_prepare(self.plan.handle, int(branches.size), nat.ptr(cp, nat.i32p), nat.ptr(rows, nat.i32p),
                               nat.ptr(cols, nat.i32p), nat.cptr(vals), nat.ptr(solv, nat.i32p),
                               nat.ptr(optr, nat.i32p), nat.ptr(opos, nat.i32p), nat.cptr(oval), cap)
        if nw < 0:
            raise RuntimeError(nat.last_error(lib))
        ns = int(solv.sum())
        return solv.astype(bool), optr[:ns + 1].copy(), opos[:nw].copy(), oval[:nw].copy()


class NativeServer:
    """The library's serving core (``pf_server_*``) over ``GridService`` objects."""

    def __init__(self, services, hbm_budget, slots, max_instances=64, reserved_sms=None, large_request_ctas=0,
                 device_loop=False):
        self._lib = nat.load()
        self.names = list(services)
        self.index = {nm: i for i, nm in enumerate(self.names)}
        self.services = services
        self._keep = []
        grids = (nat.PfServerGrid * len(self.names))()
        for i, nm in enumerate(self.names):
            sv = services[nm]
            arrs = [sv.Vbase, sv.Sbase, sv.cptr, sv.rows, sv.cols, sv.vals]
            self._keep.append(arrs)
            grids[i] = nat.PfServerGrid(plan=sv.plan.handle, V0_ri=sv.Vbase.ctypes.data, Sbus_ri=sv.Sbase.ctypes.data,
                                        nbr=int(sv.nbranch), case_ptr=sv.cptr.ctypes.data, rows=sv.rows.ctypes.data,
                                        cols=sv.cols.ctypes.data, vals_ri=sv.vals.ctypes.data,
                                        max_iter=sv.max_iter, tol=sv.tol)
        h = nat.ctypes.c_void_p()
        nat.check(self._lib.pf_server_create(grids, len(self.names), int(hbm_budget), int(slots), int(max_instances),
                                             nat.ctypes.byref(h)), "pf_server_create", self._lib)
        self._h = h
        if reserved_sms is not None or large_request_ctas:
            self.configure(reserved_sms, large_request_ctas)
        if device_loop:
            self.set_device_loop(True)
        self._done = np.zeros(1024, np.int64)
        self.live = {}

    def configure(self, reserved_sms=None, large_request_ctas=0):
        """SM reservation for small requests (pf_server_configure): large requests are admitted
        only while their CTAs leave ``reserved_sms`` SMs free (None: an eighth of the SMs), each
        launched on at most ``large_request_ctas`` CTAs (0: no cap)."""
        if reserved_sms is None:
            import torch

            reserved_sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count // 8
        nat.check(self._lib.pf_server_configure(self._h, int(reserved_sms), int(large_request_ctas)),
                  "pf_server_configure", self._lib)

    device_loop = False

    def set_device_loop(self, enable=True, ctas_shared=0, ctas_global=0):
        """Serve through persistent device loops (pf_server_device_loop) instead of one launch per
        request; only while nothing is queued or running."""
        nat.check(self._lib.pf_server_device_loop(self._h, 1 if enable else 0, int(ctas_shared), int(ctas_global)),
                  "pf_server_device_loop", self._lib)
        self.device_loop = bool(enable)

    def submit(self, req):
        """Queues a request; its result arrays are allocated here (case order)."""
        sv = self.services[req.grid]
        if req.kind == PF:
            rows = 1
            scale = np.ascontiguousarray(req.scale, dtype=np.float64)
            br, nbr, kind = None, 0, 0
        else:
            br = np.ascontiguousarray(req.branches, dtype=np.int32)
            rows, nbr, kind, scale = br.size, br.size, 1, None
        req.V = np.empty((rows, sv.n), np.complex128)
        req.iters = np.empty(rows, np.int32)
        req.errs = np.empty(rows, np.int32)
        rc = self._lib.pf_server_submit(self._h, int(req.rid), self.index[req.grid], kind,
                                        None if scale is None else scale.ctypes.data, nbr,
                                        None if br is None else br.ctypes.data, req.V.ctypes.data,
                                        req.iters.ctypes.data, req.errs.ctypes.data)
        if rc != 0:
            return False
        req.ninst = rows
        self.live[req.rid] = (req, scale, br)
        return True

    def poll(self):
        nd = self._lib.pf_server_poll(self._h, self._done.ctypes.data, self._done.size)
        if nd < 0:
            raise RuntimeError(nat.last_error(self._lib))
        out = []
        for rid in self._done[:nd].tolist():
            req = self.live.pop(rid)[0]
            req.converged = req.errs == 0
            out.append(req)
        return out

    def latency_split(self, grid, kind, reset=False):
        """Admission wait and device time of the finished requests of one grid and kind
        (pf_server_latency_split): p50 / p99 in ms and the count."""
        out = np.zeros(5)
        nat.check(self._lib.pf_server_latency_split(self._h, self.index[grid], 1 if kind == N1 else 0,
                                                    out.ctypes.data, 1 if reset else 0),
                  "pf_server_latency_split", self._lib)
        return {"wait_p50_ms": float(out[0]), "wait_p99_ms": float(out[1]), "device_p50_ms": float(out[2]),
                "device_p99_ms": float(out[3]), "count": int(out[4])}

    def state(self):
        p, f, b = nat.ctypes.c_int(0), nat.ctypes.c_int(0), nat.ctypes.c_longlong(0)
        nat.check(self._lib.pf_server_state(self._h, nat.ctypes.byref(p), nat.ctypes.byref(f), nat.ctypes.byref(b)),
                  "pf_server_state", self._lib)
        return p.value, f.value, b.value

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pf_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ServeRun:
    """Bookkeeping of one ``PowerFlowServer.serve`` call."""

    def __init__(self):
        self.done, self.rejected = [], []
        self.peak_inflight = 0
        self.peak_bytes = 0
        self.poll_s = []     # duration of each pf_server_poll call (admissions, launches, deliveries)
        self.submit_s = []   # duration of each batch of submissions

    def host_stats(self):
        """p50/p99/max of the host loop's poll and submit calls (ms), and the time spent in
        calls longer than 1 ms."""
        out = {}
        for k, v in (("poll_ms", self.poll_s), ("submit_ms", self.submit_s)):
            a = np.asarray(v) * 1e3
            if a.size:
                out[k] = {"p50": float(np.percentile(a, 50)), "p99": float(np.percentile(a, 99)),
                          "max": float(a.max()), "calls": int(a.size), "over_1ms": int((a > 1.0).sum()),
                          "ms_in_calls_over_1ms": float(a[a > 1.0].sum())}
        return out


class PowerFlowServer:
    """Grids served from one GPU.  ``grids``: name -> GridModel."""

    def __init__(self, grids, device=None, hbm_budget=2 << 30, slots=32, precision=1, max_iter=10, tol=1e-8,
                 max_instances=64, reserved_sms=None, large_request_ctas=0, device_loop=False, **plan_options):
        self.services = {name: GridService(name, g, precision=precision, max_iter=max_iter, tol=tol, **plan_options)
                         for name, g in grids.items()}
        self.native = NativeServer(self.services, hbm_budget, slots, max_instances, reserved_sms, large_request_ctas,
                                   device_loop)

    def serve(self, requests, realtime=True, clock=time.perf_counter):
        """Serves ``requests`` (sorted by arrival).  ``realtime``: a request is submitted when
        the clock reaches its arrival time; else all are submitted at once.  Arrival and
        completion times are seconds from the start."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        run = ServeRun()
        # no cyclic garbage collection inside the loop: a full collection walks every request
        # object held so far (10^5 in a minute at 2,000 requests/s) and stalls polling for
        # milliseconds; reference counting still frees the finished requests' temporaries
        gc_on = gc.isenabled()
        gc.collect()
        gc.disable()
        try:
            self._serve_loop(reqs, run, realtime, clock)
        finally:
            if gc_on:
                gc.enable()
        self.last = run
        return run.done

    def _serve_loop(self, reqs, run, realtime, clock):
        t0 = clock()
        now = lambda: clock() - t0
        i, total = 0, len(reqs)
        while len(run.done) + len(run.rejected) < total:
            t = now()
            i0 = i
            while i < total and (not realtime or reqs[i].arrival <= t):
                r = reqs[i]
                if not realtime:
                    r.arrival = t
                r.t_admit = t  # handed to the serving core (queued there until admitted)
                if not self.native.submit(r):
                    r.t_done = now()
                    run.rejected.append(r)
                i += 1
            t1 = now()
            if i > i0:
                run.submit_s.append(t1 - t)
            fin = self.native.poll()
            run.poll_s.append(now() - t1)
            if fin:
                td = now()
                for r in fin:
                    r.t_done = td
                run.done.extend(fin)
            pend, infl, nbytes = self.native.state()
            run.peak_inflight = max(run.peak_inflight, infl)
            run.peak_bytes = max(run.peak_bytes, nbytes)
            if not fin and infl == 0 and pend == 0 and i < total:
                wait = reqs[i].arrival - now()
                if wait > 0:
                    time.sleep(min(wait, 1e-3))

    def solve_alone(self, req):
        """The request on an otherwise idle GPU (same path), for comparisons."""
        r = Request(req.rid, req.grid, req.kind, 0.0, scale=req.scale, branches=req.branches)
        self.serve([r], realtime=False)
        return r
