"""Serving loop: power-flow and N-1 requests over several grids on one GPU, continuously
batched.

The reference solves one grid at a time from Python (``ContingencyAnalysisCPP.compute``,
``TimeSeriesCPP.compute_Vs``; ``src/main.cpp:1158-1251``); it has no request loop.  This
module serves both request kinds for many grids at once:

* every grid keeps its plan (pattern, ordering, pivots, phase programs), its base-case
  voltages and its Ybus on the device across requests (``GridService``);
* a request is admitted as soon as it has arrived, a stream slot is free and its device
  memory (inputs, outputs and the kernel's per-CTA working memory) fits the HBM budget;
  admitted requests run as their own launches on their own streams, so work that arrives
  while other requests are on the GPU overlaps with them (continuous batching);
* each instance is solved by one CTA from its own inputs, so a request's result does not
  depend on what else is in flight.

``Dispatcher`` holds the admission policy and bookkeeping and runs against any executor;
``CudaExecutor`` launches through the C ABI (``pf_batch_device_scratch``).

CUDA maps streams onto ``CUDA_DEVICE_MAX_CONNECTIONS`` hardware queues (8 unless set), and
launches that share a queue wait for one another; a serving process sets it to 32 before
CUDA starts (``configure_process``) so that a short request is not queued behind a long one.
"""
import collections
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


class Dispatcher:
    """Admission and bookkeeping.  FIFO: the oldest waiting request is admitted first, when a
    slot is free and ``executor.bytes_needed(req)`` fits in what the budget has left; a
    request larger than the whole budget is rejected (``errs`` = None, ``t_done`` set)."""

    def __init__(self, executor, hbm_budget, slots):
        self.ex = executor
        self.budget = int(hbm_budget)
        self.slots = int(slots)
        self.in_use = 0
        self.pending = collections.deque()
        self.inflight = {}
        self.done = []
        self.rejected = []
        self.peak_bytes = 0
        self.peak_inflight = 0
        self.host_s = {"submit": 0.0, "launch": 0.0, "poll": 0.0}  # host seconds spent per step

    def submit(self, req):
        req.nbytes = self.ex.bytes_needed(req)
        if req.nbytes > self.budget:
            self.rejected.append(req)
            return
        self.pending.append(req)

    def admit(self, now):
        n = 0
        while self.pending and len(self.inflight) < self.slots:
            req = self.pending[0]
            if self.in_use + req.nbytes > self.budget or not self.ex.reserve(req):
                break
            self.pending.popleft()
            self.in_use += req.nbytes
            req.t_admit = now
            self.inflight[req.rid] = req
            self.ex.launch(req)
            n += 1
        self.peak_bytes = max(self.peak_bytes, self.in_use)
        self.peak_inflight = max(self.peak_inflight, len(self.inflight))
        return n

    def complete(self, now):
        n = 0
        for rid in self.ex.poll():
            req = self.inflight.pop(rid)
            self.in_use -= req.nbytes
            req.t_done = now()
            self.done.append(req)
            n += 1
        return n

    def run(self, requests, clock=time.perf_counter, realtime=True):
        """Serves ``requests`` (sorted by arrival).  ``realtime``: a request is submitted when
        the clock reaches its arrival time; else all are submitted at once.  Arrival and
        completion times are seconds from the start."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        t0 = clock()
        now = lambda: clock() - t0
        i, total = 0, len(reqs)
        while len(self.done) + len(self.rejected) < total:
            t = now()
            h0 = clock()
            while i < total and (not realtime or reqs[i].arrival <= t):
                if not realtime:
                    reqs[i].arrival = t
                self.submit(reqs[i])
                i += 1
            h1 = clock()
            self.admit(t)
            h2 = clock()
            finished = self.complete(now)
            h3 = clock()
            self.host_s["submit"] += h1 - h0
            self.host_s["launch"] += h2 - h1
            self.host_s["poll"] += h3 - h2
            if not finished and not self.inflight and not self.pending and i < total:
                # idle until the next arrival
                wait = reqs[i].arrival - now()
                if wait > 0:
                    time.sleep(min(wait, 1e-3))
        for req in self.rejected:
            req.t_done = now()
        return self.done


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
    """Device-resident state of one grid: its plan, base-case voltages and injections, and its
    N-1 removal coefficients (reference conventions: ``ContingencyAnalysis.cpp:14-45``)."""

    def __init__(self, name, grid, device, precision=1, max_iter=10, tol=1e-8, **plan_options):
        import torch

        self.name, self.device, self.max_iter, self.tol = name, device, int(max_iter), float(tol)
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
        self.Vbase_dev = torch.from_numpy(self.Vbase.view(np.float64).copy()).to(device)
        self.Sbase_dev = torch.from_numpy(self.Sbase.view(np.float64).copy()).to(device)
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


def _align(n, a=256):
    return (int(n) + a - 1) // a * a


class DeviceArena:
    """First-fit allocator over one device allocation of ``nbytes`` (the serving budget):
    every request's inputs, outputs and kernel working memory live in one region of it, so
    serving allocates no device memory after start-up."""

    def __init__(self, nbytes, device):
        import torch

        self.size = _align(nbytes)
        self.buf = torch.empty(self.size, dtype=torch.uint8, device=device)
        self.base = self.buf.data_ptr()
        self.holes = [(0, self.size)]  # (offset, size), sorted by offset, coalesced

    def alloc(self, n):
        n = _align(n)
        for i, (o, sz) in enumerate(self.holes):
            if sz >= n:
                if sz == n:
                    del self.holes[i]
                else:
                    self.holes[i] = (o + n, sz - n)
                return o
        return None

    def release(self, o, n):
        n = _align(n)
        h = self.holes
        i = 0
        while i < len(h) and h[i][0] < o:
            i += 1
        h.insert(i, (o, n))
        if i + 1 < len(h) and h[i][0] + h[i][1] == h[i + 1][0]:
            h[i] = (h[i][0], h[i][1] + h[i + 1][1])
            del h[i + 1]
        if i > 0 and h[i - 1][0] + h[i - 1][1] == h[i][0]:
            h[i - 1] = (h[i - 1][0], h[i - 1][1] + h[i][1])
            del h[i]

    def free_bytes(self):
        return sum(sz for _, sz in self.holes)


class CudaExecutor:
    """Runs each admitted request as its own launch on its own stream slot.  A request's
    device region (from the arena) holds its inputs, outputs and the kernel's working memory;
    inputs are copied from the slot's pinned host buffer, results back to the slot's pinned
    output buffer; ``poll`` reports finished requests.  Pinned buffers are sized once for the
    largest grid and ``max_instances`` instances."""

    def __init__(self, services, device, slots, arena, max_instances=64):
        import torch

        self.torch = torch
        self.sv = services
        self.device = device
        self.arena = arena
        self.max_k = int(max_instances)
        nmax = max(s.n for s in services.values())
        in_bytes = max(nmax * 16, self.max_k * 4 * 24 + 8 * (self.max_k + 1)) + 1024
        out_bytes = self.max_k * nmax * 16 + 16 * self.max_k + 1024
        self.free = [(torch.cuda.Stream(device), torch.empty(in_bytes, dtype=torch.uint8, pin_memory=True),
                      torch.empty(out_bytes, dtype=torch.uint8, pin_memory=True)) for _ in range(slots)]
        # job lists (instance j = job j) shared by every launch: read only
        self.jf = torch.arange(self.max_k, dtype=torch.int32, device=device)
        self.jc = torch.ones(self.max_k, dtype=torch.int32, device=device)
        self.active = {}
        self.prepared = {}

    def bytes_needed(self, req):
        """Region layout: [scratch | outputs (V, iters, errs) | inputs]; returns its size."""
        s = self.sv[req.grid]
        if req.kind == PF:
            k, ov = 1, None
            inputs = [_align(s.n * 16)]
        else:
            ov = s.n1_overrides(req.branches)
            k = int(ov[0].sum())
            inputs = [_align(4 * (k + 1)), _align(4 * max(ov[2].size, 1)), _align(16 * max(ov[3].size, 1))]
        if k > self.max_k:
            raise ValueError("request {} has {} instances (at most {})".format(req.rid, k, self.max_k))
        req.ninst = k
        ctas = max(1, min(k, s.grid_ctas))
        scratch = _align(s.plan._lib.pf_scratch_bytes(s.plan.handle, ctas)) if k else 0
        outs = _align(k * s.n * 16 + 8 * k)
        self.prepared[req.rid] = [ov, scratch, outs, inputs, None]
        return scratch + outs + sum(inputs)

    def reserve(self, req):
        prep = self.prepared[req.rid]
        o = self.arena.alloc(req.nbytes)
        if o is None:
            return False
        prep[4] = o
        return True

    def launch(self, req):
        torch = self.torch
        s = self.sv[req.grid]
        ov, scratch, outs, inputs, off = self.prepared.pop(req.rid)
        st, pin_in, pin_out = self.free.pop()
        k = req.ninst
        buf, base = self.arena.buf, self.arena.base
        with torch.cuda.stream(st):
            if k == 0:
                ev = torch.cuda.Event()
                ev.record(st)
                self.active[req.rid] = (req, (st, pin_in, pin_out), ev, off)
                return
            o_scr, o_out = off, off + scratch
            o_in = o_out + outs
            pin = pin_in.numpy()

            def upload(arr, size):
                nonlocal o_in
                b = np.ascontiguousarray(arr).view(np.uint8).ravel()
                p0 = o_in - (off + scratch + outs)
                pin[p0:p0 + b.size] = b
                buf[o_in:o_in + b.size].copy_(pin_in[p0:p0 + b.size], non_blocking=True)
                ptr = base + o_in
                o_in += size
                return ptr

            if req.kind == PF:
                sbus = upload((s.Sbase * req.scale).astype(np.complex128), inputs[0])
                optr_d = opos_d = oval_d = 0
            else:
                solv, optr, opos, oval = ov
                optr_d = upload(optr, inputs[0])
                opos_d = upload(opos if opos.size else np.zeros(1, np.int32), inputs[1])
                oval_d = upload(oval if oval.size else np.zeros(1, np.complex128), inputs[2])
                sbus = s.Sbase_dev.data_ptr()
            vo = base + o_out
            b = nat.PfDeviceBatch(n_inst=k, V0=s.Vbase_dev.data_ptr(), v0_stride=0, Sbus=sbus, sbus_stride=0,
                                  ovr_ptr=optr_d, ovr_pos=opos_d, ovr_val=oval_d, max_iter=s.max_iter, tol=s.tol,
                                  chain=0, job_first=self.jf.data_ptr(), job_count=self.jc.data_ptr(),
                                  njobs=k, Vout=vo, iters=vo + k * s.n * 16, errs=vo + k * s.n * 16 + 4 * k)
            rc = s.plan._lib.pf_batch_device_scratch(s.plan.handle, nat.ctypes.byref(b), base + o_scr, scratch,
                                                     st.cuda_stream)
            if rc != 0:
                raise RuntimeError(nat.last_error(s.plan._lib))
            nout = k * s.n * 16 + 8 * k
            pin_out[:nout].copy_(buf[o_out:o_out + nout], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(st)
        self.active[req.rid] = (req, (st, pin_in, pin_out), ev, off)

    def poll(self):
        fin = []
        for rid, (req, slot, ev, off) in list(self.active.items()):
            if not ev.query():
                continue
            s = self.sv[req.grid]
            k = req.ninst
            if k == 0:
                req.V = np.zeros((0, s.n), np.complex128)
                req.converged = np.zeros(0, bool)
                req.iters = req.errs = np.zeros(0, np.int32)
            else:
                raw = slot[2].numpy()
                nv = k * s.n * 16
                req.V = raw[:nv].view(np.complex128).reshape(k, s.n).copy()
                req.iters = raw[nv:nv + 4 * k].view(np.int32).copy()
                req.errs = raw[nv + 4 * k:nv + 8 * k].view(np.int32).copy()
                req.converged = req.errs == 0
                req.V[~req.converged] = 0.0
            self.arena.release(off, req.nbytes)
            del self.active[rid]
            self.free.append(slot)
            fin.append(rid)
        return fin


class PowerFlowServer:
    """Grids served from one GPU.  ``grids``: name -> GridModel."""

    def __init__(self, grids, device=None, hbm_budget=2 << 30, slots=32, precision=1, max_iter=10, tol=1e-8,
                 max_instances=64, **plan_options):
        import torch

        self.device = torch.device("cuda", 0) if device is None else torch.device(device)
        self.services = {name: GridService(name, g, self.device, precision=precision, max_iter=max_iter, tol=tol,
                                           **plan_options) for name, g in grids.items()}
        self.hbm_budget, self.slots, self.max_instances = int(hbm_budget), int(slots), int(max_instances)

    def executor(self):
        if getattr(self, "_ex", None) is None:
            self.arena = DeviceArena(self.hbm_budget, self.device)
            self._ex = CudaExecutor(self.services, self.device, self.slots, self.arena, self.max_instances)
        return self._ex

    def serve(self, requests, realtime=True):
        ex = self.executor()
        d = Dispatcher(ex, self.hbm_budget, self.slots)
        done = d.run(requests, realtime=realtime)
        self.last = d
        return done

    def solve_alone(self, req):
        """The request on an otherwise idle GPU (same launch path), for comparisons."""
        r = Request(req.rid, req.grid, req.kind, 0.0, scale=req.scale, branches=req.branches)
        self.serve([r], realtime=False)
        return r
