#!/usr/bin/env python
"""Benchmark: converged AC power flows per second of a batched N-1 analysis on the seeded
synthetic 2,848-bus grid (3,776 branches, 500 PV buses), tolerance 1e-8 pu.

One step = every single-branch outage of the grid that keeps it connected (islanded
outages are skipped exactly as the reference's check_invertible does), solved by one
persistent kernel launch.  Each outage starts from the base-case solution (the grid state
a security analysis is run from).  Only converged power flows are counted.

Arms:
  (default)          this engine; ``value`` = mixed form (FP32 LU, FP64 mismatch/update)
                     with inputs resident in HBM, plus the FP64 form, the host-API ``e2e``
                     figure, the roofline of the kernel, the CPU oracle baseline (all host
                     threads and one core) and each result's distance to the FP64 oracle.
                     Extra keys measure the other workloads: ``config1`` (118-bus FP64 N-1),
                     ``config2`` (8,760-snapshot time series, FP64 and mixed, device and host
                     API, against the oracle's chains), ``config3`` (4,096 outages over three
                     grids in one graph-captured launch, autotuned schedules, flags against
                     the oracle) and ``serve`` (config 4).
  --impl reference   the CPU restatement of the reference's loop (oracle/, the reference
                     itself cannot be built here) on all host threads, same metric and the
                     same outage set.

The ``serve`` object is the serving leg: Poisson arrivals (2,000 requests/s, 60 s by default)
over six synthetic grids of 14 to 6,515 buses, half single power flows with perturbed
injections and half N-1 batches of 8 to 64 outages, continuously batched on the GPU; it
reports p50/p99 latency and throughput.

Multi-GPU (torchrun): every rank runs the whole batch on its own GPU (replicas; the cases
are independent and nothing is exchanged); value = total converged PFs / max-over-ranks time.

Profiling mode: ``python bench.py case [--grid G --cases N --precision P ...]`` runs one N-1
batch through ``pf_batch_device`` (``--warmup`` untimed and ``--repeat`` timed launches) and
prints the CUDA-event times, the per-phase cycle shares and a phase trace: the command the
ncu summaries under profiles/ were captured with.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

# the serving leg runs one stream per in-flight request: give them 32 hardware queues
# (must be set before CUDA starts)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "converged PFs/s (N-1, 2848-bus, 1e-8 pu) mixed vs FP64 GPU; serve p50/p99 ms"
GRID = "grid2848"
TOL = 1e-8
MAX_ITER = 10
WORKLOAD = ("N-1 all single-branch outages, synthetic grid2848 (2848 buses, 3776 branches, 500 PV; geometric "
            "topology, seed 2848), start = base-case solution, tol 1e-8 pu, max_iter 10")


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _profile_figures():
    """Per instance-iteration figures of the mixed kernel from the committed ncu summary:
    DRAM bytes, L2 bytes, shared-memory wavefronts, issue-active and the capture's plan."""
    path = os.path.join(ROOT, "profiles", "nr_batch_kernel_n1_grid2848.md")
    out = {}
    try:
        for line in open(path):
            if ":" in line and line.split(":")[0].strip() in (
                    "traffic_bytes_per_instance_iteration", "l2_bytes_per_instance_iteration",
                    "smem_wavefronts_per_instance_iteration", "smem_wavefronts_per_sm_cycle",
                    "issue_active_fraction", "profile_levels_refactor"):
                k, v = line.split(":", 1)
                out[k.strip()] = float(v)
    except Exception:
        pass
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
            return
        # nvidia-smi takes a while to start: wait for its first sample, keep only later ones
        t_end = time.time() + 5.0
        while not self.lines and time.time() < t_end and self.proc.poll() is None:
            time.sleep(0.005)
        self.first = len(self.lines)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        first = getattr(self, "first", 0)
        for ln in (self.lines[first:] if len(self.lines) > first else self.lines):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _grid(name=GRID):
    from lightsim2grid_b200 import synthetic

    return synthetic.make_named_grid(name)[0]


def _n1_arrays(g, branches=None):
    """Removal coefficients of the single-branch outages (every branch by default) as flat
    arrays: (coefficient lists, case_ptr, rows, cols, values)."""
    branches = range(g.nb_powerline()) if branches is None else branches
    coeffs = [g.branch_coeffs([int(b)]) for b in branches]
    cp = np.zeros(len(coeffs) + 1, np.int32)
    rows, cols, vals = [], [], []
    for k, lst in enumerate(coeffs):
        cp[k + 1] = cp[k] + len(lst)
        for (r, c, y) in lst:
            rows.append(r)
            cols.append(c)
            vals.append(y)
    return coeffs, cp, np.asarray(rows, np.int32), np.asarray(cols, np.int32), np.asarray(vals, np.complex128)


def _algorithmic_bytes(info, iters, b):
    """Bytes one launch must move at minimum (north-star per-unit figure x units).

    Per instance-iteration: mismatch + J fill 16n (V) + 16n (Sbus) + 8m (F) + b zJ (J);
    refactorisation b (zJ + zLU); substitutions b zLU + 16m; update 8m + 48n.
    Per instance once: V0 read + initial mismatch 32n + 8m, V written 16n.
    """
    n, m, zJ, zLU = info["n"], info["m"], info["nnz_j"], info["nnz_lu"]
    per_it = 80 * n + 32 * m + 2 * b * (zJ + zLU)
    per_inst = 64 * n + 8 * m
    return float(np.sum(iters) * per_it + len(iters) * per_inst), per_it


def _launch_bound(threads):
    """The Newton kernel's launch-bound template argument for a thread count (the library runs
    the 512-, 640- or 768-thread variant)."""
    return 768 if threads > 640 else (640 if threads > 512 else 512)


def _dv(a, b):
    """Per row: max over buses of max(|d|V||, |d angle|) (pu, rad)."""
    dm = np.abs(np.abs(a) - np.abs(b))
    da = np.abs(np.angle(a) - np.angle(b))
    da = np.minimum(da, 2 * np.pi - da)
    return np.maximum(dm, da).max(axis=-1)


def _err_stats(dv):
    if dv.size == 0:
        return {"max": None, "p99": None, "median": None, "count": 0}
    return {"max": float(dv.max()), "p99": float(np.percentile(dv, 99)), "median": float(np.median(dv)),
            "count": int(dv.size)}


def _host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def _cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return None


def _dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class N1Device:
    """The N-1 batch of a grid resident on the device for pf_batch_device: the solvable outages
    (pf_n1_prepare's islanding check) as instances, jobs hardest first (pf_n1_order)."""

    def __init__(self, g, Vn, dev, precision, branches=None, case_order=False, **plan_options):
        import torch
        from lightsim2grid_b200 import Plan, _native as nat

        self.nat = nat
        Y, S = g.get_Ybus(), g.get_Sbus()
        sl, w, pv, pq = g.get_slack_ids(), g.get_slack_weights(), g.get_pv(), g.get_pq()
        self.n = n = g.n_bus
        self.coeffs, cp, rows, cols, vals = _n1_arrays(g, branches)
        self.plan = plan = Plan(Y, Vn, S, sl, w, pv, pq, precision=precision, **plan_options)
        lib = self.lib = plan._lib
        ncases = len(self.coeffs)
        solv = np.zeros(ncases, np.int32)
        optr = np.zeros(ncases + 1, np.int32)
        cap = max(int(cp[-1]), 1)
        opos = np.zeros(cap, np.int32)
        oval = np.zeros(cap, np.complex128)
        nw = lib.pf_n1_prepare(plan.handle, ncases, nat.ptr(cp, nat.i32p), nat.ptr(rows, nat.i32p),
                               nat.ptr(cols, nat.i32p), nat.cptr(vals), nat.ptr(solv, nat.i32p),
                               nat.ptr(optr, nat.i32p), nat.ptr(opos, nat.i32p), nat.cptr(oval), cap)
        assert nw >= 0, nat.last_error(lib)
        self.solvable = np.flatnonzero(solv)
        ns = self.ns = int(solv.sum())
        self.prep = (solv, optr, opos, oval, nw)
        if case_order or plan.dc or plan.fdpf:
            order = np.arange(max(ns, 1), dtype=np.int32)
        else:
            order = np.zeros(max(ns, 1), np.int32)
            V0c = nat.as_c128(Vn).ravel()
            assert lib.pf_n1_order(plan.handle, ns, nat.ptr(optr, nat.i32p), nat.ptr(opos, nat.i32p),
                                   nat.cptr(oval), nat.cptr(V0c), nat.ptr(order, nat.i32p)) == 0, nat.last_error(lib)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        self.bufs = bufs = dict(
            V0=t(nat.as_c128(Vn).ravel().view(np.float64)), S=t(nat.as_c128(S).ravel().view(np.float64)),
            optr=t(optr[:ns + 1]), opos=t(opos[:max(nw, 1)]), oval=t(oval[:max(nw, 1)].view(np.float64)),
            jf=t(order[:max(ns, 1)]), jc=t(np.ones(max(ns, 1), np.int32)),
            Vout=torch.zeros(max(ns, 1) * n * 2, dtype=torch.float64, device=dev),
            it=torch.zeros(max(ns, 1), dtype=torch.int32, device=dev),
            er=torch.zeros(max(ns, 1), dtype=torch.int32, device=dev))
        self.batch = nat.PfDeviceBatch(
            n_inst=ns, V0=bufs["V0"].data_ptr(), v0_stride=0, Sbus=bufs["S"].data_ptr(), sbus_stride=0,
            ovr_ptr=bufs["optr"].data_ptr(), ovr_pos=bufs["opos"].data_ptr(), ovr_val=bufs["oval"].data_ptr(),
            max_iter=MAX_ITER, tol=TOL, chain=0, job_first=bufs["jf"].data_ptr(), job_count=bufs["jc"].data_ptr(),
            njobs=ns, Vout=bufs["Vout"].data_ptr(), iters=bufs["it"].data_ptr(), errs=bufs["er"].data_ptr())

    def launch(self, stream):
        rc = self.lib.pf_batch_device(self.plan.handle, self.nat.ctypes.byref(self.batch), stream)
        assert rc == 0, self.nat.last_error(self.lib)

    def results(self):
        """(V[ns, n], iters, errs) of the solvable instances, in case order of the solvable cases."""
        V = self.bufs["Vout"].cpu().numpy().view(np.complex128).reshape(-1, self.n)[:self.ns]
        return V, self.bufs["it"].cpu().numpy()[:self.ns], self.bufs["er"].cpu().numpy()[:self.ns]


def _time_device(launch, stream, K, W, flush, barrier=None):
    """W untimed launches, then K launches each timed with CUDA events on `stream`, L2 flushed
    (a write larger than L2) before each; returns seconds per launch."""
    import torch

    for _ in range(W):
        launch()
    torch.cuda.synchronize()
    if barrier:
        barrier()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    for k in range(K):
        flush.zero_()
        evs[k][0].record(stream)
        launch()
        evs[k][1].record(stream)
    torch.cuda.synchronize()
    if barrier:
        barrier()
    torch.cuda.synchronize()
    return [a.elapsed_time(e) * 1e-3 for a, e in evs]


# ----------------------------------------------------------------------------- config legs

def _config1(dev, stream, flush, K, W, threads):
    """Config 1: N-1 over every branch of the 118-bus grid, FP64, device-resident inputs; the
    host-API figure and the oracle's flags and voltages beside it."""
    from lightsim2grid_b200 import GPUNRSolverSingleSlack
    from oracle.oracle import ContingencyBatch

    g = _grid("grid118")
    base = GPUNRSolverSingleSlack()
    assert base.compute_pf(g.get_Ybus(), g.flat_start(), g.get_Sbus(), g.get_slack_ids(), g.get_slack_weights(),
                           g.get_pv(), g.get_pq(), MAX_ITER, TOL)
    Vn = base.get_V()
    d = N1Device(g, Vn, dev, precision=0)
    times = _time_device(lambda: d.launch(stream.cuda_stream), stream, K, W, flush)
    V, it, er = d.results()
    nconv = int((er == 0).sum())
    _, cp, rows, cols, vals = _n1_arrays(g)
    d.plan.batch_n1_arrays(cp, rows, cols, vals, Vn, g.get_Sbus(), MAX_ITER, TOL)
    e2e = []
    for _ in range(5):
        t0 = time.perf_counter()
        Vh, convh, _, _ = d.plan.batch_n1_arrays(cp, rows, cols, vals, Vn, g.get_Sbus(), MAX_ITER, TOL)
        e2e.append(time.perf_counter() - t0)
    ob = ContingencyBatch(g.get_Ybus(), g.get_Sbus(), Vn, g.get_slack_ids(), g.get_slack_weights(), g.get_pv(),
                          g.get_pq(), d.coeffs)
    _, Vo, conv_o, it_o, err_o, _ = ob.run(threads)
    sol = d.solvable
    both = (er == 0) & conv_o[sol]
    return {"workload": "N-1 all 186 single-branch outages, synthetic grid118 (118 buses, 54 PV), FP64, start = "
                        "base-case solution, tol 1e-8 pu",
            "value": nconv / float(np.mean(times)), "unit": "PF/s", "ms_per_step": 1e3 * float(np.mean(times)),
            "cases": len(d.coeffs), "solved": d.ns, "converged": nconv,
            "e2e": {"value": int(convh.sum()) / float(np.mean(e2e)), "unit": "PF/s",
                    "ms_per_step": 1e3 * float(np.mean(e2e)), "path": "pf_batch_n1 (host arrays)"},
            "vs_oracle": {"flags_equal": bool(np.array_equal(er == 0, conv_o[sol])),
                          "iterations_equal": bool(np.array_equal(it[both], it_o[sol][both])),
                          "dV": _err_stats(_dv(V[both], Vo[sol][both]))}}


def _config2(dev, stream, flush, K, W, threads, nsteps=8760):
    """Config 2: the 8,760-snapshot time series on the 2,848-bus grid, FP64 and mixed, chunked
    chains on the device (one chunk per resident CTA) and the whole series through the host
    API (pf_batch_ts, pinned host arrays); each form against the oracle's chains over the same
    chunks (TimeSeries::compute_Vs per chunk)."""
    import torch
    from lightsim2grid_b200 import Plan, synthetic
    from lightsim2grid_b200.timeseries import DeviceSeries, chunk_jobs
    from oracle.oracle import time_series_chunks

    g = _grid(GRID)
    Y, S = g.get_Ybus(), g.get_Sbus()
    sl, w, pv, pq = g.get_slack_ids(), g.get_slack_weights(), g.get_pv(), g.get_pq()
    Sb = g.sbuses_from_injections(*synthetic.time_series_injections(g, nsteps, seed=8760, level=0.9))
    base = Plan(Y, g.flat_start(), S, sl, w, pv, pq, precision=0)
    V0, conv, _, _ = base.solve(g.flat_start(), S, MAX_ITER, TOL)
    assert conv
    out = {"workload": "time series, {} snapshots on synthetic grid2848 (per-bus AR(1) phi 0.9 sigma 0.03 x shared "
                       "daily +-15 %, around 0.9 x base injections), warm start, chunked chains (one per resident "
                       "CTA, each from the base-case solution), tol 1e-8 pu".format(nsteps)}
    res = {}
    for label, prec in (("fp64", 0), ("mixed", 1)):
        plan = Plan(Y, V0, S, sl, w, pv, pq, precision=prec)
        nch = plan.info()["grid"]
        ds = DeviceSeries(plan, Sb, V0, nch, dev, MAX_ITER, TOL)
        times = _time_device(lambda: ds.launch(stream.cuda_stream), stream, K, W, flush)
        V, it, er = ds.results()
        res[label] = (V, it, er, nch)
        out[label] = {"value": float((er == 0).sum() / np.mean(times)), "unit": "PF/s",
                      "ms_per_step": 1e3 * float(np.mean(times)), "chunks": int(nch),
                      "converged": int((er == 0).sum()), "iterations_mean": float(it.mean())}
        if label == "mixed":
            n = g.n_bus
            Sp = torch.empty(nsteps * n * 2, dtype=torch.float64, pin_memory=True).numpy()
            Sp = Sp.view(np.complex128).reshape(nsteps, n)
            Sp[:] = Sb
            Vp = torch.empty(nsteps * n * 2, dtype=torch.float64, pin_memory=True).numpy()
            Vp = Vp.view(np.complex128).reshape(nsteps, n)
            ints = [torch.empty(nsteps, dtype=torch.int32, pin_memory=True).numpy() for _ in range(3)]
            plan.batch_ts(Sp, V0, nch, MAX_ITER, TOL, out=(Vp, *ints))
            e2e = []
            for _ in range(3):
                t0 = time.perf_counter()
                _, _, conv_h, _, _ = plan.batch_ts(Sp, V0, nch, MAX_ITER, TOL, out=(Vp, *ints))
                e2e.append(time.perf_counter() - t0)
            out["e2e"] = {"value": float(conv_h.sum() / np.mean(e2e)), "unit": "PF/s",
                          "ms_per_step": 1e3 * float(np.mean(e2e)), "h2d_bytes_per_step": int(nsteps * n * 16),
                          "d2h_bytes_per_step": int(nsteps * n * 16 + 3 * nsteps * 4),
                          "path": "Plan.batch_ts -> pf_batch_ts (pinned host injections in, voltages out)"}
    out["mixed_over_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    # the oracle's chains over each form's chunks (both forms use the same chunking)
    jf, jc = chunk_jobs(nsteps, res["mixed"][3])
    Vo, conv_o, it_o, err_o = time_series_chunks(Y, S, Sb, V0, sl, w, pv, pq, jf, jc, MAX_ITER, TOL, threads)
    vs = {}
    for label in ("fp64", "mixed"):
        V, it, er, nch = res[label]
        if nch != res["mixed"][3]:
            jf2, jc2 = chunk_jobs(nsteps, nch)
            Vo2, co2, io2, _ = time_series_chunks(Y, S, Sb, V0, sl, w, pv, pq, jf2, jc2, MAX_ITER, TOL, threads)
        else:
            Vo2, co2, io2 = Vo, conv_o, it_o
        both = (er == 0) & co2
        vs[label] = {"flags_equal": bool(np.array_equal(er == 0, co2)), "dV": _err_stats(_dv(V[both], Vo2[both]))}
        if label == "fp64":
            vs[label]["iterations_equal"] = bool(np.array_equal(it[both], io2[both]))
    out["vs_oracle"] = vs
    return out


def _config3(dev, stream, flush, K, W, threads, total=4096, seed=4096):
    """Config 3: 4,096 outages drawn over the 118/1,354/2,848-bus grids (1:2:5), mixed
    precision, one persistent launch captured in a CUDA graph and replayed; schedules picked by
    the autotuner on a sample of the mix; flags against the oracle's."""
    from lightsim2grid_b200 import synthetic
    from lightsim2grid_b200.autotune import tune_uneven
    from lightsim2grid_b200.multi import build_uneven, draw_outages
    from oracle.oracle import ContingencyBatch

    names, weights = ("grid118", "grid1354", "grid2848"), (1, 2, 5)
    counts = [total * w // sum(weights) for w in weights]
    counts[-1] += total - sum(counts)
    grids = [(nm, _grid(nm), k) for nm, k in zip(names, counts)]
    t0 = time.perf_counter()
    sample = draw_outages([(nm, g, max(8, k // 8)) for nm, g, k in grids], seed + 1)
    best, table = tune_uneven(sample, precision=1, device=dev)
    tune_s = time.perf_counter() - t0
    mb, cases = build_uneven(draw_outages(grids, seed), dev, precision=1, **best)
    for _ in range(W):
        mb.launch(stream.cuda_stream)
    graph = mb.capture()
    times = _time_device(graph.replay, stream, K, 1, flush)
    conv_tot, flags_equal, dvs = 0, True, []
    per = {}
    for gc in cases:
        V, conv, it, er = gc.results()
        g = gc.grid
        ob = ContingencyBatch(g.get_Ybus(), gc.Sbase, gc.Vbase, g.get_slack_ids(), g.get_slack_weights(), g.get_pv(),
                              g.get_pq(), [g.branch_coeffs([int(b)]) for b in gc.branches])
        _, Vo, conv_o, _, _, _ = ob.run(threads)
        eq = bool(np.array_equal(conv, conv_o))
        flags_equal &= eq
        both = conv & conv_o
        dvs.append(_dv(V[both], Vo[both]))
        conv_tot += int(conv.sum())
        per[gc.name] = {"cases": len(gc.branches), "solvable": gc.ninst, "converged": int(conv.sum()),
                        "flags_equal": eq}
    info = mb.info()
    mb.close()
    return {"workload": "uneven N-1: {} outages drawn over synthetic grid118/grid1354/grid2848 (1:2:5), mixed "
                        "precision, one persistent launch captured in a CUDA graph".format(total),
            "value": conv_tot / float(np.mean(times)), "unit": "PF/s", "ms_per_step": 1e3 * float(np.mean(times)),
            "converged": conv_tot, "grids": per, "launch": info,
            "autotune": {"chosen": best, "seconds": tune_s, "table": table},
            "vs_oracle": {"flags_equal": flags_equal, "dV": _err_stats(np.concatenate(dvs) if dvs else np.zeros(0))}}


def _largest_grid(dev, stream, flush, K, W, threads, hbm_peak):
    """N-1 over every branch of the 6,515-bus grid, mixed and FP64, through the default layout (the
    batch-interleaved kernel: the LU cannot stay in shared memory), with the algorithmic-bytes
    roofline of each; each result against the oracle on all outages (flags, iterations, |dV|)."""
    from lightsim2grid_b200 import GPUNRSolverSingleSlack
    from oracle.oracle import ContingencyBatch

    g = _grid("grid6515")
    base = GPUNRSolverSingleSlack()
    assert base.compute_pf(g.get_Ybus(), g.flat_start(), g.get_Sbus(), g.get_slack_ids(), g.get_slack_weights(),
                           g.get_pv(), g.get_pq(), MAX_ITER, TOL)
    Vn = base.get_V()
    out = {"workload": "N-1 all 8,796 single-branch outages, synthetic grid6515 (seed 6516), start = base-case "
                       "solution, tol 1e-8 pu; default layout (batch-interleaved, stragglers handed to the one-CTA "
                       "kernel)"}
    oracle = None
    for label, prec in (("mixed", 1), ("fp64", 0)):
        d = N1Device(g, Vn, dev, prec)
        times = _time_device(lambda: d.launch(stream.cuda_stream), stream, max(3, K // 2), W, flush)
        V, it, er = d.results()
        info = d.plan.info()
        abytes, per_it = _algorithmic_bytes(info, it, 4 if prec else 8)
        t = float(np.mean(times))
        out[label] = {"value": float((er == 0).sum() / t), "unit": "PF/s", "ms_per_step": 1e3 * t,
                      "solved": d.ns, "converged": int((er == 0).sum()), "iterations": int(it.sum()),
                      "roofline": {"achieved_gbs": abytes / t / 1e9, "peak_gbs": hbm_peak,
                                   "frac": abytes / t / 1e9 / hbm_peak,
                                   "algorithmic_bytes_per_instance_iteration": per_it,
                                   "note": "launch = batch-interleaved kernel + its follow-up launches"}}
        if oracle is None:
            ob = ContingencyBatch(g.get_Ybus(), g.get_Sbus(), Vn, g.get_slack_ids(), g.get_slack_weights(),
                                  g.get_pv(), g.get_pq(), d.coeffs, MAX_ITER, TOL)
            _, Vo, conv_o, it_o, _, _ = ob.run(threads)
            oracle = (Vo, conv_o, it_o)
        Vo, conv_o, it_o = oracle
        sol = d.solvable
        ok_g = er == 0
        both = ok_g & conv_o[sol]
        dv = _dv(V[both], Vo[sol][both])
        tol_v = 1e-8 if prec else 1e-10
        out[label]["vs_oracle"] = {"flags_equal": bool(np.array_equal(ok_g, conv_o[sol])),
                                   "iterations_equal": int((it[both] == it_o[sol][both]).sum()),
                                   "dV": _err_stats(dv), "tolerance": tol_v,
                                   "beyond_tolerance": int((dv > tol_v).sum())}
        del d
    out["mixed_over_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    return out


def _high_fill(dev, stream, flush, K, W, threads, name="grid2848c300"):
    """N-1 over every branch of the 2,848-bus grid with 300 of its extra branches drawn as
    long-range chords (126k LU entries, 259 elimination levels): the dense-tail path, mixed and
    FP64, against the CPU oracle on the same outages (its time on all host threads, its flags and
    voltages)."""
    from oracle.oracle import ContingencyBatch

    g = _grid(name)
    Vn = _oracle_base(g)
    out = {"workload": "N-1 all 3,776 single-branch outages, synthetic {} (the 2848-bus grid with 300 of its "
                       "929 extra branches as uniformly random long-range chords), start = base-case solution, "
                       "tol 1e-8 pu; default plan (dense tail)".format(name)}
    res = {}
    for label, prec in (("mixed", 1), ("fp64", 0)):
        d = N1Device(g, Vn, dev, prec)
        times = _time_device(lambda: d.launch(stream.cuda_stream), stream, max(3, K // 2), W, flush)
        V, it, er = d.results()
        t = float(np.mean(times))
        info = d.plan.info()
        out[label] = {"value": float((er == 0).sum() / t), "unit": "PF/s", "ms_per_step": 1e3 * t,
                      "solved": d.ns, "converged": int((er == 0).sum()), "iterations": int(it.sum()),
                      "tail_k": info["tail_k"], "nnz_lu": info["nnz_lu"]}
        res[label] = (d.solvable, V, er)
        coeffs = d.coeffs
        del d
    ob = ContingencyBatch(g.get_Ybus(), g.get_Sbus(), Vn, g.get_slack_ids(), g.get_slack_weights(), g.get_pv(),
                          g.get_pq(), coeffs, MAX_ITER, TOL)
    ob.prepare(threads)
    ok, Vo, conv_o, _, _, dt = ob.run(threads)
    out["cpu_oracle"] = {"value": float(conv_o.sum() / dt), "unit": "PF/s", "cores": threads, "kind": "port",
                         "ms": 1e3 * dt}
    for label in ("mixed", "fp64"):
        sol, V, er = res[label]
        ok_g = er == 0
        both = ok_g & conv_o[sol]
        out[label]["vs_oracle"] = {"flags_equal": bool(np.array_equal(ok_g, conv_o[sol])),
                                   "dV": _err_stats(_dv(V[both], Vo[sol][both]))}
        out[label]["over_cpu"] = out[label]["value"] / out["cpu_oracle"]["value"]
    return out


SERVE_GRIDS = ("grid14", "grid118", "grid300", "grid1354", "grid2848", "grid6515")


def _serve(seconds, rate, device, reserved_sms=None, large_request_ctas=0, device_loop=False, loop_ctas=(0, 0)):
    """Serving leg: Poisson arrivals at `rate` requests/s for `seconds` over the six synthetic
    grids (14 to 6,515 buses); half the requests are one power flow with injections scaled by
    U[0.9, 1.1] per bus, half an N-1 batch of 8 to 64 outages; mixed precision, tol 1e-8.
    reserved_sms / large_request_ctas: the serving core's SM reservation (pf_server_configure)."""
    from lightsim2grid_b200 import synthetic
    from lightsim2grid_b200.serving import PowerFlowServer, latency_stats, make_requests

    grids = {g: synthetic.make_named_grid(g)[0] for g in SERVE_GRIDS}
    budget, slots = 4 << 30, 32
    srv = PowerFlowServer(grids, device=device, hbm_budget=budget, slots=slots, precision=1, max_iter=MAX_ITER,
                          tol=TOL, reserved_sms=reserved_sms, large_request_ctas=large_request_ctas)
    if device_loop:
        srv.native.set_device_loop(True, *loop_ctas)
    nb = {k: v.n_bus for k, v in grids.items()}
    nbr = {k: v.nb_powerline() for k, v in grids.items()}
    srv.serve(make_requests(nb, rate=rate, duration=min(1.0, seconds), seed=12345, branches_of=nbr))  # warm-up
    for g in SERVE_GRIDS:
        for kind in ("pf", "n1"):
            srv.native.latency_split(g, kind, reset=True)
    reqs = make_requests(nb, rate=rate, duration=seconds, seed=2024, branches_of=nbr)
    done = srv.serve(reqs, realtime=True)
    st = latency_stats(done)
    per = {}
    for g in SERVE_GRIDS:
        for kind in ("pf", "n1"):
            rs = [r for r in done if r.grid == g and r.kind == kind]
            lat = np.array([r.latency for r in rs])
            if lat.size:
                # host lag: arrival to the submission by the serving loop
                lag = np.array([r.t_admit - r.arrival for r in rs if r.t_admit is not None])
                per["{}/{}".format(g, kind)] = {"p50_ms": float(np.percentile(lat, 50) * 1e3),
                                                "p99_ms": float(np.percentile(lat, 99) * 1e3), "count": int(lat.size),
                                                "submit_lag_p99_ms": float(np.percentile(lag, 99) * 1e3) if lag.size
                                                else None,
                                                # the serving core's clock: admission wait and device time
                                                "core": srv.native.latency_split(g, kind)}
    st.update({"duration_s": seconds, "arrival_rate": rate, "grids": list(SERVE_GRIDS), "per_class": per,
               "reserved_sms": reserved_sms, "large_request_ctas": large_request_ctas,
               "mode": "device-resident request loop" if device_loop else "one launch per request",
               "loop_ctas": list(loop_ctas) if device_loop else None,
               "slots": slots, "hbm_budget_bytes": budget, "peak_inflight": srv.last.peak_inflight,
               "peak_bytes": srv.last.peak_bytes, "rejected": len(srv.last.rejected),
               "latency": "arrival to result in the caller's host arrays (host clock)",
               "host_loop": srv.last.host_stats()})
    return st


# ----------------------------------------------------------------------------- arms

def _oracle_batch(g, Vn, coeffs):
    from oracle.oracle import ContingencyBatch

    return ContingencyBatch(g.get_Ybus(), g.get_Sbus(), Vn, g.get_slack_ids(), g.get_slack_weights(), g.get_pv(),
                            g.get_pq(), coeffs, MAX_ITER, TOL)


def _oracle_base(g):
    from oracle.oracle import OracleNR

    s = OracleNR(False)
    assert s.compute_pf(g.get_Ybus(), g.flat_start(), g.get_Sbus(), g.get_slack_ids(), g.get_slack_weights(),
                        g.get_pv(), g.get_pq(), MAX_ITER, TOL)
    return s.get_V()


def run_reference(args):
    ws, rank, _ = _dist_init()
    if rank != 0:
        return 0
    from oracle import oracle as orc

    orc.build()
    g = _grid()
    Vn = _oracle_base(g)
    coeffs = _n1_arrays(g)[0]
    P = _host_threads()
    ob = _oracle_batch(g, Vn, coeffs)
    ob.prepare(P)  # coefficient layout per thread, outside the timed steps
    times, convs = [], []
    for step in range(args.warmup + args.steps):
        ok, _, conv, _, _, dt = ob.run(P)
        assert ok
        if step >= args.warmup:
            times.append(dt)
            convs.append(int(conv.sum()))
    value = float(sum(convs) / sum(times))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "PF/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(times)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "cases_per_step": len(coeffs), "converged_per_step": convs[-1],
                   "same_config": True},
        "cpu_baseline": {"value": value, "unit": "PF/s", "cores": P, "kind": "port", "cpu_model": _cpu_model(),
                         "sample": "all {} single-branch outages per step over {} host threads (contiguous slices, "
                                   "one computer per thread, each with its base power flow)".format(len(coeffs), P)},
        "e2e": {"value": value, "unit": "PF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference cannot be built here (Eigen and SuiteSparse submodules are empty); this is the "
                "oracle's C restatement of its NR loop with its own Gilbert-Peierls LU",
    }
    print(json.dumps(line))
    return 0


def run_ours(args):
    import torch
    import torch.distributed as dist

    ws, rank, local = _dist_init()
    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    from lightsim2grid_b200 import GPUNRSolverSingleSlack

    g = _grid()
    S = g.get_Sbus()
    n = g.n_bus
    base = GPUNRSolverSingleSlack()
    assert base.compute_pf(g.get_Ybus(), g.flat_start(), S, g.get_slack_ids(), g.get_slack_weights(), g.get_pv(),
                           g.get_pq(), MAX_ITER, TOL), "base case must converge"
    Vn = base.get_V()
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2
    barrier = dist.barrier if ws > 1 else None

    results = {}
    sampler = ClockSampler(local)
    for label, precision in (("mixed", 1), ("fp64", 0)):
        d = N1Device(g, Vn, dev, precision)
        if label == "mixed":
            sampler.start()
        times = _time_device(lambda: d.launch(stream.cuda_stream), stream, args.steps, args.warmup, flush, barrier)
        if label == "mixed":
            clocks = sampler.stop()
        V, it, er = d.results()
        nconv = int((er == 0).sum())
        tot = float(sum(times))
        if ws > 1:
            tt = torch.tensor([tot], dtype=torch.float64, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            tot = float(tt.item())
        info = d.plan.info()
        abytes, per_it = _algorithmic_bytes(info, it, 4 if precision else 8)
        results[label] = dict(dev=d, nconv=nconv, times=times, total=tot, info=info, V=V, iters=it, errs=er,
                              value=ws * nconv * args.steps / tot, abytes=abytes, per_it=per_it)

    mixed, fp64 = results["mixed"], results["fp64"]
    hbm_peak, peak_kind = _peaks()
    kt = float(np.mean(mixed["times"]))
    achieved = mixed["abytes"] / kt / 1e9
    prof = _profile_figures()
    units = float(np.sum(mixed["iters"]))
    traffic = prof["traffic_bytes_per_instance_iteration"] * units if "traffic_bytes_per_instance_iteration" in prof \
        else None

    # e2e through the host C-ABI (host buffers, copies in the timed region); results land in
    # pinned host arrays, inputs are the host coefficient arrays
    d_mixed = mixed["dev"]
    plan_e2e = d_mixed.plan
    coeffs, cp, rows, cols, vals = _n1_arrays(g)
    nc = len(coeffs)
    pinned = (torch.empty(nc * n * 2, dtype=torch.float64, pin_memory=True).numpy().view(np.complex128).reshape(nc, n),
              *(torch.empty(nc, dtype=torch.int32, pin_memory=True).numpy() for _ in range(3)))
    for _ in range(max(1, min(args.warmup, 2))):
        plan_e2e.batch_n1_arrays(cp, rows, cols, vals, Vn, S, MAX_ITER, TOL, out=pinned)
    torch.cuda.synchronize()
    e2e_times, e2e_conv = [], 0
    ke = max(2, min(args.steps, 5))
    for _ in range(ke):
        t0 = time.perf_counter()
        Vout, conv, iters, errs = plan_e2e.batch_n1_arrays(cp, rows, cols, vals, Vn, S, MAX_ITER, TOL, out=pinned)
        e2e_times.append(time.perf_counter() - t0)
        e2e_conv = int(conv.sum())
    e2e_t = float(np.mean(e2e_times))
    tm = plan_e2e.timers()  # the last call: total, host preparation, uploads, kernel, downloads, FP64 re-solves
    e2e_breakdown = {"total_ms": 1e3 * tm[0], "host_prep_ms": 1e3 * tm[1], "h2d_ms": 1e3 * tm[2],
                     "kernel_ms": 1e3 * tm[3], "d2h_ms": 1e3 * tm[4], "fp64_resolves": int(tm[5])}
    if ws > 1:
        tt = torch.tensor([e2e_t], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_t = float(tt.item())
    ns = d_mixed.ns
    h2d = 2 * n * 16 + (ns + 1) * 4 + int(cp[-1]) * (4 + 16) + 2 * ns * 4
    d2h = nc * n * 16 + 2 * ns * 4  # every case's voltage row (zero rows included), iterations, errors

    legs = {}
    P = _host_threads()
    if rank == 0 and ws == 1 and not args.no_configs:
        from oracle import oracle as orc

        orc.build()
        for key, fn in (("config1", _config1), ("config2", _config2), ("config3", _config3)):
            try:
                legs[key] = fn(dev, stream, flush, args.steps, args.warmup, P)
            except Exception as e:  # report, do not lose the headline line
                legs[key] = {"error": "{}: {}".format(type(e).__name__, e)}
        try:
            legs["grid6515"] = _largest_grid(dev, stream, flush, args.steps, args.warmup, P, _peaks()[0])
        except Exception as e:
            legs["grid6515"] = {"error": "{}: {}".format(type(e).__name__, e)}
        try:
            legs["high_fill"] = _high_fill(dev, stream, flush, args.steps, args.warmup, P)
        except Exception as e:
            legs["high_fill"] = {"error": "{}: {}".format(type(e).__name__, e)}

    serve = None
    if ws == 1 and args.serve_seconds > 0:
        serve = _serve(args.serve_seconds, args.serve_rate, dev, device_loop=not args.serve_launches)

    cpu, err_vs_oracle = None, None
    if rank == 0 and ws == 1 and not args.no_cpu:
        from oracle import oracle as orc

        orc.build()
        ob = _oracle_batch(g, Vn, coeffs)
        ob.prepare(P)
        ok, Vo, conv_o, it_o, err_o, dt_all = ob.run(P)
        nconv_cpu = int(conv_o.sum())
        # one core: a bounded contiguous sample of the same outages, one computer
        k1 = min(nc, 400)
        ob1 = _oracle_batch(g, Vn, coeffs[:k1])
        ob1.prepare(1)
        _, _, conv1, _, _, dt1 = ob1.run(1)
        cpu = {"value": nconv_cpu / dt_all, "unit": "PF/s", "cores": P, "kind": "port", "cpu_model": _cpu_model(),
               "sample": "all {} single-branch outages of grid2848 on {} host threads (contiguous slices, one oracle "
                         "computer per thread, each with its base power flow), {:.2f} s".format(nc, P, dt_all),
               "one_core": {"value": int(conv1.sum()) / dt1, "unit": "PF/s", "cores": 1,
                            "sample": "the first {} outages on one computer, {:.2f} s".format(k1, dt1)}}
        # each result's distance to the FP64 oracle (the converged cases of the timed batches)
        err_vs_oracle = {"unit": "max over buses of |d|V|| (pu) and |d angle| (rad), per result",
                         "tolerance": {"fp64": 1e-10, "mixed": 1e-8}}
        for label in ("mixed", "fp64"):
            r = results[label]
            sol = r["dev"].solvable
            ok_g = r["errs"] == 0
            both = ok_g & conv_o[sol]
            dv = _dv(r["V"][both], Vo[sol][both])
            err_vs_oracle[label] = dict(_err_stats(dv), flags_equal=bool(np.array_equal(ok_g, conv_o[sol])),
                                        errors_equal=bool(np.array_equal(r["errs"], err_o[sol])),
                                        iterations_equal=bool(np.array_equal(r["iters"][both], it_o[sol][both])),
                                        within_tolerance=bool(dv.size == 0 or dv.max() <= (
                                            1e-8 if label == "mixed" else 1e-10)))

    if rank == 0:
        info = mixed["info"]
        smem_frac = prof.get("smem_wavefronts_per_sm_cycle")
        line = {
            "metric": METRIC,
            "value": mixed["value"],
            "unit": "PF/s",
            "n_gpus": ws,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": 1e3 * mixed["total"] / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 LU + f64 residual/update",
            "data": "synthetic",
            "config": {
                "workload": WORKLOAD,
                "cases_per_step": int(ns), "converged_per_step": mixed["nconv"],
                "islanded_skipped": int(nc - ns),
                "l2": "flushed (256 MB write) before every timed step",
                "job_order": "hardest outages first (pf_n1_order: power mismatch of the outage at the start voltages)",
                "parallelism": "replicas" if ws > 1 else "single GPU",
                "plan": dict({k: info[k] for k in ("m", "nnz_j", "nnz_lu", "flops_refactor", "levels_refactor",
                                                   "groups_refactor", "threads", "lu_in_shared", "ctas_per_sm",
                                                   "grid", "smem_wavefronts_factor", "smem_wavefronts_backward",
                                                   "smem_wavefronts_forward")}),
                "iterations_mean": float(np.mean(mixed["iters"])),
            },
            "fp64": {"value": fp64["value"], "unit": "PF/s", "ms_per_step": 1e3 * fp64["total"] / args.steps,
                     "converged_per_step": fp64["nconv"], "lu_in_shared": fp64["info"]["lu_in_shared"]},
            "mixed_over_fp64": mixed["value"] / fp64["value"],
            "e2e": {"value": ws * e2e_conv / e2e_t, "unit": "PF/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": 1e3 * e2e_t,
                    "path": "Plan.batch_n1_arrays -> pf_batch_n1 (host buffers; islanding check, uploads, kernel, "
                            "download of all voltages into pinned host arrays)",
                    "breakdown": e2e_breakdown},
            "error_vs_oracle": err_vs_oracle,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "nr_batch_kernel<float,float,1,1,0,{}>".format(
                             _launch_bound(mixed["dev"].plan.info()["threads"])),
                         "algorithmic_bytes_per_launch": mixed["abytes"],
                         "algorithmic_bytes_per_instance_iteration": mixed["per_it"],
                         "kernel_ms": 1e3 * kt,
                         "binding": {
                             "resource": "not HBM: the LU and solve vector stay in shared memory and the slab in L2; "
                                         "the SM's issue and latency set the time (dependent ALU chains, L2 round "
                                         "trips, one barrier per elimination level, shared-memory wavefronts)",
                             "dram_bytes_per_instance_iteration": prof.get("traffic_bytes_per_instance_iteration"),
                             "l2_bytes_per_instance_iteration": prof.get("l2_bytes_per_instance_iteration"),
                             "smem_wavefronts_per_instance_iteration": prof.get(
                                 "smem_wavefronts_per_instance_iteration"),
                             "smem_pipe_frac": smem_frac,
                             "issue_active_frac": prof.get("issue_active_fraction"),
                             "profile": "profiles/nr_batch_kernel_n1_grid2848.md (ncu, reduced case, plan with {} "
                                        "levels)".format(int(prof.get("profile_levels_refactor", 0)) or "?")}},
            "serve": serve if serve is not None else {"skipped": "serving is measured at n_gpus = 1"},
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": args.steps,
            "gpu_launches_note": "one nr_batch_kernel launch per timed step of the mixed form (value); the FP64 "
                                 "form's timed region has another one per step",
        }
        line.update(legs)
        print(json.dumps(line))
    if ws > 1:
        torch.cuda.synchronize()
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ----------------------------------------------------------------------------- profiling mode

def run_case(argv):
    """One N-1 batch of a grid through pf_batch_device, for profilers (ncu) and quick timing."""
    ap = argparse.ArgumentParser(prog="bench.py case")
    ap.add_argument("--grid", default="grid2848")
    ap.add_argument("--cases", type=int, default=0, help="N branches from --first (0: all)")
    ap.add_argument("--first", type=int, default=0, help="first branch")
    ap.add_argument("--precision", type=int, default=1)
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--lu-placement", type=int, default=0)
    ap.add_argument("--ctas-per-sm", type=int, default=0)
    ap.add_argument("--refine", type=int, default=0, help="0 default (on), 1 on, 2 off")
    ap.add_argument("--lu-reuse", type=float, default=0.0, help="LU reuse threshold (<= 0: never, the default)")
    ap.add_argument("--refine-below", type=float, default=0.0,
                    help="mixed form: refine the steps taken from ||F||_inf below this (0: the default, 1e-3)")
    ap.add_argument("--check", action="store_true", help="compare the voltages with an FP64 plan's")
    ap.add_argument("--dc", action="store_true", help="DC power flows (DC Ybus, DC outage coefficients)")
    ap.add_argument("--fdpf", type=int, default=-1, help="fast decoupled power flows: 0 XB, 1 BX (-1: Newton)")
    ap.add_argument("--max-iter", type=int, default=10)
    ap.add_argument("--case-order", action="store_true", help="jobs in case order (default: hardest first)")
    ap.add_argument("--batch-layout", type=int, default=0, help="0 auto, 1 one CTA per instance, 2 batch-interleaved")
    ap.add_argument("--ordering", type=int, default=0)
    ap.add_argument("--placement", type=int, default=0)
    ap.add_argument("--level-slack", type=int, default=0)
    ap.add_argument("--handoff-lanes", type=int, default=0)
    ap.add_argument("--no-trace", action="store_true", help="skip the phase-cycle and trace launches")
    ap.add_argument("--cpu", action="store_true",
                    help="also time the CPU oracle's N-1 loop on the same outages (all host threads)")
    args = ap.parse_args(argv)

    import torch
    from lightsim2grid_b200 import GPUNRSolverSingleSlack, Plan, _native as nat

    g = _grid(args.grid)
    base = GPUNRSolverSingleSlack()
    if not base.compute_pf(g.get_Ybus(), g.flat_start(), g.get_Sbus(), g.get_slack_ids(), g.get_slack_weights(),
                           g.get_pv(), g.get_pq(), 10, 1e-8):
        raise SystemExit("base case did not converge")
    Vn = base.get_V()
    first = max(0, min(args.first, g.nb_powerline()))
    nb = g.nb_powerline() - first if args.cases <= 0 else min(args.cases, g.nb_powerline() - first)
    branches = range(first, first + nb)
    dev = torch.device("cuda:0")
    opts = dict(threads=args.threads, lu_placement=args.lu_placement, max_ctas_per_sm=args.ctas_per_sm,
                refine=args.refine, refine_threshold=args.refine_below, lu_reuse_threshold=args.lu_reuse,
                batch_layout=args.batch_layout,
                ordering=args.ordering, placement=args.placement, level_slack=args.level_slack,
                handoff_lanes=args.handoff_lanes)
    if args.dc or args.fdpf >= 0:
        # DC / FDPF: the grid's DC Ybus and outage coefficients, or its B' / B''
        gd = _DCView(g) if args.dc else g
        opts.update(dc=args.dc, fdpf=g.get_Bp_Bpp(args.fdpf) if args.fdpf >= 0 else None)
        d = N1Device(gd, Vn, dev, 0, branches=branches, case_order=True, **opts)
    else:
        d = N1Device(g, Vn, dev, args.precision, branches=branches, case_order=args.case_order, **opts)
    d.batch.max_iter = args.max_iter
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        d.launch(stream.cuda_stream)
    torch.cuda.synchronize()
    times = []
    for _ in range(args.repeat):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        d.launch(stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    V, it, er = d.results()
    phase_share, trace, cpi = None, None, None
    if not args.no_trace:
        lib, plan, b = d.lib, d.plan, d.batch
        cyc = np.zeros(8)
        assert lib.pf_batch_device_phase_cycles(plan.handle, nat.ctypes.byref(b), stream.cuda_stream,
                                                nat.ptr(cyc, nat.f64p)) == 0, nat.last_error(lib)
        names = ["mismatch", "jfill", "refactor", "forward", "backward", "refine", "update", "instances"]
        tot = cyc[:7].sum()
        # the DC and fast-decoupled kernels do not record phase cycles
        phase_share = {k: round(float(v / tot), 4) for k, v in zip(names[:7], cyc[:7])} if tot > 0 else None
        cpi = float(tot / max(1, int(it.sum()))) if tot > 0 else None
        tr = np.zeros(2048)
        ntr = lib.pf_batch_device_phase_trace(plan.handle, nat.ctypes.byref(b), stream.cuda_stream,
                                              nat.ptr(tr, nat.f64p), 2048)
        assert ntr >= 0, nat.last_error(lib)
        trace = np.diff(tr[:ntr]).astype(int).tolist()
    check = None
    if args.check:
        ref = N1Device(g, Vn, dev, 0, branches=branches, case_order=args.case_order)
        ref.launch(stream.cuda_stream)
        torch.cuda.synchronize()
        Vf, itf, ef = ref.results()
        both = (er == 0) & (ef == 0)
        check = {"flags_equal": bool(np.array_equal(er == 0, ef == 0)),
                 "max_dV_vs_fp64": float(_dv(V[both], Vf[both]).max()) if both.any() else None,
                 "iterations_fp64": int(itf.sum())}
    cpu = None
    if args.cpu and not (args.dc or args.fdpf >= 0):
        from oracle import oracle as orc

        orc.build()
        P = _host_threads()
        ob = _oracle_batch(g, Vn, _n1_arrays(g, branches)[0])
        ob.prepare(P)
        ob.run(P)
        ok, _, conv, _, _, dt = ob.run(P)
        assert ok
        cpu = {"pf_per_s": float(conv.sum() / dt), "ms": 1e3 * dt, "threads": P, "converged": int(conv.sum()),
               "cpu_model": _cpu_model(), "kind": "port"}
    out = {"grid": args.grid, "cases": d.ns, "precision": args.precision, "ms": times, "check": check, "cpu": cpu,
           "converged": int((er == 0).sum()), "iterations": int(it.sum()),
           "pf_per_s": float((er == 0).sum() / (np.mean(times) * 1e-3)),
           "cycles_per_iteration_per_cta": cpi, "phase_share": phase_share, "plan": d.plan.info(),
           "phase_trace_cycles": trace}
    print(json.dumps(out))
    return 0


class _DCView:
    """A grid seen through its DC admittance matrix and DC outage coefficients."""

    def __init__(self, g):
        self.g = g
        self.n_bus = g.n_bus

    def get_Ybus(self):
        return self.g.get_dcYbus()

    def branch_coeffs(self, b):
        return self.g.dc_branch_coeffs(b)

    def __getattr__(self, k):
        return getattr(self.g, k)


def run_serve(argv):
    """The serving leg alone: ``python bench.py serve [--seconds S --rate R --reserve K --large-ctas C]``."""
    ap = argparse.ArgumentParser(prog="bench.py serve")
    ap.add_argument("--seconds", type=float, default=10.0)
    ap.add_argument("--rate", type=float, default=2000.0)
    ap.add_argument("--reserve", type=int, default=-1, help="SMs reserved for small requests (-1: default)")
    ap.add_argument("--large-ctas", type=int, default=0, help="CTAs per large request (0: no cap)")
    ap.add_argument("--loop", action="store_true", help="device-resident request loop")
    ap.add_argument("--loop-ctas", default="0,0", help="CTAs of the shared-memory and global-LU loops (0: default)")
    args = ap.parse_args(argv)
    import torch

    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    out = _serve(args.seconds, args.rate, dev, None if args.reserve < 0 else args.reserve, args.large_ctas,
                 args.loop, tuple(int(x) for x in args.loop_ctas.split(",")))
    print(json.dumps(out))
    return 0


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "case":
        return run_case(sys.argv[2:])
    if len(sys.argv) > 1 and sys.argv[1] == "serve":
        return run_serve(sys.argv[2:])
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle baseline leg")
    ap.add_argument("--no-configs", action="store_true", help="skip the config 1-3 legs")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="serving leg duration (0: skip)")
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="serving leg arrival rate (requests/s)")
    ap.add_argument("--serve-launches", action="store_true",
                    help="serving leg with one launch per request (default: the device-resident loop for the small "
                         "requests)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
