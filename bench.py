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
                     figure, the roofline of the kernel and the CPU oracle baseline.
  --impl reference   the CPU restatement of the reference's loop (oracle/, the reference
                     itself cannot be built here) on all host threads, same metric.

The ``serve`` object is the serving leg: Poisson arrivals (2,000 requests/s, 10 s by
default) over six synthetic grids of 14 to 6,515 buses, half single power flows with
perturbed injections and half N-1 batches of 8 to 64 outages, continuously batched on the
GPU; it reports p50/p99 latency and throughput.

Multi-GPU (torchrun): every rank runs the whole batch on its own GPU (replicas; the cases
are independent and nothing is exchanged); value = total converged PFs / max-over-ranks time.
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


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _traffic_from_profile():
    """Per-launch DRAM bytes of the kernel from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "nr_batch_kernel_n1_grid2848.md")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_instance_iteration:"):
                return float(line.split(":")[1])
    except Exception:
        pass
    return None


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


def _setup_problem():
    from lightsim2grid_b200 import synthetic

    g, _ = synthetic.make_named_grid(GRID)
    return g


def _n1_arrays(g):
    coeffs = [g.branch_coeffs([b]) for b in range(g.nb_powerline())]
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


def _cpu_oracle_n1(g, Vn, coeffs, threads):
    """The oracle's sequential N-1 loop on `threads` host threads, contiguous slices."""
    from oracle.oracle import contingency_analysis

    Y, S = g.get_Ybus(), g.get_Sbus()
    sl, w, pv, pq = g.get_slack_ids(), g.get_slack_weights(), g.get_pv(), g.get_pq()
    slices = np.array_split(np.arange(len(coeffs)), threads)
    res = [None] * threads

    def work(t):
        idx = slices[t]
        res[t] = contingency_analysis(Y, S, Vn, sl, w, pv, pq, [coeffs[i] for i in idx], MAX_ITER, TOL)

    th = [threading.Thread(target=work, args=(t,)) for t in range(threads)]
    t0 = time.perf_counter()
    for x in th:
        x.start()
    for x in th:
        x.join()
    dt = time.perf_counter() - t0
    nconv = sum(int(r[2].sum()) for r in res)
    return nconv, dt


SERVE_GRIDS = ("grid14", "grid118", "grid300", "grid1354", "grid2848", "grid6515")


def _serve(seconds, rate, device):
    """Serving leg: Poisson arrivals at `rate` requests/s for `seconds` over the six synthetic
    grids (14 to 6,515 buses); half the requests are one power flow with injections scaled by
    U[0.9, 1.1] per bus, half an N-1 batch of 8 to 64 outages; mixed precision, tol 1e-8."""
    from lightsim2grid_b200 import synthetic
    from lightsim2grid_b200.serving import PowerFlowServer, latency_stats, make_requests

    grids = {g: synthetic.make_named_grid(g)[0] for g in SERVE_GRIDS}
    budget, slots = 4 << 30, 32
    srv = PowerFlowServer(grids, device=device, hbm_budget=budget, slots=slots, precision=1, max_iter=MAX_ITER,
                          tol=TOL)
    nb = {k: v.n_bus for k, v in grids.items()}
    nbr = {k: v.nb_powerline() for k, v in grids.items()}
    srv.serve(make_requests(nb, rate=rate, duration=min(1.0, seconds), seed=12345, branches_of=nbr))  # warm-up
    reqs = make_requests(nb, rate=rate, duration=seconds, seed=2024, branches_of=nbr)
    done = srv.serve(reqs, realtime=True)
    st = latency_stats(done)
    per = {}
    for g in SERVE_GRIDS:
        lat = np.array([r.latency for r in done if r.grid == g])
        if lat.size:
            per[g] = {"p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3)}
    st.update({"duration_s": seconds, "arrival_rate": rate, "grids": list(SERVE_GRIDS), "per_grid": per,
               "slots": slots, "hbm_budget_bytes": budget, "peak_inflight": srv.last.peak_inflight,
               "peak_bytes": srv.last.peak_bytes, "rejected": len(srv.last.rejected),
               "latency": "arrival to result in pinned host memory (host clock)",
               "kernel_launches": len([r for r in done if r.ninst > 0])})
    return st


def _host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def _dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def run_reference(args):
    ws, rank, _ = _dist_init()
    if rank != 0:
        return 0
    from oracle import oracle as orc

    orc.build()
    from oracle.oracle import OracleNR

    g = _setup_problem()
    s = OracleNR(False)
    assert s.compute_pf(g.get_Ybus(), g.flat_start(), g.get_Sbus(), g.get_slack_ids(), g.get_slack_weights(),
                        g.get_pv(), g.get_pq(), MAX_ITER, TOL)
    Vn = s.get_V()
    coeffs = _n1_arrays(g)[0]
    P = _host_threads()
    rng = np.random.default_rng(0)
    sample = min(len(coeffs), 120 * P)
    times, convs = [], []
    for step in range(args.warmup + args.steps):
        idx = rng.choice(len(coeffs), size=sample, replace=False)
        nconv, dt = _cpu_oracle_n1(g, Vn, [coeffs[i] for i in sorted(idx)], P)
        if step >= args.warmup:
            times.append(dt)
            convs.append(nconv)
    value = float(sum(convs) / sum(times))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "PF/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(times)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "N-1 all single-branch outages, synthetic grid2848 (2848 buses, 3776 branches, "
                               "500 PV), start = base-case solution, tol 1e-8 pu, max_iter 10",
                   "sample_per_step": sample},
        "cpu_baseline": {"value": value, "unit": "PF/s", "cores": P, "kind": "port",
                         "sample": "{} random outages per step over {} threads (contiguous slices, one solver "
                                   "per thread)".format(sample, P)},
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
    from lightsim2grid_b200 import Plan, GPUNRSolverSingleSlack, _native as nat

    g = _setup_problem()
    Y, S = g.get_Ybus(), g.get_Sbus()
    sl, w, pv, pq = g.get_slack_ids(), g.get_slack_weights(), g.get_pv(), g.get_pq()
    n = g.n_bus
    base = GPUNRSolverSingleSlack()
    assert base.compute_pf(Y, g.flat_start(), S, sl, w, pv, pq, MAX_ITER, TOL), "base case must converge"
    Vn = base.get_V()
    coeffs, cp, rows, cols, vals = _n1_arrays(g)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)

    def make(precision):
        plan = Plan(Y, Vn, S, sl, w, pv, pq, precision=precision)
        lib = plan._lib
        ncases = len(coeffs)
        solv = np.zeros(ncases, np.int32)
        optr = np.zeros(ncases + 1, np.int32)
        cap = int(cp[-1])
        opos = np.zeros(cap, np.int32)
        oval = np.zeros(cap, np.complex128)
        nw = lib.pf_n1_prepare(plan.handle, ncases, nat.ptr(cp, nat.i32p), nat.ptr(rows, nat.i32p),
                               nat.ptr(cols, nat.i32p), nat.cptr(vals), nat.ptr(solv, nat.i32p),
                               nat.ptr(optr, nat.i32p), nat.ptr(opos, nat.i32p), nat.cptr(oval), cap)
        assert nw >= 0, nat.last_error(lib)
        ns = int(solv.sum())
        # the library's job order: hardest outages first (pf_n1_order)
        order = np.zeros(max(ns, 1), np.int32)
        V0c = nat.as_c128(Vn).ravel()
        assert lib.pf_n1_order(plan.handle, ns, nat.ptr(optr, nat.i32p), nat.ptr(opos, nat.i32p), nat.cptr(oval),
                               nat.cptr(V0c), nat.ptr(order, nat.i32p)) == 0, nat.last_error(lib)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        bufs = dict(V0=t(nat.as_c128(Vn).ravel().view(np.float64)), S=t(nat.as_c128(S).ravel().view(np.float64)),
                    optr=t(optr[:ns + 1]), opos=t(opos[:nw]), oval=t(oval[:nw].view(np.float64)),
                    jf=t(order[:ns]), jc=t(np.ones(ns, np.int32)),
                    Vout=torch.zeros(ns * n * 2, dtype=torch.float64, device=dev),
                    it=torch.zeros(ns, dtype=torch.int32, device=dev),
                    er=torch.zeros(ns, dtype=torch.int32, device=dev))
        b = nat.PfDeviceBatch(n_inst=ns, V0=bufs["V0"].data_ptr(), v0_stride=0, Sbus=bufs["S"].data_ptr(),
                              sbus_stride=0, ovr_ptr=bufs["optr"].data_ptr(), ovr_pos=bufs["opos"].data_ptr(),
                              ovr_val=bufs["oval"].data_ptr(), max_iter=MAX_ITER, tol=TOL, chain=0,
                              job_first=bufs["jf"].data_ptr(), job_count=bufs["jc"].data_ptr(), njobs=ns,
                              Vout=bufs["Vout"].data_ptr(), iters=bufs["it"].data_ptr(), errs=bufs["er"].data_ptr())
        return plan, b, bufs, ns

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2

    def timed(plan, b, K, W):
        lib = plan._lib
        for _ in range(W):
            rc = lib.pf_batch_device(plan.handle, nat.ctypes.byref(b), stream.cuda_stream)
            assert rc == 0, nat.last_error(lib)
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
        for k in range(K):
            flush.zero_()
            evs[k][0].record(stream)
            rc = lib.pf_batch_device(plan.handle, nat.ctypes.byref(b), stream.cuda_stream)
            evs[k][1].record(stream)
            assert rc == 0, nat.last_error(lib)
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()
        return [a.elapsed_time(e) * 1e-3 for a, e in evs]

    results = {}
    sampler = ClockSampler(local)
    for label, precision in (("mixed", 1), ("fp64", 0)):
        plan, b, bufs, ns = make(precision)
        if label == "mixed":
            sampler.start()
        times = timed(plan, b, args.steps, args.warmup)
        if label == "mixed":
            clocks = sampler.stop()
        it = bufs["it"].cpu().numpy()
        er = bufs["er"].cpu().numpy()
        nconv = int((er == 0).sum())
        tot = float(sum(times))
        if ws > 1:
            tt = torch.tensor([tot], dtype=torch.float64, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            tot = float(tt.item())
        info = plan.info()
        abytes, per_it = _algorithmic_bytes(info, it[er == 0] if nconv else it, 4 if precision else 8)
        abytes_all, _ = _algorithmic_bytes(info, it, 4 if precision else 8)
        results[label] = dict(plan=plan, b=b, bufs=bufs, ns=ns, nconv=nconv, times=times, total=tot, info=info,
                              iters=it, errs=er, value=ws * nconv * args.steps / tot, abytes=abytes_all,
                              per_it=per_it)

    mixed, fp64 = results["mixed"], results["fp64"]
    hbm_peak, peak_kind = _peaks()
    kt = float(np.mean(mixed["times"]))
    achieved = mixed["abytes"] / kt / 1e9
    traffic_per_unit = _traffic_from_profile()
    traffic = None
    if traffic_per_unit is not None:
        traffic = float(traffic_per_unit * float(np.sum(mixed["iters"])))

    # e2e through the host C-ABI (host buffers, copies in the timed region); results land in
    # pinned host arrays, inputs are the host coefficient arrays
    plan_e2e = mixed["plan"]
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
    if ws > 1:
        tt = torch.tensor([e2e_t], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_t = float(tt.item())
    ns = mixed["ns"]
    h2d = 2 * n * 16 + (ns + 1) * 4 + int(cp[-1]) * (4 + 16) + 2 * ns * 4
    d2h = nc * n * 16 + 2 * ns * 4  # every case's voltage row (zero rows included), iterations, errors

    serve = None
    if ws == 1 and args.serve_seconds > 0:
        serve = _serve(args.serve_seconds, args.serve_rate, dev)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        from oracle import oracle as orc

        orc.build()
        P = _host_threads()
        nconv_cpu, dt_cpu = _cpu_oracle_n1(g, Vn, coeffs, P)
        cpu = {"value": nconv_cpu / dt_cpu, "unit": "PF/s", "cores": P, "kind": "port",
               "sample": "all {} single-branch outages of grid2848 on {} host threads (contiguous slices, one "
                         "oracle solver per thread), {:.1f} s wall".format(len(coeffs), P, dt_cpu)}

    if rank == 0:
        info = mixed["info"]
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
                "workload": "N-1 all single-branch outages, synthetic grid2848 (2848 buses, 3776 branches, 500 PV; "
                            "geometric topology, seed 2848), start = base-case solution, tol 1e-8 pu, max_iter 10",
                "cases_per_step": int(ns), "converged_per_step": mixed["nconv"],
                "islanded_skipped": int(len(coeffs) - ns),
                "l2": "flushed (256 MB write) before every timed step",
                "job_order": "hardest outages first (pf_n1_order: power mismatch of the outage at the start voltages)",
                "parallelism": "replicas" if ws > 1 else "single GPU",
                "plan": dict({k: info[k] for k in ("m", "nnz_j", "nnz_lu", "flops_refactor", "levels_refactor",
                                                   "groups_refactor", "threads", "lu_in_shared", "ctas_per_sm",
                                                   "grid", "smem_wavefronts_factor", "smem_wavefronts_backward",
                                                   "smem_wavefronts_forward")},
                             ordering="minimum degree of 8 relabellings, each with its least-depth equivalent",
                             placement="packed programs placed for few shared-memory bank conflicts"),
                "iterations_mean": float(np.mean(mixed["iters"])),
            },
            "fp64": {"value": fp64["value"], "unit": "PF/s", "ms_per_step": 1e3 * fp64["total"] / args.steps,
                     "converged_per_step": fp64["nconv"], "lu_in_shared": fp64["info"]["lu_in_shared"]},
            "mixed_over_fp64": mixed["value"] / fp64["value"],
            "e2e": {"value": ws * e2e_conv / e2e_t, "unit": "PF/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": 1e3 * e2e_t,
                    "path": "Plan.batch_n1_arrays -> pf_batch_n1 (host buffers; islanding check, uploads, kernel, "
                            "download of all voltages into pinned host arrays)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "nr_batch_kernel<float,float>",
                         "algorithmic_bytes_per_launch": mixed["abytes"],
                         "algorithmic_bytes_per_instance_iteration": mixed["per_it"],
                         "kernel_ms": 1e3 * kt},
            "serve": serve if serve is not None else {"skipped": "serving is measured at n_gpus = 1"},
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": args.steps,
            "gpu_launches_note": "one nr_batch_kernel launch per timed step of the mixed form (value); the FP64 "
                                 "form's timed region has another one per step",
        }
        print(json.dumps(line))
    if ws > 1:
        torch.cuda.synchronize()
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle baseline leg")
    ap.add_argument("--serve-seconds", type=float, default=10.0, help="serving leg duration (0: skip)")
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="serving leg arrival rate (requests/s)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
