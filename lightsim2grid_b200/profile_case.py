"""One N-1 batch launch of the engine, for profilers (ncu) and quick timing.

    python -m lightsim2grid_b200.profile_case --grid grid2848 --cases 600 --precision 1 --repeat 3

Builds the plan, prepares the outages (islanding check), runs ``--warmup`` untimed launches
and ``--repeat`` timed launches of ``nr_batch_kernel`` through ``pf_batch_device``, and prints
the CUDA-event time per launch and the converged count.
"""
import argparse
import json
import os
import sys

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", default="grid2848")
    ap.add_argument("--cases", type=int, default=0, help="first N branches (0: all)")
    ap.add_argument("--precision", type=int, default=1)
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--lu-placement", type=int, default=0)
    ap.add_argument("--fuse-forward", type=int, default=0)
    ap.add_argument("--ctas-per-sm", type=int, default=0)
    ap.add_argument("--refine", type=int, default=0, help="0 default (on), 1 on, 2 off")
    ap.add_argument("--refine-threshold", type=float, default=0.0)
    ap.add_argument("--lu-reuse", type=float, default=0.0, help="LU reuse threshold (<= 0: never, the default)")
    ap.add_argument("--check", action="store_true", help="compare the voltages with an FP64 plan's")
    ap.add_argument("--dc", action="store_true", help="DC power flows (DC Ybus, DC outage coefficients)")
    ap.add_argument("--fdpf", type=int, default=-1, help="fast decoupled power flows: 0 XB, 1 BX (-1: Newton)")
    ap.add_argument("--max-iter", type=int, default=10)
    ap.add_argument("--order", action="store_true", help="also time job orders by iterations and by mismatch")
    ap.add_argument("--case-order", action="store_true", help="jobs in case order (default: hardest first)")
    ap.add_argument("--batch-layout", type=int, default=0, help="0 auto, 1 one CTA per instance, 2 batch-interleaved")
    ap.add_argument("--ordering", type=int, default=0,
                    help="0: minimum degree + least-depth equivalent reordering, 1: minimum degree only")
    ap.add_argument("--placement", type=int, default=0,
                    help="packed programs: 0 clusters in first slots, 1 clusters spread")
    args = ap.parse_args()

    import torch
    from lightsim2grid_b200 import Plan, GPUNRSolverSingleSlack, synthetic, _native as nat

    g, _ = synthetic.make_named_grid(args.grid)
    Y, S = g.get_Ybus(), g.get_Sbus()
    sl, w, pv, pq = g.get_slack_ids(), g.get_slack_weights(), g.get_pv(), g.get_pq()
    base = GPUNRSolverSingleSlack()
    if not base.compute_pf(Y, g.flat_start(), S, sl, w, pv, pq, 10, 1e-8):
        raise SystemExit("base case did not converge")
    Vn = base.get_V()
    nb = g.nb_powerline() if args.cases <= 0 else min(args.cases, g.nb_powerline())
    coeffs = [g.branch_coeffs([b]) for b in range(nb)]
    if args.dc:
        Y = g.get_dcYbus()
        coeffs = [g.dc_branch_coeffs([b]) for b in range(nb)]
    fdpf = g.get_Bp_Bpp(args.fdpf) if args.fdpf >= 0 else None
    plan = Plan(Y, Vn, S, sl, w, pv, pq, precision=args.precision, dc=args.dc, fdpf=fdpf, threads=args.threads,
                lu_placement=args.lu_placement, fuse_forward=args.fuse_forward, max_ctas_per_sm=args.ctas_per_sm,
                refine=args.refine, refine_threshold=args.refine_threshold, lu_reuse_threshold=args.lu_reuse,
                batch_layout=args.batch_layout, ordering=args.ordering, placement=args.placement)
    lib = plan._lib
    cp = np.zeros(nb + 1, np.int32)
    rows, cols, vals = [], [], []
    for k, lst in enumerate(coeffs):
        cp[k + 1] = cp[k] + len(lst)
        for (r, c, y) in lst:
            rows.append(r)
            cols.append(c)
            vals.append(y)
    rows, cols, vals = nat.as_i32(rows), nat.as_i32(cols), nat.as_c128(vals).ravel()
    solv = np.zeros(nb, np.int32)
    optr = np.zeros(nb + 1, np.int32)
    cap = int(cp[-1])
    opos = np.zeros(cap, np.int32)
    oval = np.zeros(cap, np.complex128)
    nw = lib.pf_n1_prepare(plan.handle, nb, nat.ptr(cp, nat.i32p), nat.ptr(rows, nat.i32p), nat.ptr(cols, nat.i32p),
                           nat.cptr(vals), nat.ptr(solv, nat.i32p), nat.ptr(optr, nat.i32p), nat.ptr(opos, nat.i32p),
                           nat.cptr(oval), cap)
    assert nw >= 0, nat.last_error(lib)
    ns = int(solv.sum())
    dev = torch.device("cuda:0")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    bufs = [t(nat.as_c128(Vn).ravel().view(np.float64)), t(nat.as_c128(S).ravel().view(np.float64)),
            t(optr[:ns + 1]), t(opos[:nw]), t(oval[:nw].view(np.float64)), t(np.arange(ns, dtype=np.int32)),
            t(np.ones(ns, np.int32)), torch.zeros(ns * g.n_bus * 2, dtype=torch.float64, device=dev),
            torch.zeros(ns, dtype=torch.int32, device=dev), torch.zeros(ns, dtype=torch.int32, device=dev)]
    if not args.case_order and not args.dc and args.fdpf < 0:
        # jobs hardest first (pf_n1_order), as pf_batch_n1 and the bench run them
        order = np.zeros(max(ns, 1), np.int32)
        V0c = nat.as_c128(Vn).ravel()
        assert lib.pf_n1_order(plan.handle, ns, nat.ptr(optr, nat.i32p), nat.ptr(opos, nat.i32p), nat.cptr(oval),
                               nat.cptr(V0c), nat.ptr(order, nat.i32p)) == 0, nat.last_error(lib)
        bufs[5] = t(order[:ns])
    b = nat.PfDeviceBatch(n_inst=ns, V0=bufs[0].data_ptr(), v0_stride=0, Sbus=bufs[1].data_ptr(), sbus_stride=0,
                          ovr_ptr=bufs[2].data_ptr(), ovr_pos=bufs[3].data_ptr(), ovr_val=bufs[4].data_ptr(),
                          max_iter=args.max_iter, tol=1e-8, chain=0, job_first=bufs[5].data_ptr(),
                          job_count=bufs[6].data_ptr(), njobs=ns, Vout=bufs[7].data_ptr(), iters=bufs[8].data_ptr(),
                          errs=bufs[9].data_ptr())
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        assert lib.pf_batch_device(plan.handle, nat.ctypes.byref(b), stream.cuda_stream) == 0, nat.last_error(lib)
    torch.cuda.synchronize()
    times = []
    for _ in range(args.repeat):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        assert lib.pf_batch_device(plan.handle, nat.ctypes.byref(b), stream.cuda_stream) == 0, nat.last_error(lib)
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    order_times = {}
    if args.order:
        # job orders: by the iterations each instance took (ideal), and by the outage's power
        # mismatch at the start voltages (|V o conj(dY V)|, known before solving)
        it0 = bufs[8].cpu().numpy().copy()
        er0 = bufs[9].cpu().numpy().copy()
        sol = np.nonzero(solv)[0]
        dS = np.zeros(ns)
        for i, cidx in enumerate(sol):
            acc = {}
            for (r, cc, y) in coeffs[cidx]:
                acc[r] = acc.get(r, 0) + Vn[r] * np.conj(y * Vn[cc])
            dS[i] = max(abs(v) for v in acc.values()) if acc else 0.0
        for label, key in (("by_iterations", -(it0 + 100 * (er0 != 0))), ("by_mismatch", -dS)):
            order = np.argsort(key, kind="stable").astype(np.int32)
            bufs[5].copy_(torch.from_numpy(order).to(dev))
            for _ in range(args.warmup):
                assert lib.pf_batch_device(plan.handle, nat.ctypes.byref(b), stream.cuda_stream) == 0
            ts = []
            for _ in range(args.repeat):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                assert lib.pf_batch_device(plan.handle, nat.ctypes.byref(b), stream.cuda_stream) == 0
                e1.record(stream)
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1))
            order_times[label] = ts
            assert np.array_equal(bufs[8].cpu().numpy(), it0) and np.array_equal(bufs[9].cpu().numpy(), er0)
    cyc = np.zeros(8)
    assert lib.pf_batch_device_phase_cycles(plan.handle, nat.ctypes.byref(b), stream.cuda_stream,
                                            nat.ptr(cyc, nat.f64p)) == 0, nat.last_error(lib)
    names = ["mismatch", "jfill", "refactor", "forward", "backward", "refine", "update", "instances"]
    tot = cyc[:7].sum()
    # the DC and fast-decoupled kernels do not record phase cycles
    phase_share = {k: round(float(v / tot), 4) for k, v in zip(names[:7], cyc[:7])} if tot > 0 else None
    tr = np.zeros(2048)
    ntr = lib.pf_batch_device_phase_trace(plan.handle, nat.ctypes.byref(b), stream.cuda_stream,
                                          nat.ptr(tr, nat.f64p), 2048)
    assert ntr >= 0, nat.last_error(lib)
    trace = np.diff(tr[:ntr]).astype(int).tolist()
    it = bufs[8].cpu().numpy()
    er = bufs[9].cpu().numpy()
    check = None
    if args.check:
        ref = Plan(Y, Vn, S, sl, w, pv, pq, precision=0)
        Vf = torch.zeros_like(bufs[7])
        itf = torch.zeros_like(bufs[8])
        erf = torch.zeros_like(bufs[9])
        b2 = nat.PfDeviceBatch(n_inst=ns, V0=bufs[0].data_ptr(), v0_stride=0, Sbus=bufs[1].data_ptr(), sbus_stride=0,
                               ovr_ptr=bufs[2].data_ptr(), ovr_pos=bufs[3].data_ptr(), ovr_val=bufs[4].data_ptr(),
                               max_iter=10, tol=1e-8, chain=0, job_first=bufs[5].data_ptr(),
                               job_count=bufs[6].data_ptr(), njobs=ns, Vout=Vf.data_ptr(), iters=itf.data_ptr(),
                               errs=erf.data_ptr())
        assert ref._lib.pf_batch_device(ref.handle, nat.ctypes.byref(b2), stream.cuda_stream) == 0
        torch.cuda.synchronize()
        ef = erf.cpu().numpy()
        both = (er == 0) & (ef == 0)
        Vm = bufs[7].cpu().numpy().view(np.complex128).reshape(ns, -1)
        Vr = Vf.cpu().numpy().view(np.complex128).reshape(ns, -1)
        check = {"flags_equal": bool(np.array_equal(er == 0, ef == 0)),
                 "max_abs_dV_vs_fp64": float(np.abs(Vm[both] - Vr[both]).max()) if both.any() else None,
                 "iterations_fp64": int(itf.cpu().numpy().sum())}
    out = {"grid": args.grid, "cases": ns, "precision": args.precision, "ms": times, "ms_ordered": order_times,
           "check": check,
           "converged": int((er == 0).sum()), "iterations": int(it.sum()),
           "pf_per_s": float((er == 0).sum() / (np.mean(times) * 1e-3)),
           "cycles_per_iteration_per_cta": float(tot / max(1, int(it.sum()))) if tot > 0 else None,
           "phase_share": phase_share,
           "plan": plan.info(), "phase_trace_cycles": trace}
    print(json.dumps(out))


if __name__ == "__main__":
    sys.exit(main())
