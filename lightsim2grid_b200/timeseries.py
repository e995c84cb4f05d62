"""Time series on the GPU: warm-started power flows over many snapshots.

The reference's ``TimeSeries::compute_Vs`` (``src/batch_algorithm/TimeSeries.cpp:14-109``)
solves the snapshots one after the other, each starting from the previous solution, and stops
at the first divergence.  On the device a chain is one CTA's job: the snapshots are cut into
contiguous chunks (one job each; ``nchunks = 1`` is the reference's exact chain), each chunk
starts from the given start voltages and then warm-starts step to step.  Every snapshot's
answer is the converged state for its injections, so chunking changes the iteration counts of
chunk heads, not the answer beyond the tolerance.

``python -m lightsim2grid_b200.timeseries`` measures the 8,760-snapshot series on the 2,848-bus
synthetic grid (per-bus AR(1) profiles, phi 0.9, sigma 0.03, times a shared daily +-15%
sinusoid) in FP64 and in mixed precision on the device, the mixed form's distance to the FP64
results, and the whole series through the host API (``pf_batch_ts`` into pinned arrays).  The
parity of both forms against the CPU oracle's exact chain is the test suite's
(``tests/test_gpu_parity.py``).
"""
import argparse
import json
import sys
import time

import numpy as np

from . import _native as nat
from .solver import Plan


def chunk_jobs(nsteps, nchunks):
    """(first, count) of each contiguous chunk."""
    nchunks = max(1, min(int(nchunks), nsteps))
    edges = (np.arange(nchunks + 1, dtype=np.int64) * nsteps) // nchunks
    return edges[:-1].astype(np.int32), np.diff(edges).astype(np.int32)


class DeviceSeries:
    """A time series resident on the device: injections (steps x n), outputs, chunk jobs."""

    def __init__(self, plan, Sbuses, V0, nchunks, device, max_iter=10, tol=1e-8):
        import torch

        self.plan, self.n = plan, plan.n
        Sb = nat.as_c128(Sbuses)
        self.nsteps = Sb.shape[0]
        jf, jc = chunk_jobs(self.nsteps, nchunks)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
        self.d = dict(S=t(Sb.view(np.float64).ravel()), V0=t(nat.as_c128(V0).ravel().view(np.float64)), jf=t(jf),
                      jc=t(jc), V=torch.zeros(self.nsteps * self.n * 2, dtype=torch.float64, device=device),
                      it=torch.zeros(self.nsteps, dtype=torch.int32, device=device),
                      er=torch.zeros(self.nsteps, dtype=torch.int32, device=device))
        d = self.d
        self.batch = nat.PfDeviceBatch(n_inst=self.nsteps, V0=d["V0"].data_ptr(), v0_stride=0, Sbus=d["S"].data_ptr(),
                                       sbus_stride=self.n, ovr_ptr=0, ovr_pos=0, ovr_val=0, max_iter=max_iter,
                                       tol=tol, chain=1, job_first=d["jf"].data_ptr(), job_count=d["jc"].data_ptr(),
                                       njobs=int(jf.size), Vout=d["V"].data_ptr(), iters=d["it"].data_ptr(),
                                       errs=d["er"].data_ptr())
        self.nchunks = int(jf.size)

    def launch(self, stream):
        lib = self.plan._lib
        nat.check(lib.pf_batch_device(self.plan.handle, nat.ctypes.byref(self.batch), stream), "pf_batch_device", lib)

    def results(self):
        V = self.d["V"].cpu().numpy().view(np.complex128).reshape(self.nsteps, self.n)
        return V, self.d["it"].cpu().numpy(), self.d["er"].cpu().numpy()


def main(argv=None):
    ap = argparse.ArgumentParser(description="8,760-snapshot time series on the 2,848-bus synthetic grid")
    ap.add_argument("--grid", default="grid2848")
    ap.add_argument("--steps", type=int, default=8760)
    ap.add_argument("--chunks", type=int, default=0, help="0: one per resident CTA")
    ap.add_argument("--repeat", type=int, default=5)
    ap.add_argument("--seed", type=int, default=8760)
    ap.add_argument("--level", type=float, default=0.9,
                    help="profiles around this fraction of the base injections: at 1.0 the daily peak drives "
                         "the 2,848-bus synthetic grid into voltage collapse (snapshot 389 diverges)")
    args = ap.parse_args(argv)
    import torch

    from . import synthetic

    dev = torch.device("cuda:0")
    g, _ = synthetic.make_named_grid(args.grid)
    Y, S = g.get_Ybus(), g.get_Sbus()
    sl, w, pv, pq = g.get_slack_ids(), g.get_slack_weights(), g.get_pv(), g.get_pq()
    Sb = g.sbuses_from_injections(*synthetic.time_series_injections(g, args.steps, seed=args.seed, level=args.level))
    base = Plan(Y, g.flat_start(), S, sl, w, pv, pq, precision=0)
    V0, conv, _, _ = base.solve(g.flat_start(), S, 10, 1e-8)
    assert conv, "base case must converge"
    out = {"workload": "time series, {} snapshots on synthetic {} (AR(1) phi 0.9 sigma 0.03 x daily +-15%, around "
                       "{:.2f} x base injections), warm start, tol 1e-8 pu".format(args.steps, args.grid, args.level)}
    results = {}
    st = torch.cuda.current_stream()
    flush = torch.empty(256 << 20 >> 2, dtype=torch.float32, device=dev)
    for label, prec in (("fp64", 0), ("mixed", 1)):
        plan = Plan(Y, V0, S, sl, w, pv, pq, precision=prec)
        nch = args.chunks if args.chunks > 0 else plan.info()["grid"]
        ds = DeviceSeries(plan, Sb, V0, nch, dev)
        ds.launch(st.cuda_stream)
        torch.cuda.synchronize()
        times = []
        for _ in range(args.repeat):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            ds.launch(st.cuda_stream)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) * 1e-3)
        V, it, er = ds.results()
        results[label] = (V, er)
        out[label] = {"chunks": ds.nchunks, "ms": 1e3 * float(np.mean(times)), "converged": int((er == 0).sum()),
                      "pf_per_s": float((er == 0).sum() / np.mean(times)), "iterations_mean": float(it.mean())}
        if label == "mixed":
            # the whole series through the host API, injections from and results into pinned arrays
            nst = Sb.shape[0]
            Sp = torch.empty(nst * g.n_bus * 2, dtype=torch.float64, pin_memory=True).numpy()
            Sp = Sp.view(np.complex128).reshape(nst, g.n_bus)
            Sp[:] = Sb
            Vp = torch.empty(nst * g.n_bus * 2, dtype=torch.float64, pin_memory=True).numpy()
            Vp = Vp.view(np.complex128).reshape(nst, g.n_bus)
            ints = [torch.empty(nst, dtype=torch.int32, pin_memory=True).numpy() for _ in range(3)]
            plan.batch_ts(Sp, V0, nch, 10, 1e-8, out=(Vp, *ints))
            e2e = []
            for _ in range(max(2, args.repeat // 2)):
                t0 = time.perf_counter()
                st_h, _, conv_h, _, _ = plan.batch_ts(Sp, V0, nch, 10, 1e-8, out=(Vp, *ints))
                e2e.append(time.perf_counter() - t0)
            out[label]["e2e"] = {"ms": 1e3 * float(np.mean(e2e)), "pf_per_s": float(conv_h.sum() / np.mean(e2e)),
                                 "h2d_bytes": int(nst * g.n_bus * 16), "d2h_bytes": int(nst * g.n_bus * 16)}
    (Vf, ef), (Vm, em) = results["fp64"], results["mixed"]
    both = (ef == 0) & (em == 0)
    out["flags_equal_mixed_fp64"] = bool(np.array_equal(ef == 0, em == 0))
    out["max_abs_dV_mixed_vs_fp64"] = float(np.abs(Vm[both] - Vf[both]).max()) if both.any() else None
    out["mixed_over_fp64"] = out["mixed"]["pf_per_s"] / out["fp64"]["pf_per_s"]
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
