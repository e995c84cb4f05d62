"""Ybus and Sbus assembled on the GPU from element data.

The reference assembles Ybus from its elements' triplets on the host for every topology or
parameter change (``GridModel::fillYbus``, ``src/GridModel.cpp:676-699``) and Sbus from the
injections (``fillSbus_me``, ``:701-716``; per snapshot ``TimeSeries::compute_Sbuses``,
``src/batch_algorithm/TimeSeries.hpp:79-151``).  ``DeviceAssembly`` keeps a grid's branch data
and bus-to-element lists on the device next to a plan, so that a request that changes
impedances or branch statuses, or a time series given as injection matrices, gets its Ybus
values / Sbus rows on the device without host assembly.

``python -m lightsim2grid_b200.assembly`` measures the Sbus rows of the 8,760-snapshot series
of the 2,848-bus grid and one Ybus assembly against the HBM roofline.
"""
import argparse
import json
import sys

import numpy as np

from . import _native as nat


def _bus_lists(buses, n):
    """CSR (ptr, ids) of the elements at each bus, in element order."""
    buses = np.asarray(buses, np.int64)
    order = np.argsort(buses, kind="stable")
    ptr = np.zeros(n + 1, np.int32)
    np.cumsum(np.bincount(buses, minlength=n), out=ptr[1:])
    ids = order.astype(np.int32)
    return ptr, (ids if ids.size else np.zeros(1, np.int32))


class DeviceAssembly:
    """Device-side assembly for a ``GridModel`` and a plan built on its Ybus pattern."""

    def __init__(self, plan, grid, device):
        import torch

        self.plan, self.grid, self.device = plan, grid, device
        lib = plan._lib
        nb = int(grid.line_from.size)
        f, t = np.asarray(grid.line_from, np.int64), np.asarray(grid.line_to, np.int64)
        # contribution c = 4 k + kind at (row, col): ff (f,f), tt (t,t), ft (f,t), tf (t,f)
        rows = np.stack([f, t, f, t], axis=1).ravel().astype(np.int32)
        cols = np.stack([f, t, t, f], axis=1).ravel().astype(np.int32)
        pos = np.zeros(rows.size, np.int32)
        nat.check(lib.pf_ybus_positions(plan.handle, int(rows.size), rows.ctypes.data, cols.ctypes.data,
                                        pos.ctypes.data), "pf_ybus_positions", lib)
        if np.any(pos < 0):
            raise RuntimeError("a branch of the grid is not in the plan's Ybus pattern")
        self.nnz = int(plan.info()["nnz_ybus"])
        # per entry, its contributions in branch order (the reference's triplet order)
        order = np.argsort(pos, kind="stable")
        cptr = np.zeros(self.nnz + 1, np.int32)
        np.cumsum(np.bincount(pos, minlength=self.nnz), out=cptr[1:])
        self.positions = pos.reshape(nb, 4)
        tt = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
        self.d = dict(cptr=tt(cptr), cids=tt(order.astype(np.int32)))
        self.set_branches(grid.line_r, grid.line_x, grid.line_h, grid.line_status)
        n = int(grid.n_bus)
        self.n = n
        gp, gi = _bus_lists(grid.gen_bus, n)
        lp, li = _bus_lists(grid.load_bus, n)
        self.d.update(gen_ptr=tt(gp), gen_ids=tt(gi), load_ptr=tt(lp), load_ids=tt(li))
        self.nsgen = int(np.asarray(grid.sgen_bus).size)
        if self.nsgen:
            sp, si = _bus_lists(grid.sgen_bus, n)
            self.d.update(sgen_ptr=tt(sp), sgen_ids=tt(si))
        self.layout = nat.PfSbusLayout(
            n=n, ngen=int(np.asarray(grid.gen_bus).size), nsgen=self.nsgen, nload=int(np.asarray(grid.load_bus).size),
            gen_ptr=self.d["gen_ptr"].data_ptr(), gen_ids=self.d["gen_ids"].data_ptr(),
            sgen_ptr=self.d["sgen_ptr"].data_ptr() if self.nsgen else None,
            sgen_ids=self.d["sgen_ids"].data_ptr() if self.nsgen else None,
            load_ptr=self.d["load_ptr"].data_ptr(), load_ids=self.d["load_ids"].data_ptr())

    def set_branches(self, r, x, h, status):
        """Branch data on the device (per unit; h the total shunt, complex)."""
        import torch

        tt = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.device)
        self.d.update(r=tt(np.asarray(r, np.float64)), x=tt(np.asarray(x, np.float64)),
                      h=tt(np.asarray(h, np.complex128).view(np.float64)),
                      status=tt(np.asarray(status, np.uint8)))

    def ybus(self, stream, out=None):
        """Ybus values in the plan's storage order (device tensor of 2 * nnz doubles)."""
        import torch

        if out is None:
            out = torch.empty(2 * self.nnz, dtype=torch.float64, device=self.device)
        d = self.d
        lib = self.plan._lib
        nat.check(lib.pf_assemble_ybus_device(self.nnz, d["cptr"].data_ptr(), d["cids"].data_ptr(), d["r"].data_ptr(),
                                              d["x"].data_ptr(), d["h"].data_ptr(), d["status"].data_ptr(),
                                              out.data_ptr(), stream), "pf_assemble_ybus_device", lib)
        return out

    def apply(self, values, stream):
        """The plan's later launches use these Ybus values (device, storage order)."""
        lib = self.plan._lib
        nat.check(lib.pf_set_ybus_values_device(self.plan.handle, values.data_ptr(), stream),
                  "pf_set_ybus_values_device", lib)

    def sbus(self, gen_p, load_p, load_q, stream, sgen_p=None, out=None):
        """Sbus rows (device tensor of steps x n complex as doubles) from injection matrices
        (device float64 tensors, one row per snapshot)."""
        import torch

        steps = int(gen_p.shape[0]) if gen_p.dim() == 2 else 1
        if out is None:
            out = torch.empty(steps * self.n * 2, dtype=torch.float64, device=self.device)
        lib = self.plan._lib
        nat.check(lib.pf_assemble_sbus_device(nat.ctypes.byref(self.layout), steps, gen_p.data_ptr(),
                                              sgen_p.data_ptr() if sgen_p is not None else None,
                                              load_p.data_ptr(), load_q.data_ptr(), float(self.grid.sn_mva),
                                              out.data_ptr(), stream), "pf_assemble_sbus_device", lib)
        return out

    def host_ybus_in_storage_order(self, Y):
        """A host Ybus (scipy, same pattern or a sub-pattern) in the plan's storage order."""
        Y = Y.tocoo()
        vals = np.zeros(self.nnz, np.complex128)
        pos = np.zeros(Y.nnz, np.int32)
        r, c = Y.row.astype(np.int32), Y.col.astype(np.int32)
        nat.check(self.plan._lib.pf_ybus_positions(self.plan.handle, int(Y.nnz), r.ctypes.data, c.ctypes.data,
                                                   pos.ctypes.data), "pf_ybus_positions", self.plan._lib)
        if np.any(pos < 0):
            raise RuntimeError("the host Ybus has entries outside the plan's pattern")
        vals[pos] = Y.data
        return vals


def main(argv=None):
    ap = argparse.ArgumentParser(description="device Ybus / Sbus assembly on the 2,848-bus grid")
    ap.add_argument("--grid", default="grid2848")
    ap.add_argument("--steps", type=int, default=8760)
    ap.add_argument("--repeat", type=int, default=10)
    args = ap.parse_args(argv)
    import torch

    from . import synthetic
    from .solver import Plan

    dev = torch.device("cuda:0")
    g, _ = synthetic.make_named_grid(args.grid)
    plan = Plan(g.get_Ybus(), g.flat_start(), g.get_Sbus(), g.get_slack_ids(), g.get_slack_weights(), g.get_pv(),
                g.get_pq(), precision=1)
    asm = DeviceAssembly(plan, g, dev)
    gp, _, lp, lq = synthetic.time_series_injections(g, args.steps, seed=1, level=0.9)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    dgp, dlp, dlq = t(gp), t(lp), t(lq)
    st = torch.cuda.current_stream()
    out = asm.sbus(dgp, dlp, dlq, st.cuda_stream)
    yv = asm.ybus(st.cuda_stream)
    torch.cuda.synchronize()
    flush = torch.empty(256 << 20 >> 2, dtype=torch.float32, device=dev)

    def timed(fn):
        ts = []
        for _ in range(args.repeat):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1) * 1e-3)
        return float(np.median(ts))

    ts = timed(lambda: asm.sbus(dgp, dlp, dlq, st.cuda_stream, out=out))
    ty = timed(lambda: asm.ybus(st.cuda_stream, out=yv))
    sbytes = (gp.size + lp.size + lq.size) * 8 + args.steps * g.n_bus * 16
    try:
        with open("MEASURED_PEAKS.json") as fh:
            peak = float(json.load(fh)["hbm_gbs"])
    except Exception:
        peak = 6650.0
    print(json.dumps({"workload": "device Sbus rows of {} snapshots ({} buses, {} gens, {} loads) and one Ybus "
                                  "assembly ({} entries, {} branches)".format(args.steps, g.n_bus, gp.shape[1],
                                                                              lp.shape[1], asm.nnz, g.nb_powerline()),
                      "sbus_ms": 1e3 * ts, "sbus_algorithmic_bytes": sbytes, "sbus_gbs": sbytes / ts / 1e9,
                      "sbus_frac": sbytes / ts / 1e9 / peak, "ybus_ms": 1e3 * ty, "peak_gbs": peak}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
