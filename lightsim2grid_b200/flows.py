"""Branch flows of batches of power-flow results, on the GPU.

The reference computes, after a batch, the current magnitude (kA) and the active power (MW) at
the from side of every branch for every case or snapshot
(``BaseBatchSolverSynch::compute_amps_flows`` / ``compute_active_power_flows``,
``src/batch_algorithm/BaseBatchSolverSynch.hpp:87-192``), then zeroes each contingency's
removed branches (``ContingencyAnalysis::clean_flows``,
``src/batch_algorithm/ContingencyAnalysis.cpp:237-250``).  Here one kernel does both
(``pf_flows_device``); ``flows_host`` runs it from host arrays.

``python -m lightsim2grid_b200.flows`` measures the kernel on the device-resident results of
the 2,848-bus N-1 batch (3,050 cases x 3,776 branches) against the HBM roofline.
"""
import argparse
import json
import sys

import numpy as np

from . import _native as nat


class BranchSet:
    """A grid's branches as the flow kernel reads them (host arrays; ``device`` copies them)."""

    def __init__(self, grid):
        y_ff, y_ft, _, _ = grid.branch_admittances()
        self.nbr = int(grid.line_from.size)
        self.n = int(grid.n_bus)
        self.from_ = nat.as_i32(grid.line_from)
        self.to = nat.as_i32(grid.line_to)
        self.yff = nat.as_c128(y_ff).ravel().copy()
        self.yft = nat.as_c128(y_ft).ravel().copy()
        self.vn_kv_from = nat.as_f64(np.asarray(grid.bus_vn_kv)[grid.line_from])
        self.status = np.ascontiguousarray(np.asarray(grid.line_status, dtype=np.uint8))
        self.sn_mva = float(grid.sn_mva)

    def host_struct(self):
        return nat.PfBranchSet(nbr=self.nbr, from_=self.from_.ctypes.data, to=self.to.ctypes.data,
                               yff_ri=self.yff.ctypes.data, yft_ri=self.yft.ctypes.data,
                               vn_kv_from=self.vn_kv_from.ctypes.data, status=self.status.ctypes.data,
                               sn_mva=self.sn_mva)

    def device(self, device):
        """(PfBranchSet of device pointers, tensors that keep them alive)."""
        import torch

        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
        keep = [t(self.from_), t(self.to), t(self.yff.view(np.float64)), t(self.yft.view(np.float64)),
                t(self.vn_kv_from), t(self.status)]
        st = nat.PfBranchSet(nbr=self.nbr, from_=keep[0].data_ptr(), to=keep[1].data_ptr(),
                             yff_ri=keep[2].data_ptr(), yft_ri=keep[3].data_ptr(), vn_kv_from=keep[4].data_ptr(),
                             status=keep[5].data_ptr(), sn_mva=self.sn_mva)
        return st, keep


def outage_lists(removed):
    """CSR (ptr, ids) of each row's removed branches from a list of lists (None: none)."""
    if removed is None:
        return None, None
    ptr = np.zeros(len(removed) + 1, np.int32)
    for i, lst in enumerate(removed):
        ptr[i + 1] = ptr[i] + len(lst)
    ids = np.asarray([b for lst in removed for b in lst], np.int32)
    return ptr, (ids if ids.size else np.zeros(1, np.int32))


def flows_host(branches, V, removed=None, amps=True, power=True):
    """Flows of result rows ``V`` (rows x n complex, host) on the GPU.  ``removed``: per row, the
    branch ids zeroed where finite (clean_flows).  Returns (amps or None, p_mw or None)."""
    lib = nat.load()
    V = np.ascontiguousarray(np.asarray(V, dtype=np.complex128))
    if V.ndim != 2 or V.shape[1] != branches.n:
        raise RuntimeError("V must be (rows, {}) complex".format(branches.n))
    rows = V.shape[0]
    a = np.empty((rows, branches.nbr)) if amps else None
    p = np.empty((rows, branches.nbr)) if power else None
    ptr, ids = outage_lists(removed)
    st = branches.host_struct()
    rc = lib.pf_flows_host(nat.ctypes.byref(st), branches.n, rows, V.ctypes.data,
                           None if ptr is None else ptr.ctypes.data, None if ids is None else ids.ctypes.data,
                           None if a is None else a.ctypes.data, None if p is None else p.ctypes.data)
    nat.check(rc, "pf_flows_host", lib)
    return a, p


def flows_device(branch_struct, n, V_ptr, rows, stream, v_stride=None, map_ptr=0, errs_ptr=0, out_ptr=0,
                 out_ids=0, amps_ptr=0, p_ptr=0):
    """The kernel on device-resident data (all arguments device pointers); asynchronous."""
    lib = nat.load()
    rc = lib.pf_flows_device(nat.ctypes.byref(branch_struct), int(n), int(rows), V_ptr,
                             int(n if v_stride is None else v_stride), map_ptr or None, errs_ptr or None,
                             out_ptr or None, out_ids or None, amps_ptr or None, p_ptr or None, stream)
    nat.check(rc, "pf_flows_device", lib)


def main(argv=None):
    ap = argparse.ArgumentParser(description="branch flows of the 2,848-bus N-1 batch on the device")
    ap.add_argument("--grid", default="grid2848")
    ap.add_argument("--repeat", type=int, default=10)
    args = ap.parse_args(argv)
    import torch

    from . import synthetic
    from .multi import GridCases

    dev = torch.device("cuda:0")
    g, _ = synthetic.make_named_grid(args.grid)
    c = GridCases("n1", g, np.arange(g.nb_powerline()), dev, precision=1)
    k = c.ninst
    jf = torch.arange(k, dtype=torch.int32, device=dev)
    jc = torch.ones(k, dtype=torch.int32, device=dev)
    b = c.batch
    b2 = nat.PfDeviceBatch(n_inst=k, V0=b.V0, v0_stride=0, Sbus=b.Sbus, sbus_stride=0, ovr_ptr=b.ovr_ptr,
                           ovr_pos=b.ovr_pos, ovr_val=b.ovr_val, max_iter=10, tol=1e-8, chain=0,
                           job_first=jf.data_ptr(), job_count=jc.data_ptr(), njobs=k, Vout=b.Vout, iters=b.iters,
                           errs=b.errs)
    st = torch.cuda.current_stream()
    nat.check(c.plan._lib.pf_batch_device(c.plan.handle, nat.ctypes.byref(b2), st.cuda_stream), "pf_batch_device")
    torch.cuda.synchronize()
    # rows in case order: map case -> compact instance (-1 islanded); removed branch per case
    cmap = np.full(len(c.branches), -1, np.int32)
    cmap[np.flatnonzero(c.solvable)] = np.arange(k, dtype=np.int32)
    ptr, ids = outage_lists([[int(x)] for x in c.branches])
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    dmap, dptr, dids = t(cmap), t(ptr), t(ids)
    bs = BranchSet(g)
    bst, keep = bs.device(dev)
    rows = len(c.branches)
    A = torch.empty(rows * bs.nbr, dtype=torch.float64, device=dev)
    P = torch.empty(rows * bs.nbr, dtype=torch.float64, device=dev)

    def launch():
        flows_device(bst, bs.n, b.Vout, rows, st.cuda_stream, map_ptr=dmap.data_ptr(), errs_ptr=b.errs,
                     out_ptr=dptr.data_ptr(), out_ids=dids.data_ptr(), amps_ptr=A.data_ptr(), p_ptr=P.data_ptr())

    launch()
    torch.cuda.synchronize()
    flush = torch.empty(256 << 20 >> 2, dtype=torch.float32, device=dev)
    ts = []
    for _ in range(args.repeat):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        launch()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1) * 1e-3)
    sec = float(np.median(ts))
    # algorithmic bytes: each solved row's voltages read once, both outputs written, the
    # branch data and row maps read once
    solved = int((cmap >= 0).sum())
    abytes = solved * bs.n * 16 + rows * bs.nbr * 16 + bs.nbr * (4 + 4 + 16 + 16 + 8 + 1) + rows * 12
    try:
        with open("MEASURED_PEAKS.json") as fh:
            peak = float(json.load(fh)["hbm_gbs"])
    except Exception:
        peak = 6650.0
    out = {"workload": "branch flows (amps and MW, clean_flows) of the {} N-1 results: {} cases x {} branches"
                       .format(args.grid, rows, bs.nbr),
           "ms": 1e3 * sec, "rows_per_s": rows / sec, "algorithmic_bytes": abytes,
           "achieved_gbs": abytes / sec / 1e9, "peak_gbs": peak, "frac": abytes / sec / 1e9 / peak}
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
