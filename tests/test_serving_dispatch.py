"""Admission and bookkeeping of the serving loop, on the CPU with a fake executor: FIFO
admission, the device-memory budget and the slot limit are never exceeded, every request
completes, requests larger than the whole budget are rejected, and the Poisson request
generator is seeded and shaped as specified."""
import numpy as np

from lightsim2grid_b200.serving import N1, PF, Dispatcher, Request, latency_stats, make_requests


class FakeClock:
    def __init__(self, step=1e-4):
        self.t, self.step = 0.0, step

    def __call__(self):
        self.t += self.step
        return self.t


class FakeExecutor:
    """Request r needs r.ninst * 1000 bytes and runs for 2 ms of fake time per instance."""

    def __init__(self, clock, budget_check):
        self.clock = clock
        self.running = {}
        self.order = []
        self.check = budget_check

    def bytes_needed(self, req):
        req.ninst = 1 if req.kind == PF else len(req.branches)
        return req.ninst * 1000

    def reserve(self, req):
        return True

    def launch(self, req):
        self.order.append(req.rid)
        self.running[req.rid] = self.clock.t + 2e-3 * req.ninst
        self.check()

    def poll(self):
        fin = [rid for rid, t in self.running.items() if self.clock.t >= t]
        for rid in fin:
            del self.running[rid]
        return fin


def _requests(n, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        if rng.random() < 0.5:
            out.append(Request(i, "g", PF, i * 1e-3, scale=np.ones(4)))
        else:
            out.append(Request(i, "g", N1, i * 1e-3, branches=np.arange(int(rng.integers(1, 9)))))
    return out


def test_budget_slots_fifo_and_completion():
    clock = FakeClock()
    state = {}

    def check():
        d = state["d"]
        assert d.in_use <= d.budget
        assert len(d.inflight) <= d.slots

    ex = FakeExecutor(clock, check)
    d = Dispatcher(ex, hbm_budget=12000, slots=3)
    state["d"] = d
    reqs = _requests(60)
    done = d.run(reqs, clock=clock, realtime=True)
    assert len(done) == 60 and not d.rejected
    assert ex.order == sorted(ex.order)  # FIFO admission
    assert d.peak_bytes <= 12000 and d.peak_inflight <= 3
    assert d.in_use == 0 and not d.inflight
    for r in done:
        assert r.t_admit >= r.arrival - 1e-12 and r.t_done >= r.t_admit
    st = latency_stats(done)
    assert st["requests"] == 60 and st["p99_ms"] >= st["p50_ms"] > 0


def test_oversize_request_is_rejected():
    clock = FakeClock()
    ex = FakeExecutor(clock, lambda: None)
    d = Dispatcher(ex, hbm_budget=5000, slots=4)
    reqs = [Request(0, "g", N1, 0.0, branches=np.arange(8)), Request(1, "g", PF, 0.0, scale=np.ones(3))]
    done = d.run(reqs, clock=clock, realtime=False)
    assert [r.rid for r in done] == [1]
    assert [r.rid for r in d.rejected] == [0]


def test_request_generator_is_seeded_and_shaped():
    grids = {"a": 14, "b": 118}
    nbr = {"a": 20, "b": 186}
    r1 = make_requests(grids, rate=2000, duration=0.5, seed=3, branches_of=nbr)
    r2 = make_requests(grids, rate=2000, duration=0.5, seed=3, branches_of=nbr)
    assert len(r1) == len(r2) and 800 < len(r1) < 1200
    assert all(a.arrival == b.arrival and a.kind == b.kind and a.grid == b.grid for a, b in zip(r1, r2))
    arr = np.array([r.arrival for r in r1])
    assert np.all(np.diff(arr) > 0) and arr[-1] < 0.5
    for r in r1:
        if r.kind == PF:
            assert r.scale.size == grids[r.grid] and np.all(np.abs(r.scale - 1) <= 0.1)
        else:
            k = r.branches.size
            assert min(8, nbr[r.grid]) <= k <= 64 and np.unique(r.branches).size == k
            assert r.branches.max() < nbr[r.grid]
    frac_pf = np.mean([r.kind == PF for r in r1])
    assert 0.4 < frac_pf < 0.6


def test_device_arena_first_fit_and_coalescing():
    """The serving arena on a CPU buffer: random allocations never overlap, stay aligned and
    inside the arena, and freeing everything coalesces back to one hole."""
    from lightsim2grid_b200.serving import DeviceArena

    a = DeviceArena(1 << 20, "cpu")
    rng = np.random.default_rng(4)
    live = {}
    for step in range(2000):
        if live and (rng.random() < 0.45 or len(live) > 40):
            key = list(live)[int(rng.integers(len(live)))]
            o, n = live.pop(key)
            a.release(o, n)
        else:
            n = int(rng.integers(1, 60000))
            o = a.alloc(n)
            if o is None:
                assert a.free_bytes() < 1 << 20
                continue
            assert o % 256 == 0 and o + n <= a.size
            for (p, m) in live.values():
                assert o + n <= p or p + m <= o
            live[step] = (o, n)
        # holes sorted, disjoint, coalesced
        h = a.holes
        assert all(h[i][0] + h[i][1] < h[i + 1][0] for i in range(len(h) - 1))
    for o, n in live.values():
        a.release(o, n)
    assert a.holes == [(0, a.size)]
