"""The serving loop's request generator (CPU): seeded Poisson arrivals, the grid mix, power
flows with injections scaled within +-10 % and N-1 batches of 8 to 64 distinct branches."""
import numpy as np

from lightsim2grid_b200.serving import PF, make_requests


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
