"""Shared fixtures.  GPU tests carry ``@pytest.mark.gpu``; the rest run on CPU."""
import glob
import os
import sys

import numpy as np
import pytest
from scipy import sparse

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden_cases():
    """The reference's five NR golden cases (tests/golden/make_golden.py)."""
    out = []
    for f in sorted(glob.glob(os.path.join(GOLDEN, "case*.npz"))):
        d = np.load(f)
        Y = sparse.csc_matrix((d["Ybus_data"], d["Ybus_indices"], d["Ybus_indptr"]))
        n = Y.shape[0]
        pv, pq = d["pv"].astype(np.int64), d["pq"].astype(np.int64)
        ref = np.array(sorted(set(range(n)) - set(pv.tolist()) - set(pq.tolist())), dtype=np.int64)
        w = np.zeros(n)
        w[ref] = 1.0 / len(ref)
        J = sparse.csc_matrix((d["J_data"], d["J_indices"], d["J_indptr"]), shape=tuple(d["J_shape"]))
        out.append(dict(name=os.path.basename(f)[:-4], Ybus=Y, Sbus=d["Sbus"], V0=d["V0"], pv=pv, pq=pq, ref=ref,
                        weights=w, V_ref=d["V_ref"], J_ref=J, n_iter=int(d["n_iter"])))
    return out


def grid_problem(name):
    from lightsim2grid_b200 import synthetic

    g, Vt = synthetic.make_named_grid(name)
    return dict(name=name, grid=g, V_true=Vt, Ybus=g.get_Ybus(), Sbus=g.get_Sbus(), V0=g.flat_start(),
                ref=g.get_slack_ids(), weights=g.get_slack_weights(), pv=g.get_pv(), pq=g.get_pq())


@pytest.fixture(scope="session")
def golden():
    return golden_cases()
