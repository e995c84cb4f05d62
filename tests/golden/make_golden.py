"""Convert the reference's Newton-Raphson golden vectors into compact fixtures.

The reference ships five zip archives next to its solver tests
(lightsim2grid/tests/case{14,30,118,300,1888}.zip, read by
lightsim2grid/tests/test_KLUSolver.py:49-74 and test_NewtonPF.py).  Each holds a
dense complex ``Ybus.npy``, ``Sbus.npy``, ``V0.npy``, ``pv.npy``, ``pq.npy`` and
the pandapower results ``J_<k>.npy`` / ``V_<k>.npy`` after k iterations.

This script stores the same arrays as sparse CSC triplets in one ``.npz`` per
case (the dense 1888-bus Ybus alone is 57 MB) so that the CPU tests can run
without the reference tree.  Run it from the repository root:

    python tests/golden/make_golden.py /path/to/reference/lightsim2grid/tests
"""
import os
import re
import sys
import zipfile
import io

import numpy as np
from scipy import sparse


def _load(zf, name):
    with zf.open(name) as fh:
        return np.load(io.BytesIO(fh.read()))


def convert(src_dir, dst_dir):
    written = []
    for fname in sorted(os.listdir(src_dir)):
        if not (fname.startswith("case") and fname.endswith(".zip")):
            continue
        with zipfile.ZipFile(os.path.join(src_dir, fname)) as zf:
            names = zf.namelist()
            k = None
            for nm in names:
                m = re.match(r"V_(\d+)\.npy", nm)
                if m:
                    k = int(m.group(1))
            Y = sparse.csc_matrix(_load(zf, "Ybus.npy"))
            Y.sort_indices()
            J = sparse.csc_matrix(_load(zf, "J_{}.npy".format(k)))
            J.sort_indices()
            out = dict(
                Ybus_data=Y.data.astype(np.complex128),
                Ybus_indices=Y.indices.astype(np.int32),
                Ybus_indptr=Y.indptr.astype(np.int32),
                Sbus=_load(zf, "Sbus.npy").astype(np.complex128),
                V0=_load(zf, "V0.npy").astype(np.complex128),
                pv=_load(zf, "pv.npy").astype(np.int32),
                pq=_load(zf, "pq.npy").astype(np.int32),
                V_ref=_load(zf, "V_{}.npy".format(k)).astype(np.complex128),
                J_data=J.data.astype(np.float64),
                J_indices=J.indices.astype(np.int32),
                J_indptr=J.indptr.astype(np.int32),
                J_shape=np.array(J.shape, dtype=np.int64),
                n_iter=np.array(k, dtype=np.int64),
            )
        dst = os.path.join(dst_dir, fname.replace(".zip", ".npz"))
        np.savez_compressed(dst, **out)
        written.append(dst)
    return written


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_golden.py <reference checkout>/lightsim2grid/tests  (the folder holding "
                 "case14.zip ... case1888.zip)")
    src = sys.argv[1]
    dst = os.path.dirname(os.path.abspath(__file__))
    for path in convert(src, dst):
        print(path, os.path.getsize(path))
