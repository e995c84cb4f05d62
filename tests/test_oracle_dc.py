"""The DC oracle on known answers (CPU): on a lossless 3-bus ring the angles solve B theta = P
exactly, the slack keeps its start angle, magnitudes are the start magnitudes, and slacks after
the first behave as PV buses (BaseAlgo.hpp:201-216)."""
import numpy as np
from scipy import sparse

from oracle.dc import dc_pf


def _ring(x):
    n = 3
    Y = np.zeros((n, n), complex)
    for (a, b), xx in zip(((0, 1), (1, 2), (0, 2)), x):
        y = 1.0 / xx
        Y[a, a] += y
        Y[b, b] += y
        Y[a, b] -= y
        Y[b, a] -= y
    return sparse.csc_matrix(Y)


def test_ring_angles_solve_b_theta():
    Y = _ring([0.1, 0.2, 0.25])
    V = np.array([1.02 * np.exp(0.1j), 1.0, 0.98])
    S = np.array([0.0, -0.5, 0.3])
    Vd, ok = dc_pf(Y, V, S, [0], [1], [2])
    assert ok
    theta = np.angle(Vd) - 0.1
    B = Y.toarray().real
    assert np.allclose(B[1:, 1:] @ theta[1:], S.real[1:], atol=1e-12)
    assert np.allclose(np.abs(Vd), np.abs(V)) and abs(np.angle(Vd[0]) - 0.1) < 1e-15


def test_second_slack_counts_as_pv():
    Y = _ring([0.1, 0.2, 0.25])
    V = np.ones(3, complex)
    S = np.array([0.0, -0.5, 0.3])
    V1, ok1 = dc_pf(Y, V, S, [0, 2], [], [1])
    V2, ok2 = dc_pf(Y, V, S, [0], [2], [1])
    assert ok1 and ok2 and np.allclose(V1, V2)
