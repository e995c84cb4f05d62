"""The oracle's branch-flow restatement on known answers (CPU): a lossless line carries the same
active power out of one end as into the other, amps follow |S| / (sqrt(3) |V| kV), a case with
zero voltages gives NaN amps and 0 MW, out-of-service branches stay 0 and clean_flows zeroes
removed branches only where finite (ContingencyAnalysis.cpp:237-250)."""
import numpy as np

from oracle.flows import branch_flows


def test_lossless_line_and_units():
    x = 0.1
    ys = 1.0 / (1j * x)
    V = np.array([[1.0 + 0.0j, 0.98 * np.exp(-0.05j)]])
    sn, kv = 100.0, 138.0
    a1, p1 = branch_flows(V, [0], [1], [ys], [-ys], [kv], [True], sn)
    a2, p2 = branch_flows(V, [1], [0], [ys], [-ys], [kv], [True], sn)
    assert abs(p1[0, 0] + p2[0, 0]) < 1e-9 * abs(p1[0, 0])
    # P = |V1||V2| sin(d) / x, in MW
    assert abs(p1[0, 0] - sn * 0.98 * np.sin(0.05) / x) < 1e-9
    S = V[0, 0] * np.conj(ys * V[0, 0] - ys * V[0, 1]) * sn
    assert abs(a1[0, 0] - abs(S) / (np.sqrt(3.0) * kv)) < 1e-12


def test_zero_rows_status_and_cleaning():
    ys = 1.0 / (0.01 + 0.1j)
    V = np.array([[1.0, 0.99 * np.exp(-0.02j), 0.97 * np.exp(-0.04j)], [0.0, 0.0, 0.0]], dtype=np.complex128)
    fr, to = [0, 1, 0], [1, 2, 2]
    yff, yft = [ys] * 3, [-ys] * 3
    kv = [138.0] * 3
    status = [True, True, False]
    a, p = branch_flows(V, fr, to, yff, yft, kv, status, 1.0, removed=[[1], [0]])
    assert a[0, 1] == 0.0 and p[0, 1] == 0.0  # removed branch of case 0
    assert np.isfinite(a[0, 0]) and a[0, 0] > 0
    assert np.all(a[:, 2] == 0) and np.all(p[:, 2] == 0)  # out of service
    assert np.isnan(a[1, 0]) and np.isnan(a[1, 1]) and np.all(p[1] == 0)  # zero voltages; NaN stays
