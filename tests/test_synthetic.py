"""Seeded synthetic grids: sizes, determinism, conventions and base-case solvability."""
import numpy as np
import pytest

from lightsim2grid_b200 import synthetic
from oracle.oracle import OracleNR


def test_sizes_and_determinism():
    for name, (n, nbr, npv) in synthetic.GRID_SIZES.items():
        if n > 3000:
            continue
        g1, V1 = synthetic.make_named_grid(name)
        g2, V2 = synthetic.make_named_grid(name)
        assert g1.n_bus == n and g1.nb_powerline() == nbr and len(g1.get_pv()) == npv
        assert np.array_equal(g1.line_from, g2.line_from) and np.array_equal(V1, V2)
        Y = g1.get_Ybus()
        assert Y.nnz == n + 2 * nbr  # no parallel branches
        assert abs(np.abs(V1[g1.get_pq()]).min() - 0.95) < 0.05 and np.abs(V1).max() <= 1.06 + 1e-12


def test_ybus_conventions():
    g, _ = synthetic.make_named_grid("grid14")
    Y = g.get_Ybus().toarray()
    br = 3
    f, t = g.line_from[br], g.line_to[br]
    ys = 1.0 / (g.line_r[br] + 1j * g.line_x[br])
    assert np.isclose(Y[f, t], -ys) and np.isclose(Y[t, f], -ys)
    coeffs = g.branch_coeffs([br])
    assert [(c.row_id, c.col_id) for c in coeffs] == [(f, f), (t, t), (f, t), (t, f)]
    assert np.isclose(coeffs[0].value, ys + 0.5 * g.line_h[br])


@pytest.mark.parametrize("name", ["grid14", "grid118", "grid300", "grid1354", "grid2848"])
def test_base_case_converges_to_the_drawn_state(name):
    g, Vt = synthetic.make_named_grid(name)
    s = OracleNR(False)
    assert s.compute_pf(g.get_Ybus(), g.flat_start(), g.get_Sbus(), g.get_slack_ids(), g.get_slack_weights(),
                        g.get_pv(), g.get_pq(), 10, 1e-8)
    assert np.abs(s.get_V() - Vt).max() < 1e-8


def test_time_series_profiles():
    m = synthetic.ar1_profiles(48, 5, seed=3)
    assert m.shape == (48, 5)
    assert 0.7 < m.min() and m.max() < 1.3
