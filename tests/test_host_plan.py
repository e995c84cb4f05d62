"""Host analysis of the engine, checked on CPU: J pattern bit-exact to the reference's
construction (as restated by the oracle), device schedules emulated on the host against
scipy's sparse solve, and input validation."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

from conftest import grid_problem
from oracle.oracle import OracleNR
from lightsim2grid_b200 import _native as nat


def _args(c):
    Y = c["Ybus"].tocsc()
    Y.sort_indices()
    return (Y.shape[0], nat.as_i32(Y.indptr), nat.as_i32(Y.indices), nat.as_c128(Y.data).ravel(),
            nat.as_i32(c["ref"]), nat.as_f64(c["weights"]), nat.as_i32(c["pv"]), nat.as_i32(c["pq"]))


def host_pattern(c, distributed):
    lib = nat.load()
    n, Yp, Yi, Yx, sl, w, pv, pq = _args(c)
    m = nat.ctypes.c_int(0)
    call = lambda a, b, mm: lib.pf_host_jacobian_pattern(
        n, nat.ptr(Yp, nat.i32p), nat.ptr(Yi, nat.i32p), nat.cptr(Yx), nat.ptr(sl, nat.i32p), sl.size,
        nat.ptr(w, nat.f64p), nat.ptr(pv, nat.i32p), pv.size, nat.ptr(pq, nat.i32p), pq.size, int(distributed),
        mm, a, b)
    nz = call(None, None, nat.ctypes.byref(m))
    assert nz > 0, nat.last_error(lib)
    Jp = np.zeros(m.value + 1, np.int32)
    Ji = np.zeros(nz, np.int32)
    call(nat.ptr(Jp, nat.i32p), nat.ptr(Ji, nat.i32p), None)
    return Jp, Ji


def host_schedule_solve(c, V, b, distributed):
    lib = nat.load()
    n, Yp, Yi, Yx, sl, w, pv, pq = _args(c)
    V0 = nat.as_c128(c["V0"]).ravel()
    V = nat.as_c128(V).ravel()
    b = nat.as_f64(b)
    x = np.zeros(b.size)
    info = nat.PfPlanInfo()
    rc = lib.pf_host_schedule_solve(n, nat.ptr(Yp, nat.i32p), nat.ptr(Yi, nat.i32p), nat.cptr(Yx), nat.cptr(V0),
                                    nat.cptr(V), nat.ptr(sl, nat.i32p), sl.size, nat.ptr(w, nat.f64p),
                                    nat.ptr(pv, nat.i32p), pv.size, nat.ptr(pq, nat.i32p), pq.size,
                                    int(distributed), nat.ptr(b, nat.f64p), nat.ptr(x, nat.f64p),
                                    nat.ctypes.byref(info))
    assert rc == 0, nat.last_error(lib)
    return x, info


def _problems(golden):
    out = list(golden)
    for name in ("grid14", "grid118", "grid1354"):
        out.append(grid_problem(name))
    return out


@pytest.mark.parametrize("distributed", [False, True])
def test_jacobian_pattern_bit_exact(golden, distributed):
    for c in _problems(golden):
        o = OracleNR(distributed)
        o.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
        Jo = o.get_J()
        Jp, Ji = host_pattern(c, distributed)
        assert np.array_equal(Jp, Jo.indptr), c["name"]
        assert np.array_equal(Ji, Jo.indices), c["name"]


@pytest.mark.parametrize("distributed", [False, True])
def test_device_schedules_solve_J(golden, distributed):
    """Refactorisation + both substitutions in the device's level order solve J x = b."""
    rng = np.random.default_rng(0)
    for c in _problems(golden):
        o = OracleNR(distributed)
        o.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
        V = o.get_V()
        # oracle J at V: one iteration from V with a dummy Sbus, J of that iteration
        o2 = OracleNR(distributed)
        o2.compute_pf(c["Ybus"], V, V * np.conj(c["Ybus"] @ V) + 1.0, c["ref"], c["weights"], c["pv"], c["pq"], 1,
                      1e-30)
        J = o2.get_J().tocsc()
        b = rng.standard_normal(J.shape[0])
        x, info = host_schedule_solve(c, V, b, distributed)
        xr = spla.spsolve(J, b)
        assert np.abs(x - xr).max() <= 1e-10 * max(1.0, np.abs(xr).max()), c["name"]
        assert info.nnz_j == J.nnz
        assert info.nnz_lu >= info.nnz_j


def test_fill_reducing_order_keeps_fill_low():
    c = grid_problem("grid1354")
    _, info = host_schedule_solve(c, c["V0"], np.ones(2 * len(c["pq"]) + len(c["pv"])), False)
    assert info.nnz_lu < 2.0 * info.nnz_j


def test_default_order_is_shallow():
    """The default elimination order (minimum degree preferring low elimination levels, on 8
    relabellings, each followed by its least-depth equivalent, the shallowest kept) brings the
    refactorisation's dependent levels of the 2848-bus Jacobian to 53 (minimum degree alone: 91;
    without the level preference: 72) with no more fill than minimum degree (48,870 LU entries)."""
    c = grid_problem("grid2848")
    m = 2 * len(c["pq"]) + len(c["pv"])
    b = np.linspace(1.0, 2.0, m)
    x, info = host_schedule_solve(c, c["V0"], b, False)
    assert info.levels_refactor <= 55
    assert info.nnz_lu <= 48870
    assert np.all(np.isfinite(x))


def test_packed_programs_are_placed_for_few_bank_conflicts():
    """The packed factor program of the 2848-bus plan (FP32, LU in shared memory) makes about
    37k shared-memory wavefronts per run under the bank model it is placed for (the longest-first
    placement made 52k on the programs of the order without the level preference), and no
    placement can go below one wavefront per operand and warp-slot."""
    c = grid_problem("grid2848")
    m = 2 * len(c["pq"]) + len(c["pv"])
    _, info = host_schedule_solve(c, c["V0"], np.ones(m), False)
    floor = 5 * (info.flops_refactor + info.nnz_lu) // 32  # operations (updates + pushes) / warp
    assert floor < info.smem_wavefronts_factor <= 39000
    assert 0 < info.smem_wavefronts_backward <= 8000
    assert 0 < info.smem_wavefronts_forward <= 10500


def test_invalid_inputs_are_rejected():
    lib = nat.load()
    c = grid_problem("grid14")
    n, Yp, Yi, Yx, sl, w, pv, pq = _args(c)
    bad_pq = pq.copy()
    bad_pq[0] = pv[0]  # a bus both PV and PQ
    rc = lib.pf_host_jacobian_pattern(n, nat.ptr(Yp, nat.i32p), nat.ptr(Yi, nat.i32p), nat.cptr(Yx),
                                      nat.ptr(sl, nat.i32p), sl.size, nat.ptr(w, nat.f64p), nat.ptr(pv, nat.i32p),
                                      pv.size, nat.ptr(bad_pq, nat.i32p), bad_pq.size, 0, None, None, None)
    assert rc != 0 and "PQ" in nat.last_error(lib)
    Yi2 = Yi.copy()
    Yi2[0], Yi2[1] = Yi[1], Yi[0]  # unsorted column
    rc = lib.pf_host_jacobian_pattern(n, nat.ptr(Yp, nat.i32p), nat.ptr(Yi2, nat.i32p), nat.cptr(Yx),
                                      nat.ptr(sl, nat.i32p), sl.size, nat.ptr(w, nat.f64p), nat.ptr(pv, nat.i32p),
                                      pv.size, nat.ptr(pq, nat.i32p), pq.size, 0, None, None, None)
    assert rc != 0 and "canonical" in nat.last_error(lib)
