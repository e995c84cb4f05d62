"""Host-side pieces without a GPU: the autotuner's fingerprint and choice cache, the bench's
roofline and error arithmetic, and the oracle's threaded N-1 batch and chunked time series."""
import json

import numpy as np

from conftest import grid_problem


def test_autotune_fingerprint_and_cache(tmp_path, monkeypatch):
    from lightsim2grid_b200 import autotune, synthetic

    g = synthetic.make_named_grid("grid118")[0]
    k1 = autotune._fingerprint(g, 1, np.arange(10), "x")
    assert k1 == autotune._fingerprint(g, 1, np.arange(10), "x")
    assert k1 != autotune._fingerprint(g, 0, np.arange(10), "x")  # precision
    assert k1 != autotune._fingerprint(g, 1, np.arange(11), "x")  # sample
    path = tmp_path / "tune.json"
    monkeypatch.setenv("LIGHTSIM2GRID_B200_TUNE_CACHE", str(path))
    monkeypatch.setattr(autotune, "_CACHE", {})
    value = {"best": {"ordering": 0, "placement": 1}, "table": []}
    autotune._cache_put(k1, value)
    assert json.loads(path.read_text())[k1] == value
    monkeypatch.setattr(autotune, "_CACHE", {})  # a new process: read back from the file
    assert autotune._cache_get(k1) == value
    assert autotune._cache_get("absent") is None


def test_autotune_candidates_cover_the_schedule_knobs():
    from lightsim2grid_b200 import autotune

    c = autotune.n1_candidates(5194, 2848)
    keys = {k for d in c for k in d}
    assert {"ordering", "placement", "threads", "batch_layout"} <= keys
    assert any(d.get("level_slack") == 4 for d in c)
    assert any(d.get("batch_layout") == 2 for d in c)
    assert all(d.get("batch_layout") == 1 for d in autotune.n1_candidates(180, 118))


def test_bench_arithmetic():
    import bench

    info = {"n": 2848, "m": 5194, "nnz_j": 34986, "nnz_lu": 48682}
    total, per_it = bench._algorithmic_bytes(info, np.array([3, 2]), 4)
    assert per_it == 80 * 2848 + 32 * 5194 + 2 * 4 * (34986 + 48682) == 1063392
    assert total == 5 * per_it + 2 * (64 * 2848 + 8 * 5194)
    a = np.array([[1.0 + 0.0j, 0.0 + 1.0j]])
    b = a * np.exp(1j * 1e-9)
    assert abs(bench._dv(a, b)[0] - 1e-9) < 1e-15
    st = bench._err_stats(np.array([1e-12, 2e-12, 3e-10]))
    assert st["max"] == 3e-10 and st["count"] == 3
    # the roofline names the kernel variant the library launches for a thread count
    assert [bench._launch_bound(t) for t in (128, 512, 544, 640, 672, 768)] == [512, 512, 640, 640, 768, 768]


def test_threaded_oracle_batch_matches_sequential_slices():
    """The oracle's N-1 loop on several host threads (contiguous slices, one computer each) gives
    each slice the results of that slice run alone."""
    from oracle.oracle import ContingencyBatch, OracleNR, contingency_analysis

    c = grid_problem("grid118")
    o = OracleNR(False)
    assert o.compute_pf(c["Ybus"], c["V0"], c["Sbus"], c["ref"], c["weights"], c["pv"], c["pq"], 10, 1e-8)
    Vn = o.get_V()
    g = c["grid"]
    coeffs = [g.branch_coeffs([b]) for b in range(g.nb_powerline())]
    b = ContingencyBatch(c["Ybus"], c["Sbus"], Vn, c["ref"], c["weights"], c["pv"], c["pq"], coeffs)
    ok, V, conv, it, err, _ = b.run(3)
    assert ok
    edges = (np.arange(4) * len(coeffs)) // 3
    for lo, hi in zip(edges[:-1], edges[1:]):
        _, Vs, cs, its, errs = contingency_analysis(c["Ybus"], c["Sbus"], Vn, c["ref"], c["weights"], c["pv"],
                                                    c["pq"], coeffs[lo:hi])
        assert np.array_equal(V[lo:hi], Vs) and np.array_equal(conv[lo:hi], cs)
        assert np.array_equal(it[lo:hi], its) and np.array_equal(err[lo:hi], errs)


def test_chunked_oracle_time_series_is_each_chunks_exact_chain():
    from lightsim2grid_b200 import synthetic
    from lightsim2grid_b200.timeseries import chunk_jobs
    from oracle.oracle import time_series, time_series_chunks

    c = grid_problem("grid118")
    g = c["grid"]
    Sb = g.sbuses_from_injections(*synthetic.time_series_injections(g, 30, seed=3))
    jf, jc = chunk_jobs(30, 4)
    V, conv, it, err = time_series_chunks(c["Ybus"], c["Sbus"], Sb, c["V0"], c["ref"], c["weights"], c["pv"], c["pq"],
                                          jf, jc, threads=2)
    assert conv.all()
    for a, k in zip(jf, jc):
        st, Vk, ck, ik, _ = time_series(c["Ybus"], c["Sbus"], Sb[a:a + k], c["V0"], c["ref"], c["weights"], c["pv"],
                                        c["pq"])
        assert st == 1 and np.array_equal(V[a:a + k], Vk) and np.array_equal(it[a:a + k], ik)
