"""The request loop (b200ode_server_*, b200ode_submit, b200ode_poll) on the GPU.

Every result is compared bitwise with the synchronous entry point on the same
cells: each cell runs on its own warp (or group of lanes) with the same kernel
whatever else is in flight, so a request's result is the same alone and in a
mix of concurrent requests of other sizes, mechanisms and step lengths.
"""
import numpy as np
import pytest

from hpc_ode_b200 import native, workloads as W

pytestmark = pytest.mark.gpu


def _req(wl, n, seed, dt=None):
    b = W.make(wl, n, seed=seed)
    if dt is not None:
        b.dt = dt
    return b


def _sync(b):
    s = native.Solver(b.mech)
    T, Y = b.T.copy(), np.ascontiguousarray(b.Y.copy())
    st, _, _ = s.integrate(T, Y, b.P, b.dt)
    s.close()
    return T, Y, st


def _same(T1, Y1, T2, Y2):
    assert np.array_equal(T1, T2)
    assert np.array_equal(Y1, Y2)


def _submit(srv, b, P=None):
    T, Y = b.T.copy(), np.ascontiguousarray(b.Y.copy())
    rid = srv.submit(b.mech, T, Y, b.P if P is None else P, b.dt)
    return rid, T, Y


def test_result_same_alone_and_in_mix():
    a = _req("gri_32k", 1500, 31)
    mix = [_req("h2_1024", 3000, 32, dt=1e-4), _req("gri_32k", 600, 33, dt=1e-5),
           _req("h2_1024", 200, 34, dt=1e-5), _req("gri_1m", 900, 35)]
    srv = native.Server(max_inflight=4)
    try:
        rid, Ta, Ya = _submit(srv, a)
        st_a, info_a = srv.poll(rid, -1)
        assert (st_a == 0).all() and info_a["n_cells"] == 1500 and info_a["latency_ms"] > 0
        # the same request again, submitted together with four others
        ids = [_submit(srv, b) for b in mix[:2]]
        rid2, Ta2, Ya2 = _submit(srv, a)
        ids += [_submit(srv, b) for b in mix[2:]]
        st_a2, _ = srv.poll(rid2, -1)
        assert (st_a2 == 0).all()
        _same(Ta2, Ya2, Ta, Ya)
        for (r, T, Y), b in zip(ids, mix):
            st, info = srv.poll(r, -1)
            Ts, Ys, sts = _sync(b)
            assert np.array_equal(st, sts)
            _same(T, Y, Ts, Ys)
        rep = srv.report()
        assert rep["completed"] == 6 and rep["failed_requests"] == 0
        assert rep["max_concurrent"] >= 2          # requests overlapped on the GPU
        assert rep["cells_completed"] == 1500 * 2 + sum(b.ncells for b in mix)
        assert 0 < rep["p50_latency_ms"] <= rep["p99_latency_ms"] <= rep["max_latency_ms"]
    finally:
        srv.close()
    # alone through the synchronous entry point, too
    Ts, Ys, _ = _sync(a)
    _same(Ta, Ya, Ts, Ys)


def test_admission_by_device_footprint():
    """A budget that holds one GRI request at a time still completes every
    request (one after the other); a request larger than the budget is refused."""
    reqs = [_req("gri_32k", 800, 40 + i) for i in range(3)]
    probe = native.Server(max_inflight=4)
    try:
        rid, _, _ = _submit(probe, reqs[0])
        _, info = probe.poll(rid, -1)
    finally:
        probe.close()
    fp = info["footprint_bytes"]
    srv = native.Server(hbm_budget_bytes=int(fp * 1.5), max_inflight=4)
    try:
        subs = [_submit(srv, b) for b in reqs]
        for (r, T, Y), b in zip(subs, reqs):
            st, _ = srv.poll(r, -1)
            Ts, Ys, sts = _sync(b)
            assert np.array_equal(st, sts)
            _same(T, Y, Ts, Ys)
        rep = srv.report()
        assert rep["max_concurrent"] == 1 and rep["completed"] == 3
        assert rep["peak_bytes"] <= rep["budget_bytes"]
        big = _req("gri_32k", 200000, 49)
        with pytest.raises(native.B200Error) as e:
            _submit(srv, big)
        assert e.value.code == 1
    finally:
        srv.close()


def test_chunked_request_matches_synchronous_path():
    """A request larger than chunk_cells runs as consecutive launches (here
    3 chunks of at most 512 cells, with small requests between them); its
    results, statuses and summed step totals equal the synchronous call's, and
    it holds one chunk's device footprint."""
    big = _req("gri_32k", 1300, 70)
    small = [_req("h2_1024", 100, 71 + i, dt=1e-5) for i in range(3)]
    s = native.Solver(big.mech)
    Ts, Ys = big.T.copy(), np.ascontiguousarray(big.Y.copy())
    sts, stats, _ = s.integrate(Ts, Ys, big.P, big.dt)
    s.close()
    srv = native.Server(max_inflight=4, chunk_cells=512)
    try:
        rid, T, Y = _submit(srv, big)
        subs = [_submit(srv, b) for b in small]
        st, info = srv.poll(rid, -1)
        assert np.array_equal(st, sts)
        _same(T, Y, Ts, Ys)
        assert info["n_cells"] == 1300 and info["n_failed"] == 0 and info["total_nst"] > 0
        assert (info["total_nst"], info["total_nni"]) == (stats["total_nst"], stats["total_nni"])
        for (r, Tb, Yb), b in zip(subs, small):
            stb, _ = srv.poll(r, -1)
            Tr, Yr, str_ = _sync(b)
            assert np.array_equal(stb, str_)
            _same(Tb, Yb, Tr, Yr)
    finally:
        srv.close()
    one = native.Server(max_inflight=1, chunk_cells=512)
    try:
        rid, _, _ = _submit(one, _req("gri_32k", 512, 79))
        _, info512 = one.poll(rid, -1)
    finally:
        one.close()
    assert info["footprint_bytes"] == info512["footprint_bytes"]


def test_stream_of_small_requests_reports_latency():
    rng = np.random.default_rng(7)
    srv = native.Server(max_inflight=4)
    try:
        subs = []
        for i in range(24):
            n = int(rng.integers(16, 400))
            b = _req("h2_1024" if rng.random() < 0.6 else "gri_32k", n, 100 + i,
                     dt=float(rng.choice([1e-5, 1e-4])))
            subs.append((_submit(srv, b), b))
        for (r, T, Y), b in subs:
            st, info = srv.poll(r, -1)
            assert (st == 0).all() and info["n_failed"] == 0
        rep = srv.report()
        assert rep["completed"] == 24 and rep["cells_per_sec"] > 0
        assert rep["p50_latency_ms"] <= rep["p99_latency_ms"]
        # spot-check two results against the synchronous path
        for (r, T, Y), b in (subs[0], subs[-1]):
            Ts, Ys, _ = _sync(b)
            _same(T, Y, Ts, Ys)
    finally:
        srv.close()


def test_poll_not_ready_and_unknown_id():
    srv = native.Server(max_inflight=1)
    try:
        b = _req("gri_32k", 2000, 60)
        r, T, Y = _submit(srv, b)
        first = srv.poll(r, 0)               # almost certainly still running
        if first is None:
            assert srv.poll(r, -1) is not None
        with pytest.raises(native.B200Error):
            srv.poll(r, 0)                   # already retired
    finally:
        srv.close()
