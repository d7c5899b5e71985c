"""GPU parity tests through the C ABI (libb200ode.so) against the CPU oracle and
the reference's golden vectors.

Tolerances (float work, as the path computes in FP64 with an FP32 Newton matrix
in mixed mode):
  * chemistry RHS vs reference pyJac: |d| <= 1e-12 * (|ref| + scale), scale =
    sum of |forward| + |reverse| contributions (cancellation-aware);
  * Jacobian (FP64 form) vs reference pyJac: 1e-10 relative where |J| >
    1e-8 max|J| (pyJac's dTdot/dT excepted: it is checked against finite
    differences of the reference RHS instead); FP32 form (FP32 accumulation): 1e-4;
  * integration vs the CPU oracle at the same tolerances (rtol 1e-6, atol
    1e-10): |dT|/T <= 1e-5 for every cell; per species |dY| <= max(1e-4 |Y|,
    1e-10) for at least 99 % of entries (batches of 500+ entries), and every
    entry that misses it within the integration error of a rtol-1e-6 CVODE
    integration: |Y - Y_true| <= 10 (|Y_cpu - Y_true| + rtol |Y_true| + atol)
    against the FP64 oracle at rtol 1e-10 (the CPU integrator itself misses the
    per-entry gate against that solution for 2-4 % of entries).
"""
import numpy as np
import pytest

from conftest import y_ok
from hpc_ode_b200 import native, workloads as W

pytestmark = pytest.mark.gpu

GATE_T = 1e-5


def run_gpu(b, precision, persistent=1, use_graph=0, counters=False, **kw):
    s = native.Solver(b.mech, precision=precision, persistent=persistent, use_graph=use_graph, **kw)
    T = b.T.copy()
    Y = np.ascontiguousarray(b.Y.copy())
    st, stats, cnt = s.integrate(T, Y, b.P, b.dt, counters=counters)
    s.close()
    return T, Y, st, stats, cnt


def compare(b, T, Y, yo, label, oracle=None, min_frac=0.99):
    dT = np.abs(T - yo[:, 0]) / yo[:, 0]
    Yg = Y[:-1].T
    ok = y_ok(Yg, yo[:, 1:])
    assert dT.max() <= GATE_T, (label, dT.max())
    if ok.size >= 500:
        assert ok.mean() >= min_frac, (label, ok.mean())
    if not ok.all():
        assert oracle is not None, (label, "entries outside the gate and no oracle to bound them")
        cells = np.nonzero(~ok.all(axis=1))[0]
        sub = b.subset(cells)
        yt, st = oracle.bdf(sub.mech, sub.state_rows(), sub.P, sub.dt, rtol=1e-10, atol=1e-14, threads=8)
        assert (st["status"] == 0).all()
        true = yt[:, 1:]
        bound = 10.0 * (np.abs(yo[cells, 1:] - true) + W.RTOL * np.abs(true) + W.ATOL)
        miss = ~ok[cells]
        err = np.abs(Yg[cells] - true)
        assert (err[miss] <= bound[miss]).all(), (label, float((err[miss] / bound[miss]).max()))
    return dT, ok


def test_rhs_matches_reference_golden(oracle, golden_chem):
    y, P, ref = golden_chem["y"], golden_chem["P"], golden_chem["dydt"]
    T = np.ascontiguousarray(y[:, 0])
    Yfull = np.concatenate([y[:, 1:], (1.0 - y[:, 1:].sum(axis=1))[:, None]], axis=1)
    Y = np.ascontiguousarray(Yfull.T)
    s = native.Solver("gri30", precision=native.B200ODE_FP64)
    dT, dY = s.eval_rhs(T, Y, P)
    s.close()
    got = np.concatenate([dT[:, None], dY.T], axis=1)
    for i in range(len(P)):
        scale = oracle.dydt_scale("gri30", P[i], y[i])
        # floor: the closure mass fraction 1 - sum(Y) is summed in a different
        # order (warp tree vs pyJac's left-to-right), which moves it by an ulp and
        # gives ulp-sized rates where the reference is exactly zero
        floor = np.abs(ref[i][1:]).max()
        err = np.abs(got[i] - ref[i]) / (np.abs(ref[i]) + scale + floor)
        assert err.max() <= 1e-12, (i, err.max())


@pytest.mark.parametrize("precision,tol", [(native.B200ODE_FP64, 1e-10), (native.B200ODE_MIXED, 1e-4)])
def test_jacobian_matches_reference_golden(oracle, golden_chem, precision, tol):
    y, P, ref = golden_chem["y"], golden_chem["P"], golden_chem["jac"]
    nj = int(golden_chem["jac_count"])
    T = np.ascontiguousarray(y[:nj, 0])
    Yfull = np.concatenate([y[:nj, 1:], (1.0 - y[:nj, 1:].sum(axis=1))[:, None]], axis=1)
    s = native.Solver("gri30", precision=precision)
    J = s.eval_jacobian(T, np.ascontiguousarray(Yfull.T), P[:nj])
    s.close()
    for i in range(nj):
        Jo = oracle.jacob("gri30", P[i], y[i])       # exact derivative (J[0,0] included)
        mask = np.abs(ref[i]) > 1e-8 * np.abs(ref[i]).max()
        m2 = mask.copy()
        m2[0, 0] = False
        rel_ref = np.abs(J[i] - ref[i])[m2] / np.abs(ref[i])[m2]
        rel_or = np.abs(J[i] - Jo)[mask] / np.abs(Jo)[mask]
        assert rel_ref.max() <= tol and rel_or.max() <= tol, (i, rel_ref.max(), rel_or.max())


@pytest.mark.parametrize("wl,n", [("h2_1024", 64), ("gri_32k", 64), ("gri_1m", 48), ("gri_bimodal", 48)])
@pytest.mark.parametrize("precision", [native.B200ODE_FP64, native.B200ODE_MIXED])
def test_integration_matches_oracle(oracle, wl, n, precision):
    b = W.make(wl, n)
    yo, so = oracle.bdf(b.mech, b.state_rows(), b.P, b.dt, rtol=W.RTOL, atol=W.ATOL, threads=8)
    T, Y, st, stats, cnt = run_gpu(b, precision, counters=True)
    assert (st == 0).all() and (so["status"] == 0).all()
    compare(b, T, Y, yo, f"{wl}/{precision}", oracle)
    # mass conservation of the returned state (closure species)
    assert np.abs(Y.sum(axis=0) - 1.0).max() < 1e-12
    # step and Newton counts track the oracle's (same algorithm)
    for k in ("nst", "nni", "nje", "nsetups"):
        g, c = cnt[k].sum(), so[k].sum()
        assert abs(g - c) <= 0.1 * c + 10, (k, g, c)


@pytest.mark.parametrize("wl,n", [("gri_32k", 64), ("h2_1024", 64)])
def test_refinement_sweep_matches_oracle(oracle, wl, n):
    """options.refine = 1 (mixed precision): every Newton correction from the
    FP32 factors gets one refinement sweep, r = b - (I - gamma J) x with the
    saved Jacobian in FP64 arithmetic, x += M^-1 r.  Same parity gates and
    counter agreement as the plain mixed form, and the sweep changes the bits of
    the result (it is not skipped)."""
    b = W.make(wl, n, seed=31)
    yo, so = oracle.bdf(b.mech, b.state_rows(), b.P, b.dt, rtol=W.RTOL, atol=W.ATOL, threads=8)
    T, Y, st, stats, cnt = run_gpu(b, native.B200ODE_MIXED, counters=True, refine=1)
    T0, Y0, _, _, cnt0 = run_gpu(b, native.B200ODE_MIXED, counters=True)
    assert (st == 0).all() and (so["status"] == 0).all()
    compare(b, T, Y, yo, f"{wl}/refine", oracle)
    assert np.abs(Y.sum(axis=0) - 1.0).max() < 1e-12
    for k in ("nst", "nni", "nje", "nsetups"):
        g, c = cnt[k].sum(), so[k].sum()
        assert abs(g - c) <= 0.1 * c + 10, (k, g, c)
    assert not (np.array_equal(T, T0) and np.array_equal(Y, Y0))
    # deterministic
    T2, Y2, _, _, _ = run_gpu(b, native.B200ODE_MIXED, refine=1)
    assert np.array_equal(T, T2) and np.array_equal(Y, Y2)


def test_accuracy_vs_fp64_oracle_not_worse_than_cpu(oracle):
    """Error against the FP64 oracle at rtol 1e-10: the GPU (mixed) is as accurate
    as the CPU integrator at the same rtol 1e-6."""
    b = W.make("gri_32k", 64, seed=21)
    ys = b.state_rows()
    ytrue, _ = oracle.bdf(b.mech, ys, b.P, b.dt, rtol=1e-10, atol=1e-14, threads=8)
    ycpu, _ = oracle.bdf(b.mech, ys, b.P, b.dt, rtol=W.RTOL, atol=W.ATOL, threads=8)
    T, Y, st, _, _ = run_gpu(b, native.B200ODE_MIXED)
    eg = np.abs(T - ytrue[:, 0]) / ytrue[:, 0]
    ec = np.abs(ycpu[:, 0] - ytrue[:, 0]) / ytrue[:, 0]
    assert eg.max() <= 3 * ec.max() + 1e-7
    assert np.quantile(eg, 0.99) <= 3 * np.quantile(ec, 0.99) + 1e-7
    gY = np.abs(Y[:-1].T - ytrue[:, 1:])
    cY = np.abs(ycpu[:, 1:] - ytrue[:, 1:])
    assert np.quantile(gY, 0.99) <= 3 * np.quantile(cY, 0.99) + 1e-12


@pytest.mark.parametrize("n", [0, 1, 31, 33])
def test_ragged_batch_sizes(oracle, n):
    b = W.make("gri_32k", max(n, 1), seed=5)
    if n == 0:
        s = native.Solver("gri30")
        st, stats, _ = s.integrate(np.zeros(0), np.zeros((53, 0)), 101325.0, 1e-4)
        assert stats["n_failed"] == 0 and st.size == 0
        s.close()
        return
    yo, so = oracle.bdf(b.mech, b.state_rows(), b.P, b.dt, threads=8)
    T, Y, st, _, _ = run_gpu(b, native.B200ODE_MIXED)
    assert (st == 0).all()
    compare(b, T, Y, yo, f"n={n}", oracle)


def test_h2_1025_cells_fp64(oracle):
    b = W.make("h2_1024", 1025, seed=9)
    yo, so = oracle.bdf(b.mech, b.state_rows(), b.P, b.dt, threads=8)
    T, Y, st, _, _ = run_gpu(b, native.B200ODE_FP64)
    assert (st == 0).all()
    compare(b, T, Y, yo, "h2 1025", oracle)


def test_quiescent_reference_e2e(golden_e2e):
    """The reference's 99-cell 300 K case (tests/Integrators/data/res_gri_100.csv,
    P = 101325.15, dt = 1e-3) returns the reference's serial CVODE output."""
    g = golden_e2e
    T = np.ascontiguousarray(g["T_in"].copy())
    Y = np.ascontiguousarray(g["Y_in"].T.copy())
    for prec in (native.B200ODE_FP64, native.B200ODE_MIXED):
        s = native.Solver("gri30", precision=prec)
        T1, Y1 = T.copy(), Y.copy()
        st, _, _ = s.integrate(T1, Y1, float(g["P"]), float(g["dt"]))
        s.close()
        assert (st == 0).all()
        assert np.abs(T1 - g["T_out"]).max() <= 1e-9 * 300
        assert np.abs(Y1[:-1].T - g["Y_out"][:, :-1]).max() <= 1e-20
        # closure species as the reference computes it: 1 - sum
        assert np.abs(Y1[-1] - g["Y_out"][:, -1]).max() <= 1e-15


def test_deterministic_and_batch_independent():
    b = W.make("gri_32k", 40, seed=13)
    T1, Y1, _, _, _ = run_gpu(b, native.B200ODE_MIXED)
    T2, Y2, _, _, _ = run_gpu(b, native.B200ODE_MIXED)
    assert np.array_equal(T1, T2) and np.array_equal(Y1, Y2)
    # every cell alone gives the same bits as in the batch
    for c in (0, 17, 39):
        bc = b.subset(np.array([c]))
        Tc, Yc, _, _, _ = run_gpu(bc, native.B200ODE_MIXED)
        assert Tc[0] == T1[c] and np.array_equal(Yc[:, 0], Y1[:, c])


def test_queue_chunk_does_not_change_results():
    b = W.make("gri_bimodal", 300, seed=12)
    T1, Y1, s1, _, _ = run_gpu(b, native.B200ODE_MIXED)
    T2, Y2, s2, _, _ = run_gpu(b, native.B200ODE_MIXED, queue_chunk=7)
    assert np.array_equal(T1, T2) and np.array_equal(Y1, Y2) and np.array_equal(s1, s2)


def test_step_form_equals_persistent_form():
    """The plain one-launch-per-step form keeps the full per-cell state in HBM
    between launches, so it reproduces the persistent kernel bit for bit."""
    b = W.make("gri_1m", 24, seed=3)
    Tp, Yp, sp, _, cp = run_gpu(b, native.B200ODE_FP64, counters=True)
    Ts, Ys, ss, _, cs = run_gpu(b, native.B200ODE_FP64, persistent=0, counters=True)
    Tg, Yg, sg, _, _ = run_gpu(b, native.B200ODE_FP64, persistent=0, use_graph=1)
    assert np.array_equal(Tp, Ts) and np.array_equal(Yp, Ys) and np.array_equal(sp, ss)
    assert np.array_equal(Tp, Tg) and np.array_equal(Yp, Yg)
    for k in native.COUNTERS:
        assert np.array_equal(cp[k], cs[k]), k


def test_pressure_array_equals_scalar():
    b = W.make("h2_1024", 16)
    s = native.Solver("h2o2")
    T1, Y1 = b.T.copy(), b.Y.copy()
    s.integrate(T1, Y1, 101325.0, b.dt)
    T2, Y2 = b.T.copy(), b.Y.copy()
    s.integrate(T2, Y2, np.full(16, 101325.0), b.dt)
    s.close()
    assert np.array_equal(T1, T2) and np.array_equal(Y1, Y2)


def test_failure_paths_are_reported_and_isolated(oracle):
    """max_steps cap, t1 == t0, a poisoned (NaN) cell: statuses are CVODE codes,
    bounded work, and healthy neighbours are unaffected."""
    b = W.make("gri_1m", 8, seed=4)
    # forced cap: same state as the oracle after 5 steps
    T, Y, st, _, cnt = run_gpu(b, native.B200ODE_FP64, counters=True, max_steps=5)
    yo, so = oracle.bdf(b.mech, b.state_rows(), b.P, b.dt, max_steps=5)
    assert (st == -1).all() and (cnt["nst"] == 5).all() and (so["status"] == -1).all()
    assert np.abs(T - yo[:, 0]).max() / yo[:, 0].min() < 1e-6
    # t1 == t0
    s = native.Solver("gri30")
    T2, Y2 = b.T.copy(), b.Y.copy()
    st2, _, _ = s.integrate(T2, Y2, b.P, 0.0)
    assert (st2 == -27).all()
    # poisoned cell
    Tref, Yref = b.T.copy(), b.Y.copy()
    s.integrate(Tref, Yref, b.P, b.dt)
    Tbad, Ybad = b.T.copy(), b.Y.copy()
    Tbad[3] = np.nan
    st3, stats3, _ = s.integrate(Tbad, Ybad, b.P, b.dt)
    s.close()
    assert st3[3] != 0 and stats3["n_failed"] >= 1
    good = np.arange(8) != 3
    assert np.array_equal(Tbad[good], Tref[good]) and np.array_equal(Ybad[:, good], Yref[:, good])


@pytest.mark.parametrize("precision", [native.B200ODE_FP64, native.B200ODE_MIXED])
def test_poisoned_cells_do_not_disturb_neighbours(precision):
    """Host-side fault injection: a cell at 50 K, a cell with a negative mass
    fraction, an infinite temperature and a zero-density cell are integrated in
    one batch with healthy cells.  Every call returns, each poisoned cell gets a
    CVODE status of its own, and the healthy cells are bitwise those of a clean
    run."""
    b = W.make("gri_32k", 12, seed=11)
    s = native.Solver("gri30", precision=precision, max_steps=2000)
    Tc, Yc = b.T.copy(), b.Y.copy()
    st_clean, _, _ = s.integrate(Tc, Yc, b.P, b.dt)
    T, Y = b.T.copy(), b.Y.copy()
    T[2] = 50.0                      # far below the NASA-7 fit range
    Y[3, 5] = -0.05                  # negative O2 mass fraction
    T[7] = np.inf
    Y[:, 9] = 0.0                    # no mass at all
    st, stats, _ = s.integrate(T, Y, b.P, b.dt)
    s.close()
    poisoned = np.array([2, 5, 7, 9])
    good = np.setdiff1d(np.arange(12), poisoned)
    assert (st_clean == 0).all()
    assert np.array_equal(T[good], Tc[good]) and np.array_equal(Y[:, good], Yc[:, good])
    assert np.array_equal(st[good], st_clean[good])
    assert set(np.unique(st[poisoned])) <= {0, -1, -2, -3, -4}
    assert st[7] != 0 and stats["n_failed"] >= 1


@pytest.mark.parametrize("formulation", [native.B200ODE_CONP, native.B200ODE_CONV])
def test_bad_pressure_is_ill_input(formulation):
    """A per-cell pressure that is not > 0 (zero, negative, NaN) gives that cell
    CVODE's CV_ILL_INPUT (-22) and leaves it as given; the other cells are
    bitwise those of a clean run."""
    b = W.make("gri_32k", 10, seed=12)
    s = native.Solver("gri30", formulation=formulation)
    Tc, Yc = b.T.copy(), b.Y.copy()
    st_clean, _, _ = s.integrate(Tc, Yc, b.P, b.dt)
    P = b.P.copy()
    P[[1, 4, 8]] = [0.0, -101325.0, np.nan]
    T, Y = b.T.copy(), b.Y.copy()
    st, stats, cnt = s.integrate(T, Y, P, b.dt, counters=True)
    s.close()
    bad = np.array([1, 4, 8])
    good = np.setdiff1d(np.arange(10), bad)
    assert (st[bad] == -22).all() and stats["n_failed"] == 3 and (cnt["nst"][bad] == 0).all()
    assert np.array_equal(T[bad], b.T[bad]) and np.array_equal(Y[:, bad], b.Y[:, bad])
    assert np.array_equal(T[good], Tc[good]) and np.array_equal(Y[:, good], Yc[:, good])
    assert np.array_equal(st[good], st_clean[good])


def test_invalid_arguments_raise():
    with pytest.raises(native.B200Error):
        native.Solver("not_a_mechanism")
    with pytest.raises(native.B200Error):
        native.Solver("gri30", abstol=0.0)
    s = native.Solver("gri30")
    with pytest.raises(native.B200Error):
        s.integrate(np.full(2, 1000.0), np.full((53, 2), 1.0 / 53), -1.0, 1e-4)
    s.close()


@pytest.mark.parametrize("persistent", [1, 0])
def test_memory_sized_chunks_equal_one_launch(persistent):
    """A batch larger than max_cells_per_launch (the memory-sized batching of
    the reference's calc_gpu_points) runs as consecutive launches over
    contiguous chunks; cells are independent, so results, statuses, per-cell
    counters and call totals equal one launch over the whole batch bitwise,
    through the host-buffer and the device-buffer entry points."""
    import torch
    b = W.make("gri_1m", 333, seed=17)
    out = {}
    for chunk in (0, 100):
        s = native.Solver("gri30", precision=native.B200ODE_FP64, persistent=persistent,
                          max_cells_per_launch=chunk)
        T, Y = b.T.copy(), np.ascontiguousarray(b.Y.copy())
        st, stats, cnt = s.integrate(T, Y, b.P, b.dt, counters=True)
        dT = torch.from_numpy(b.T.copy()).cuda()
        dY = torch.from_numpy(np.ascontiguousarray(b.Y)).cuda()
        dP = torch.from_numpy(np.ascontiguousarray(b.P)).cuda()
        dst = torch.zeros(b.ncells, dtype=torch.int32, device="cuda")
        dstats = s.integrate_device(b.ncells, dP.data_ptr(), 0.0, dT.data_ptr(), dY.data_ptr(), b.dt,
                                    dstatus=dst.data_ptr())
        torch.cuda.synchronize()
        s.close()
        out[chunk] = (T, Y, st, cnt, stats, dT.cpu().numpy(), dY.cpu().numpy(), dst.cpu().numpy(), dstats)
    a, c = out[0], out[100]
    assert (a[2] == 0).all()
    for i in (0, 1, 2, 5, 6, 7):
        assert np.array_equal(a[i], c[i]), i
    assert np.array_equal(a[0], a[5]) and np.array_equal(a[1], a[6])
    for k in native.COUNTERS:
        assert np.array_equal(a[3][k], c[3][k]), k
    for k in ("total_nst", "total_nfe", "total_nje", "total_nsetups", "total_nni", "n_failed"):
        assert a[4][k] == c[4][k] == a[8][k] == c[8][k], k
    assert c[4]["gpu_launches"] > a[4]["gpu_launches"]
