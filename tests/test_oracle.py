"""CPU oracle checks: pinned against the reference's own pyJac outputs (golden
vectors generated from the compiled reference C by tests/golden/make_golden.py)
and against scipy's VODE/Radau."""
import numpy as np
import pytest

from hpc_ode_b200 import workloads as W


def test_mechanism_tables_match_pyjac_structure():
    g = W.mech_info("gri30")
    c = g["counts"]
    # src/Mechanism/CPU/mechanism.h:63-71: NSP 53, FWD_RATES 325, REV_RATES 309, PRES_MOD_RATES 50
    assert (c["species"], c["reactions"], c["reversible"], c["pres_mod"]) == (53, 325, 309, 50)
    assert c["troe"] == 26 and c["lindemann"] == 3 and c["three-body"] == 21
    assert g["species"][-1] == "CH3CHO"          # mechanism.h:5 last_spec 52
    h = W.mech_info("h2o2")
    assert h["nsp"] == 10 and h["counts"]["reactions"] == 29 and h["species"][-1] == "N2"


def test_rhs_matches_reference_pyjac(oracle, golden_chem):
    y, P, ref = golden_chem["y"], golden_chem["P"], golden_chem["dydt"]
    worst = 0.0
    for i in range(len(P)):
        got = oracle.dydt("gri30", P[i], y[i])
        scale = oracle.dydt_scale("gri30", P[i], y[i])
        err = np.abs(got - ref[i]) / (np.abs(ref[i]) + scale + 1e-300)
        worst = max(worst, err.max())
    # cancellation-aware relative tolerance (scale = |fwd| + |rev| contributions)
    assert worst <= 1e-12, worst


def test_jacobian_matches_reference_pyjac(oracle, golden_chem):
    y, P, ref = golden_chem["y"], golden_chem["P"], golden_chem["jac"]
    for i in range(int(golden_chem["jac_count"])):
        J = oracle.jacob("gri30", P[i], y[i])
        Jr = ref[i]
        mask = np.abs(Jr) > 1e-8 * np.abs(Jr).max()
        mask[0, 0] = False   # pyJac's dTdot/dT is not the derivative of its dydt (see next test)
        rel = np.abs(J - Jr)[mask] / np.abs(Jr)[mask]
        assert rel.max() <= 1e-10, (i, rel.max())


def test_jacobian_TT_is_derivative_of_reference_rhs(oracle, golden_chem):
    """J[0,0] against central differences of the reference pyJac dydt values
    (the oracle's dydt equals pyJac's to 1e-12)."""
    y, P = golden_chem["y"], golden_chem["P"]
    for i in range(8):
        J = oracle.jacob("gri30", P[i], y[i])
        h = 1e-3
        yp, ym = y[i].copy(), y[i].copy()
        yp[0] += h
        ym[0] -= h
        fd = (oracle.dydt("gri30", P[i], yp)[0] - oracle.dydt("gri30", P[i], ym)[0]) / (2 * h)
        assert abs(J[0, 0] - fd) <= 1e-5 * max(abs(fd), 1.0), (i, J[0, 0], fd)


@pytest.mark.parametrize("conv", [False, True])
@pytest.mark.parametrize("mech,wl", [("h2o2", "h2_1024"), ("gri30", "gri_32k"), ("nDodecane_Reitz", "nc12_8k"),
                                     ("ESTiMatE-Mech_04042022", "kero_2k")])
def test_jacobian_finite_difference(oracle, mech, wl, conv):
    """Analytic Jacobian against central differences of the RHS, at constant
    pressure and at constant volume (density of the cell's state fixed)."""
    b = W.make(wl, 4, seed=7)
    ys = b.state_rows()
    for c in range(4):
        y = ys[c]
        if conv:
            rho = oracle.density(mech, b.P[c], y)
            J = oracle.jacob_conv(mech, rho, y)
            f = lambda v: oracle.dydt_conv(mech, rho, v)  # noqa: E731
        else:
            J = oracle.jacob(mech, b.P[c], y)
            f = lambda v: oracle.dydt(mech, b.P[c], v)  # noqa: E731
        n = y.size
        Jfd = np.zeros((n, n))
        for j in range(n):
            h = 1e-4 if j == 0 else 1e-7 * max(abs(y[j]), 1e-8)
            yp, ym = y.copy(), y.copy()
            yp[j] += h
            ym[j] -= h
            Jfd[:, j] = (f(yp) - f(ym)) / (2 * h)
        big = np.abs(Jfd) > 1e-4 * np.abs(Jfd).max()
        rel = np.abs(J - Jfd)[big] / np.abs(Jfd)[big]
        assert np.quantile(rel, 0.99) < 1e-3 and rel.max() < 1e-2, (c, rel.max())


def test_bdf_matches_scipy_radau(oracle):
    from scipy.integrate import solve_ivp
    for wl, n in (("h2_1024", 3), ("gri_32k", 3)):
        b = W.make(wl, n)
        ys = b.state_rows()
        yt, st = oracle.bdf(b.mech, ys, b.P, b.dt, rtol=1e-10, atol=1e-14)
        assert (st["status"] == 0).all()
        for c in range(n):
            f = lambda t, y: oracle.dydt(b.mech, b.P[c], y)  # noqa: E731
            J = lambda t, y: oracle.jacob(b.mech, b.P[c], y)  # noqa: E731
            r = solve_ivp(f, (0, b.dt), ys[c], method="Radau", jac=J, rtol=1e-11, atol=1e-15)
            assert abs(yt[c, 0] - r.y[0, -1]) / r.y[0, -1] < 1e-8


def test_quiescent_e2e_fixture(oracle, golden_e2e):
    """The reference's 99-cell 300 K E2E case comes back as the reference's serial
    CVODE output (E2Etests/100/results_serial100.csv)."""
    g = golden_e2e
    y = np.concatenate([g["T_in"][:, None], g["Y_in"][:, :-1]], axis=1)
    yo, st = oracle.bdf("gri30", y, float(g["P"]), float(g["dt"]), threads=4)
    assert (st["status"] == 0).all()
    assert np.abs(yo[:, 0] - g["T_out"]).max() <= 1e-9 * 300.0
    assert np.abs(yo[:, 1:] - g["Y_out"][:, :-1]).max() <= 1e-20


def test_openmp_batch_equals_serial(oracle):
    """As the reference's testSerialvsOMP (tests/Integrators/testCVodeIntegrator.cpp:92-134):
    the threaded batch equals the serial batch bit for bit."""
    b = W.make("h2_1024", 16)
    y1, s1 = oracle.bdf(b.mech, b.state_rows(), b.P, b.dt, threads=1)
    y4, s4 = oracle.bdf(b.mech, b.state_rows(), b.P, b.dt, threads=4)
    assert np.array_equal(y1, y4) and np.array_equal(s1, s4)


def test_max_steps_cap_and_too_close(oracle):
    b = W.make("gri_1m", 2)
    y, st = oracle.bdf(b.mech, b.state_rows(), b.P, b.dt, max_steps=5)
    assert (st["status"] == -1).all() and (st["nst"] == 5).all()
    y, st = oracle.bdf(b.mech, b.state_rows(), b.P, 0.0)
    assert (st["status"] == -27).all()


def _header_arrays(mech):
    """The generated C header's static arrays, parsed as numpy arrays."""
    import os
    import re
    txt = open(os.path.join(W.MECH_DIR, f"{mech}_mech.h")).read()
    out = {}
    for m in re.finditer(r"static const (?:double|int) \w+?_(rxn_\w+|plog_\w+)\[\d+\] = \{([^}]*)\};", txt):
        out[m.group(1)] = np.array([float(v) for v in m.group(2).split(",")])
    return out


def test_plog_rates_match_log_pressure_interpolation(oracle):
    """PLOG reactions of the kerosene mechanism: the oracle's k(T, P) against a
    numpy restatement of the published definition (ln k linear in ln P between
    the bracketing levels, the end levels' k outside; a level's k is the sum of
    its Arrhenius terms), below, at, between and above the tabulated pressures."""
    mech = W.ESTIMATE
    a = _header_arrays(mech)
    nr = a["rxn_type"].size
    off, toff, lnP = a["plog_off"].astype(int), a["plog_term_off"].astype(int), a["plog_lnP"]

    def level(l, T):
        t = slice(toff[l], toff[l + 1])
        return np.sum(a["plog_A"][t] * T ** a["plog_b"][t] * np.exp(-a["plog_EaR"][t] / T))

    plog = np.flatnonzero(a["rxn_type"] == 4)
    assert plog.size == 22
    for T in (800.0, 1300.0, 2100.0):
        for P in (0.001 * 101325, 0.01 * 101325, 0.37 * 101325, 1.0 * 101325, 7.5 * 101325, 250 * 101325):
            kf = oracle.kf(mech, P, T, nr)
            for r in plog:
                levels = np.arange(off[r], off[r + 1])
                lp = np.log(P)
                if lp <= lnP[levels[0]]:
                    want = level(levels[0], T)
                elif lp >= lnP[levels[-1]]:
                    want = level(levels[-1], T)
                else:
                    i = levels[np.searchsorted(lnP[levels], lp) - 1]
                    w = (lp - lnP[i]) / (lnP[i + 1] - lnP[i])
                    want = np.exp((1 - w) * np.log(level(i, T)) + w * np.log(level(i + 1, T)))
                assert kf[r] == pytest.approx(want, rel=1e-12), (r, T, P)


RU = 8314.4621


def specific_energy(mech, T, Y, conv):
    """Mixture enthalpy (constant pressure) or internal energy (constant
    volume) per unit mass [J/kg] from the committed NASA-7 tables: T[n],
    Y[nsp, n]."""
    import os
    import re
    txt = open(os.path.join(W.MECH_DIR, f"{mech}_mech.h")).read()
    t = {}
    for m in re.finditer(r"static const double \w+?_(mw|tmid|nasa_lo|nasa_hi)\[\d+\] = \{([^}]*)\};", txt):
        t[m.group(1)] = np.array([float(v) for v in m.group(2).split(",")])
    n = t["mw"].size
    T = np.atleast_1d(T)
    lo, hi = t["nasa_lo"].reshape(n, 7), t["nasa_hi"].reshape(n, 7)
    out = np.zeros(T.size)
    for c in range(T.size):
        a = np.where((T[c] <= t["tmid"])[:, None], lo, hi)
        x = T[c]
        hRT = a[:, 0] + x * (a[:, 1] / 2 + x * (a[:, 2] / 3 + x * (a[:, 3] / 4 + a[:, 4] / 5 * x))) + a[:, 5] / x
        e = RU * x * hRT / t["mw"] - (RU * x / t["mw"] if conv else 0.0)
        out[c] = (Y[:, c] * e).sum()
    return out


@pytest.mark.parametrize("conv", [False, True])
def test_bdf_conserves_energy(oracle, conv):
    """A closed adiabatic reactor conserves enthalpy at constant pressure and
    internal energy at constant volume: after igniting H2 and CH4 cells at
    rtol 1e-10 the change is round-off / tolerance level (< 1e-9 of cp T)."""
    for wl in ("h2_1024", "gri_32k"):
        b = W.make(wl, 4, seed=3)
        ys = b.state_rows()
        yo, st = oracle.bdf(b.mech, ys, b.P, b.dt, rtol=1e-10, atol=1e-14, conv=conv)
        assert (st["status"] == 0).all()
        full = lambda r: np.vstack([r[:, 1:].T, 1.0 - r[:, 1:].sum(axis=1)])  # noqa: E731
        e0 = specific_energy(b.mech, ys[:, 0], full(ys), conv)
        e1 = specific_energy(b.mech, yo[:, 0], full(yo), conv)
        assert (yo[:, 0] - ys[:, 0]).max() > 500.0                      # they ignited
        assert (np.abs(e1 - e0) / (1000.0 * yo[:, 0])).max() < 1e-9, (wl, conv)


def test_constant_volume_raises_pressure(oracle):
    """At constant volume the density stays that of the initial state and the
    pressure P = rho R T / W rises with the heat release; at constant pressure
    the density falls instead."""
    b = W.make("h2_1024", 2, seed=3)
    ys = b.state_rows()
    rho0 = np.array([oracle.density(b.mech, b.P[c], ys[c]) for c in range(2)])
    yv, _ = oracle.bdf(b.mech, ys, b.P, b.dt, rtol=1e-10, atol=1e-14, conv=True)
    yp, _ = oracle.bdf(b.mech, ys, b.P, b.dt, rtol=1e-10, atol=1e-14)
    for c in range(2):
        rho_p = oracle.density(b.mech, b.P[c], yp[c])
        P_v = b.P[c] * (rho0[c] / oracle.density(b.mech, b.P[c], yv[c]))   # P at rho0 and the final T, Y
        assert rho_p < 0.7 * rho0[c] and P_v > 1.5 * b.P[c]


CROSSCHECK = ("h2_1024", "gri_32k", "gri_1m")


@pytest.fixture(scope="module")
def crosscheck():
    import os
    from conftest import GOLDEN
    return dict(np.load(os.path.join(GOLDEN, "crosscheck_vode_radau.npz")))


@pytest.mark.parametrize("wl", CROSSCHECK)
def test_bdf_oracle_agrees_with_vode_and_radau(oracle, crosscheck, wl):
    """Three-way pin of the CVODE-semantics oracle where the reference's CVODE
    cannot run, on 640 seeded reacting cells (256 H2, 256 + 128 GRI-Mech 3.0)
    against VODE (BDF order 5, CVODE's Fortran ancestor) and Radau IIA (an
    implicit Runge-Kutta method), both generated by
    tests/golden/make_crosscheck.py on the same restated chemistry.  The
    converged solution is Radau at rtol 1e-13 / atol 1e-16.

    * Tightened (oracle and VODE at rtol 1e-12, Radau at 1e-13) the three agree
      pairwise to <= 1e-8 relative on T on every cell, and the oracle's mass
      fractions are within max(1e-6 |Y|, 1e-13) of the converged ones.
    * At rtol 1e-10 / atol 1e-14 (the oracle's setting as the FP64 reference)
      the oracle's error in T against the converged solution is that of VODE at
      the same tolerances: p99 and max within 2x VODE's (both carry BDF global
      error of up to ~1e-8 at the ignition front), median <= 1e-10."""
    y0, P, dt = crosscheck[f"{wl}_y0"], crosscheck[f"{wl}_P"], float(crosscheck[f"{wl}_dt"])
    mech = W.make(wl, 1).mech
    truth = crosscheck[f"{wl}_radau_tight"]
    vt = crosscheck[f"{wl}_vode_tight"]
    for k in ("vode", "radau", "vode_tight", "radau_tight"):
        assert np.isfinite(crosscheck[f"{wl}_{k}"]).all(), k
    ot, st = oracle.bdf(mech, y0, P, dt, rtol=1e-12, atol=1e-16, threads=8)
    assert (st["status"] == 0).all()
    rel = lambda a, b: np.abs(a[:, 0] - b[:, 0]) / b[:, 0]  # noqa: E731
    for a, b, pair in ((ot, truth, "oracle-radau"), (ot, vt, "oracle-vode"), (vt, truth, "vode-radau")):
        assert rel(a, b).max() <= 1e-8, (wl, pair, rel(a, b).max())
    dY = np.abs(ot[:, 1:] - truth[:, 1:])
    assert (dY <= np.maximum(1e-6 * np.abs(truth[:, 1:]), 1e-13)).all(), (wl, dY.max())
    yo, st = oracle.bdf(mech, y0, P, dt, rtol=1e-10, atol=1e-14, threads=8)
    assert (st["status"] == 0).all()
    eo, ev = rel(yo, truth), rel(crosscheck[f"{wl}_vode"], truth)
    assert np.quantile(eo, 0.99) <= 2.0 * np.quantile(ev, 0.99), (wl, np.quantile(eo, 0.99), np.quantile(ev, 0.99))
    assert eo.max() <= 2.0 * ev.max(), (wl, eo.max(), ev.max())
    assert np.median(eo) <= 1e-10, (wl, np.median(eo))
    assert (yo[:, 0] - y0[:, 0]).max() > 500.0          # reacting cells, not frozen ones


def test_crosscheck_fixture_reproduces(oracle, crosscheck):
    """The committed VODE/Radau states are what those integrators give now (two
    cells per workload re-integrated live)."""
    from scipy.integrate import ode, solve_ivp
    for wl in CROSSCHECK:
        y0, P, dt = crosscheck[f"{wl}_y0"], crosscheck[f"{wl}_P"], float(crosscheck[f"{wl}_dt"])
        mech = W.make(wl, 1).mech
        for c in (0, 1):
            f = lambda t, y: oracle.dydt(mech, P[c], y)  # noqa: E731
            J = lambda t, y: oracle.jacob(mech, P[c], y)  # noqa: E731
            r = ode(f, J).set_integrator("vode", method="bdf", order=5, with_jacobian=True,
                                         rtol=1e-10, atol=1e-14, nsteps=200000)
            r.set_initial_value(y0[c], 0.0)
            assert np.allclose(r.integrate(dt), crosscheck[f"{wl}_vode"][c], rtol=1e-12, atol=1e-18)
            rr = solve_ivp(f, (0.0, dt), y0[c], method="Radau", jac=J, rtol=1e-10, atol=1e-14)
            assert np.allclose(rr.y[:, -1], crosscheck[f"{wl}_radau"][c], rtol=1e-12, atol=1e-18)


def test_reference_location_from_environment(tmp_path, monkeypatch):
    """The reference checkout the fixture scripts and the oracle's reference build read is
    HPC_ODE_REFERENCE when set (and an existing directory), and nothing when that names no
    directory."""
    from oracle import refpath
    (tmp_path / "src" / "Mechanism" / "CPU").mkdir(parents=True)
    monkeypatch.setenv("HPC_ODE_REFERENCE", str(tmp_path))
    assert refpath.reference_dir() == str(tmp_path)
    assert refpath.reference_subdir("src", "Mechanism", "CPU") == str(tmp_path / "src" / "Mechanism" / "CPU")
    assert refpath.reference_subdir("no", "such") is None
    monkeypatch.setenv("HPC_ODE_REFERENCE", str(tmp_path / "missing"))
    assert refpath.reference_dir() is None
