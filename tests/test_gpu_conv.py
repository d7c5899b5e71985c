"""Constant-volume formulation (b200ode_options.formulation = B200ODE_CONV)
through the C ABI against the oracle's constant-volume chemistry and BDF.

The reference ships pyJac's CONV branch (src/Mechanism/CPU/dydt.c:135-265,
eval_conc_rho in chem_utils.c:99-137) but it does not compile, so the oracle's
restatement is pinned by its exact Jacobian matching central differences of its
RHS and by energy conservation of its integrator (tests/test_oracle.py); here
the GPU is held to the oracle at the parity tolerances, and to internal-energy
conservation on a batch too large for the oracle.
"""
import numpy as np
import pytest

from conftest import y_ok
from hpc_ode_b200 import native, workloads as W
from test_oracle import specific_energy

pytestmark = pytest.mark.gpu

GATE_T = 1e-5


@pytest.mark.parametrize("wl,n", [("gri_32k", 24), ("h2_1024", 16), ("kero_2k", 12)])
def test_rhs_matches_oracle(oracle, wl, n):
    b = W.make(wl, n, seed=21)
    if wl == "kero_2k":
        b.P[:3] = np.array([0.003, 0.05, 150.0]) * W.ATM   # PLOG tables: both clamped ends
    s = native.Solver(b.mech, formulation=native.B200ODE_CONV)
    dT, dY = s.eval_rhs(b.T, b.Y, b.P)
    s.close()
    got = np.concatenate([dT[:, None], dY.T], axis=1)
    rows = b.state_rows()
    for i in range(b.ncells):
        rho = oracle.density(b.mech, b.P[i], rows[i])
        ref = oracle.dydt_conv(b.mech, rho, rows[i])
        scale = oracle.dydt_scale_conv(b.mech, rho, rows[i])
        err = np.abs(got[i] - ref) / (np.abs(ref) + scale + np.abs(ref[1:]).max())
        assert err.max() <= 1e-12, (i, err.max())


@pytest.mark.parametrize("wl,precision,tol", [("gri_32k", native.B200ODE_FP64, 1e-10),
                                              ("gri_32k", native.B200ODE_MIXED, 1e-4),
                                              ("kero_2k", native.B200ODE_MIXED, 1e-4)])
def test_jacobian_matches_oracle(oracle, wl, precision, tol):
    b = W.make(wl, 6, seed=22)
    b.P[0] = 0.05 * W.ATM
    s = native.Solver(b.mech, precision=precision, formulation=native.B200ODE_CONV)
    J = s.eval_jacobian(b.T, b.Y, b.P)
    s.close()
    rows = b.state_rows()
    for i in range(b.ncells):
        Jo = oracle.jacob_conv(b.mech, oracle.density(b.mech, b.P[i], rows[i]), rows[i])
        mask = np.abs(Jo) > 1e-8 * np.abs(Jo).max()
        rel = np.abs(J[i] - Jo)[mask] / np.abs(Jo)[mask]
        assert rel.max() <= tol, (i, rel.max())


@pytest.mark.parametrize("precision", [native.B200ODE_FP64, native.B200ODE_MIXED])
@pytest.mark.parametrize("wl,n", [("gri_32k", 64), ("h2_1024", 48)])
def test_integration_matches_oracle(oracle, wl, n, precision):
    b = W.make(wl, n, seed=23)
    yo, so = oracle.bdf(b.mech, b.state_rows(), b.P, b.dt, conv=True, threads=8)
    s = native.Solver(b.mech, precision=precision, formulation=native.B200ODE_CONV)
    T, Y = b.T.copy(), np.ascontiguousarray(b.Y.copy())
    st, _, cnt = s.integrate(T, Y, b.P, b.dt, counters=True)
    s.close()
    assert (st == 0).all() and (so["status"] == 0).all()
    assert (T - b.T).max() > 500.0
    assert ((np.abs(T - yo[:, 0]) / yo[:, 0]) <= GATE_T).all()
    assert y_ok(Y[:-1].T, yo[:, 1:]).mean() >= 0.99
    assert np.abs(Y.sum(axis=0) - 1.0).max() < 1e-12
    g, c = cnt["nst"].sum(), so["nst"].sum()
    assert abs(g - c) <= 0.15 * c + 10, (g, c)


def test_differs_from_constant_pressure():
    """Same cells, the two formulations: at constant volume the heat release
    raises the pressure, so ignition is faster and the final temperature
    higher (cv < cp) than at constant pressure."""
    b = W.make("h2_1024", 64, seed=24)
    out = {}
    for f in (native.B200ODE_CONP, native.B200ODE_CONV):
        s = native.Solver(b.mech, formulation=f)
        T, Y = b.T.copy(), np.ascontiguousarray(b.Y.copy())
        st, _, _ = s.integrate(T, Y, b.P, b.dt)
        s.close()
        assert (st == 0).all()
        out[f] = T
    burnt = out[native.B200ODE_CONP] > b.T + 500.0
    assert burnt.sum() > 10
    assert (out[native.B200ODE_CONV][burnt] > out[native.B200ODE_CONP][burnt] + 100.0).all()


def test_internal_energy_conserved_at_size():
    """Size-independent property on 16,384 GRI cells: a closed adiabatic
    constant-volume reactor conserves its specific internal energy; at rtol
    1e-6 the oracle's own drift is below 2e-6 of cv T (tests/test_oracle.py
    calibration), the GPU is held to 1e-5 for every cell."""
    b = W.make("gri_32k", 16384, seed=25)
    s = native.Solver(b.mech, formulation=native.B200ODE_CONV)
    T, Y = b.T.copy(), np.ascontiguousarray(b.Y.copy())
    st, _, _ = s.integrate(T, Y, b.P, b.dt)
    s.close()
    assert (st == 0).all()
    assert (T - b.T > 300).sum() > 1000
    e0 = specific_energy(b.mech, b.T, b.Y, True)
    e1 = specific_energy(b.mech, T, Y, True)
    drift = np.abs(e1 - e0) / (1000.0 * T)
    assert drift.max() < 1e-5, drift.max()


def test_persistent_equals_step_form():
    """Both batching forms run the same step code at constant volume too."""
    b = W.make("gri_32k", 64, seed=26)
    out = []
    for persistent in (1, 0):
        s = native.Solver(b.mech, precision=native.B200ODE_FP64, persistent=persistent,
                          formulation=native.B200ODE_CONV)
        T, Y = b.T.copy(), np.ascontiguousarray(b.Y.copy())
        st, _, _ = s.integrate(T, Y, b.P, b.dt)
        s.close()
        out.append((T, Y, st))
    assert np.array_equal(out[0][2], out[1][2])
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_bad_formulation_is_refused():
    with pytest.raises(native.B200Error) as e:
        native.Solver("gri30", formulation=7)
    assert e.value.code == 1 and "formulation" in str(e.value)
