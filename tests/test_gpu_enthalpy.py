"""Mixture enthalpy of the cell state (b200ode_eval_enthalpy) against the
ENTHA column of the reference's own data files (computed there by Cantera;
committed as tests/golden/enthalpy_ref.npz), and the C++ integrator's
b200.enthalpy: update option."""
import numpy as np
import pytest

import host_driver
from hpc_ode_b200 import native, workloads as W

pytestmark = pytest.mark.gpu


def test_enthalpy_matches_reference_data(golden_enthalpy):
    g = golden_enthalpy
    s = native.Solver("h2_li_2004")
    h = s.eval_enthalpy(g["h2_T"], g["h2_Y"])
    s.close()
    # the mechanism kernels use pyJac's R = 8314.4621 J/kmol/K, Cantera 8314.46261815:
    # a constant 6.2e-8 relative offset
    assert (np.abs(h - g["h2_h"]) / np.abs(g["h2_h"])).max() <= 1e-7
    s = native.Solver("gri30")
    h = s.eval_enthalpy(g["gri_T"], g["gri_Y"])
    s.close()
    # the GRI data file rounds ENTHA to 5 significant digits
    assert (np.abs(h - g["gri_h"]) / np.abs(g["gri_h"])).max() <= 2e-5


def test_integrator_updates_enthalpy_only_when_asked(tmp_path):
    exe = host_driver.build(tmp_path)
    b = W.make("h2li_grid", 32)
    P = float(b.P[0])
    rc, out, To, Yo, st = host_driver.run(exe, tmp_path, "BDFIntegratorB200", "h2_li_2004.xml", b.T, b.Y.T, b.dt, P)
    assert rc == 0 and (host_driver.run.enthalpy == 0.0).all()          # kept, as the CVODE integrators do
    rc, out, To, Yo, st = host_driver.run(exe, tmp_path, "BDFIntegratorB200", "h2_li_2004.xml", b.T, b.Y.T, b.dt, P,
                                          ["b200.enthalpy=update"])
    assert rc == 0, out
    s = native.Solver("h2_li_2004")
    h = s.eval_enthalpy(To, np.ascontiguousarray(Yo.T))
    s.close()
    assert np.array_equal(host_driver.run.enthalpy, h)
