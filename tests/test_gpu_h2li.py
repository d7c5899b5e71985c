"""The reference's H2 mechanism (h2_li_2004, read from CTML) on its H2
dataset grid (T0 1000-2100 K x phi 0.5-3.5 at 1 atm), through the C ABI against
the oracle at the tolerances of tests/test_gpu_parity.py."""
import numpy as np
import pytest

from hpc_ode_b200 import native, workloads as W
from test_gpu_parity import compare

pytestmark = pytest.mark.gpu

MECH = "h2_li_2004"


def test_rhs_and_jacobian_match_oracle(oracle):
    b = W.make("h2li_grid", 64)
    rows = b.state_rows()
    s = native.Solver(MECH, precision=native.B200ODE_FP64)
    dT, dY = s.eval_rhs(b.T, b.Y, b.P)
    J = s.eval_jacobian(b.T, b.Y, b.P)
    s.close()
    got = np.concatenate([dT[:, None], dY.T], axis=1)
    for i in range(b.ncells):
        ref = oracle.dydt(MECH, b.P[i], rows[i])
        scale = oracle.dydt_scale(MECH, b.P[i], rows[i])
        err = np.abs(got[i] - ref) / (np.abs(ref) + scale + np.abs(ref[1:]).max())
        assert err.max() <= 1e-12, (i, err.max())
        Jo = oracle.jacob(MECH, b.P[i], rows[i])
        mask = np.abs(Jo) > 1e-8 * np.abs(Jo).max()
        assert (np.abs(J[i] - Jo)[mask] / np.abs(Jo)[mask]).max() <= 1e-10, i


@pytest.mark.parametrize("precision", [native.B200ODE_FP64, native.B200ODE_MIXED])
def test_dataset_grid_matches_oracle(oracle, precision):
    b = W.make("h2li_grid", 400)
    yo, so = oracle.bdf(MECH, b.state_rows(), b.P, b.dt, threads=8)
    s = native.Solver(MECH, precision=precision)
    T, Y = b.T.copy(), np.ascontiguousarray(b.Y.copy())
    st, stats, cnt = s.integrate(T, Y, b.P, b.dt, counters=True)
    s.close()
    assert (st == 0).all() and (so["status"] == 0).all()
    compare(b, T, Y, yo, f"h2li/{precision}", oracle)
    assert np.abs(Y.sum(axis=0) - 1.0).max() < 1e-12
