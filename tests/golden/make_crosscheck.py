"""Generate the independent-integrator fixture that pins the CPU oracle's
CVODE-semantics BDF (oracle/bdf_oracle.c) where the reference cannot: the
reference's CVODE (SUNDIALS v6.3.0, an un-vendored submodule) is absent here, so
two other stiff integrators stand in for it on the same right-hand side:

  * VODE (scipy.integrate.ode 'vode', method='bdf', order 5, analytic
    Jacobian): the Fortran variable-order BDF that CVODE was written from
    (same Nordsieck form and error control);
  * Radau IIA order 5 (scipy.integrate.solve_ivp 'Radau', analytic Jacobian):
    an implicit Runge-Kutta method, unrelated to BDF.

Both call the oracle's restated chemistry (its GRI-Mech 3.0 tables are pinned to
the reference's own pyJac C by gri30_chem_golden.npz) through ctypes, over dt
from the seeded initial states of three workloads, at two tolerance levels:
rtol 1e-10 / atol 1e-14 (the oracle's own setting) and tight (VODE rtol 1e-12,
Radau rtol 1e-13, atol 1e-16; Radau there is the converged solution), so the
oracle's error at rtol 1e-10 can be judged against a converged solution and
beside VODE's:

  h2_1024   256 cells (H2/O2, 10 unknowns, dt 1e-3 s)
  gri_32k   256 cells (GRI-Mech 3.0, 53 unknowns, dt 1e-4 s)
  gri_1m    128 cells (GRI-Mech 3.0, the 1M-cell workload's wider T / P / phi)

    python tests/golden/make_crosscheck.py [--procs 8]

Writes crosscheck_vode_radau.npz: per workload the initial states (``<wl>_y0``),
pressures, dt, and the final states of VODE and Radau at rtol 1e-10
(``<wl>_vode``, ``<wl>_radau``) and tight (``<wl>_vode_tight``,
``<wl>_radau_tight``).  About ten minutes on 8 cores.  Test infrastructure only.
"""
from __future__ import annotations

import argparse
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

SETS = (("h2_1024", 256, 101), ("gri_32k", 256, 102), ("gri_1m", 128, 103))
RTOL, ATOL = 1e-10, 1e-14
VODE_TIGHT, RADAU_TIGHT, ATOL_TIGHT = 1e-12, 1e-13, 1e-16
OUT = os.path.join(HERE, "crosscheck_vode_radau.npz")


def vode(f, J, y0, dt, rtol, atol):
    from scipy.integrate import ode
    r = ode(f, J).set_integrator("vode", method="bdf", order=5, with_jacobian=True,
                                 rtol=rtol, atol=atol, nsteps=2000000)
    r.set_initial_value(y0, 0.0)
    y = r.integrate(dt)
    return y if r.successful() else np.full_like(y0, np.nan)


def radau(f, J, y0, dt, rtol, atol):
    from scipy.integrate import solve_ivp
    rr = solve_ivp(f, (0.0, dt), y0, method="Radau", jac=J, rtol=rtol, atol=atol)
    return rr.y[:, -1] if rr.success else np.full_like(y0, np.nan)


def solve_cell(args):
    """VODE and Radau final states of one cell at both tolerance levels (run in
    a worker process)."""
    mech, P, dt, y0 = args
    sys.path.insert(0, ROOT)
    from oracle import pyoracle
    o = pyoracle.get()
    f = lambda t, y: o.dydt(mech, P, y)  # noqa: E731
    J = lambda t, y: o.jacob(mech, P, y)  # noqa: E731
    return (vode(f, J, y0, dt, RTOL, ATOL), radau(f, J, y0, dt, RTOL, ATOL),
            vode(f, J, y0, dt, VODE_TIGHT, ATOL_TIGHT), radau(f, J, y0, dt, RADAU_TIGHT, ATOL_TIGHT))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--procs", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    from hpc_ode_b200 import workloads as W
    out = {}
    ctx = mp.get_context("spawn")
    with ctx.Pool(args.procs) as pool:
        for wl, n, seed in SETS:
            b = W.make(wl, n, seed=seed)
            ys = b.state_rows()
            res = pool.map(solve_cell, [(b.mech, float(b.P[c]), float(b.dt), ys[c]) for c in range(n)],
                           chunksize=1)
            out[f"{wl}_y0"] = ys
            out[f"{wl}_P"] = b.P.copy()
            out[f"{wl}_dt"] = np.float64(b.dt)
            keys = ("vode", "radau", "vode_tight", "radau_tight")
            for i, k in enumerate(keys):
                out[f"{wl}_{k}"] = np.stack([r[i] for r in res])
            bad = np.zeros(n, dtype=bool)
            for k in keys:
                bad |= np.isnan(out[f"{wl}_{k}"]).any(axis=1)
            print(f"{wl}: {n} cells, {int(bad.sum())} failed", flush=True)
    np.savez_compressed(OUT, mech=np.array([W.WORKLOADS[wl]["kind"] for wl, _, _ in SETS]),
                        rtol=RTOL, atol=ATOL, vode_tight=VODE_TIGHT, radau_tight=RADAU_TIGHT,
                        atol_tight=ATOL_TIGHT, **out)
    print(OUT)


if __name__ == "__main__":
    main()
