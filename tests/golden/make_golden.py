"""Generate the golden fixtures under tests/golden/ from the reference.

Run in a checkout that has the reference tree (REF_DIR; default oracle/refpath.py's
reference_dir(): HPC_ODE_REFERENCE, else the checkout's default location) and its pyJac C
built by ``make -C oracle ref``:

    python tests/golden/make_golden.py [REF_DIR]

Writes:
  gri30_chem_golden.npz  seeded GRI-Mech 3.0 states with the reference pyJac
                         ``dydt`` (src/Mechanism/CPU/dydt.c:7) and
                         ``eval_jacob`` (src/Mechanism/CPU/jacob.c:3) outputs;
  e2e_gri100.npz         the reference's 99-cell E2E input
                         (tests/Integrators/data/res_gri_100.csv) and its serial
                         CVODE output (E2Etests/100/results_serial100.csv);
  enthalpy_ref.npz       states with the mixture enthalpy the reference's data
                         files carry (ENTHA, computed by Cantera): every 50th
                         row of ref_data/res_h2.csv (h2_li_2004) and the 99 rows
                         of tests/Integrators/data/res_gri_100.csv (gri30).

``python tests/golden/make_golden.py REF_DIR --only enthalpy`` writes only the last.
The fixtures are small and committed; the GPU tests never read the reference.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hpc_ode_b200 import workloads as W  # noqa: E402
from oracle import pyoracle  # noqa: E402


def chem_states(n: int, seed: int = 11):
    """Premixed and partially burnt GRI states over the benchmark ranges."""
    rng = np.random.default_rng(seed)
    T = rng.uniform(300.0, 2400.0, n)
    P = rng.uniform(1.0, 40.0, n) * W.ATM
    phi = np.exp(rng.uniform(np.log(0.3), np.log(3.0), n))
    Y = W.premixed_Y("gri30", "CH4", phi)          # [53, n]
    for c in range(n):
        if c % 2:   # partially burnt: log-normal radical pool mixed in
            Yr = np.abs(rng.lognormal(-9.0, 3.0, 53))
            Yr /= Yr.sum()
            w = rng.uniform(0.05, 0.6)
            Y[:, c] = (1 - w) * Y[:, c] + w * Yr
    y = np.concatenate([T[:, None], Y[:-1].T], axis=1)
    return y, P


def main(ref_dir: str):
    o = pyoracle.get()
    if not o.has_ref():
        raise SystemExit("oracle/_ref/libpyjac_gri30.so missing: run `make -C oracle ref` first")
    y, P = chem_states(64)
    dydt = np.stack([o.ref_dydt(P[i], y[i]) for i in range(len(P))])
    nj = 16
    jac = np.stack([o.ref_jacob(P[i], y[i]) for i in range(nj)])
    np.savez_compressed(os.path.join(HERE, "gri30_chem_golden.npz"), y=y, P=P, dydt=dydt,
                        jac=jac, jac_count=np.int64(nj))

    def read_csv(path):
        d = np.loadtxt(path, delimiter=",", skiprows=1)
        return d[:, 0:53], d[:, 54]   # species, TEMPE (ENTHA is column 53)

    Yin, Tin = read_csv(os.path.join(ref_dir, "tests/Integrators/data/res_gri_100.csv"))
    Yout, Tout = read_csv(os.path.join(ref_dir, "E2Etests/100/results_serial100.csv"))
    np.savez_compressed(os.path.join(HERE, "e2e_gri100.npz"), Y_in=Yin, T_in=Tin, Y_out=Yout,
                        T_out=Tout, P=np.float64(101325.15), dt=np.float64(1e-3))
    print("wrote", os.listdir(HERE))


def enthalpy_fixture(ref_dir: str):
    h2 = np.genfromtxt(os.path.join(ref_dir, "ref_data/res_h2.csv"), delimiter=",", names=True)[::50]
    gri = np.loadtxt(os.path.join(ref_dir, "tests/Integrators/data/res_gri_100.csv"), delimiter=",", skiprows=1)
    np.savez_compressed(
        os.path.join(HERE, "enthalpy_ref.npz"),
        h2_T=h2["TEMPE"], h2_Y=np.stack([h2[f"CO{k}"] for k in range(9)]), h2_h=h2["ENTHA"],
        gri_T=gri[:, 54], gri_Y=np.ascontiguousarray(gri[:, 0:53].T), gri_h=gri[:, 53])
    print("wrote enthalpy_ref.npz")


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--") and a != "enthalpy"]
    from oracle.refpath import reference_dir
    ref = args[0] if args else reference_dir()
    if not ref:
        raise SystemExit("no reference checkout: pass REF_DIR or set HPC_ODE_REFERENCE")
    if "--only" in sys.argv and sys.argv[sys.argv.index("--only") + 1] == "enthalpy":
        enthalpy_fixture(ref)
    else:
        main(ref)
        enthalpy_fixture(ref)
