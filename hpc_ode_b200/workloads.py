"""Seeded synthetic cell batches for the benchmark workloads.

The reference's own timing dataset (``ref_data/res_gri3.0.csv``, a 55,076-cell
GRI-Mech 3.0 triple flame) is not distributed with it, so seeded synthetic
states with the benchmark's shapes and distributions stand in for it.  The
mixture rule follows the reference's generator ``ref_data/generate.py:25``:
fuel/air at equivalence ratio phi with air = O2 + 3.76 N2, converted from mole
to mass fractions with the mechanism's molecular weights.

Workloads (all rtol 1e-6, atol 1e-10):
  h2_1024      h2o2,   1,024 cells, P = 101325 Pa, T0 ~ U[1000,1500] K, phi ~ U[0.5,2.0], dt 1e-3 s
  gri_32k      gri30, 32,768 cells, P ~ U[1,10] atm, T0 ~ U[1000,1800] K, phi ~ U[0.5,1.5], dt 1e-4 s
  gri_bimodal  gri30, 262,144 cells, P = 101325 Pa, T0 70% U[300,900] / 30% U[1100,2200] K,
               phi log-uniform [0.3,3.0], dt 1e-4 s
  gri_1m       gri30, 1,048,576 cells, P ~ U[1,40] atm, T0 ~ U[900,2400] K, phi ~ U[0.4,2.5], dt 1e-4 s
  h2li_grid    h2_li_2004 (9 species, 21 reactions), 10,000 cells: the reference H2 dataset's grid,
               T0 = linspace(1000,2100,100) x phi = linspace(0.5,3.5,100), P = 101325.15 Pa, dt 1e-3 s
  nc12_8k      nDodecane_Reitz (100 species, 553 reactions), 8,192 cells, P ~ U[10,60] atm,
               T0 ~ U[800,1600] K, n-dodecane/air phi ~ U[0.5,2.0], dt 1e-4 s
  kero_2k      ESTiMatE-Mech_04042022 (214 species, 1,558 reactions), 2,048 cells, P ~ U[5,40] atm,
               T0 ~ U[900,1800] K, kerosene surrogate (60 % n-C12H26, 20 % i-C8H18, 20 % toluene
               by mole)/air phi ~ U[0.5,2.0], dt 1e-4 s.  The reference's ESTiMatE dataset
               (ref_data/res_est.csv) is not distributed, so this stands in for it.
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass
from typing import Dict, Optional

import numpy as np

MECH_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "mech")
ATM = 101325.0
ESTIMATE = "ESTiMatE-Mech_04042022"


def mech_info(mech: str) -> Dict:
    base = mech[:-5] if mech.endswith(".yaml") else mech
    with open(os.path.join(MECH_DIR, f"{base}_mech.json")) as f:
        return json.load(f)


@dataclass
class Batch:
    mech: str
    T: np.ndarray        # [n]
    Y: np.ndarray        # [nsp, n]  species-major (cell index innermost), all species
    P: np.ndarray        # [n]
    dt: float
    seed: int
    name: str

    @property
    def ncells(self) -> int:
        return self.T.size

    @property
    def nsp(self) -> int:
        return self.Y.shape[0]

    def state_rows(self) -> np.ndarray:
        """Cell-major [n, nsp] integrator state [T, Y_0..Y_{nsp-2}] (reference layout)."""
        return np.concatenate([self.T[:, None], self.Y[:-1].T], axis=1).copy()

    def subset(self, idx) -> "Batch":
        return Batch(self.mech, self.T[idx].copy(), self.Y[:, idx].copy(), self.P[idx].copy(),
                     self.dt, self.seed, self.name + "[sub]")


def premixed_Y(mech: str, fuel: str, phi: np.ndarray) -> np.ndarray:
    """Mass fractions [nsp, n] of fuel/air at equivalence ratios phi."""
    info = mech_info(mech)
    names = info["species"]
    mw = np.asarray(info["mw"])
    idx = {s.upper(): i for i, s in enumerate(names)}
    n = phi.size
    X = np.zeros((len(names), n))
    if fuel == "H2":
        X[idx["H2"]] = 2.0 * phi
        X[idx["O2"]] = 1.0
        X[idx["N2"]] = 3.76
    elif fuel == "CH4":
        X[idx["CH4"]] = phi
        X[idx["O2"]] = 2.0
        X[idx["N2"]] = 7.52
    elif fuel == "kerosene":
        # three-component kerosene surrogate (mole fractions of the fuel):
        # 60 % n-dodecane, 20 % iso-octane, 20 % toluene; O2 demand per mole
        # of fuel 0.6 * 18.5 + 0.2 * 12.5 + 0.2 * 9 = 15.4
        for nm, x in (("N-C12H26", 0.6), ("I-C8H18", 0.2), ("C7H8", 0.2)):
            X[idx[nm]] = x * phi
        X[idx["O2"]] = 15.4
        X[idx["N2"]] = 15.4 * 3.76
    elif fuel == "C12H26":
        # C12H26 + 18.5 (O2 + 3.76 N2)
        X[idx["C12H26"]] = phi
        X[idx["O2"]] = 18.5
        X[idx["N2"]] = 18.5 * 3.76
    else:
        raise ValueError(fuel)
    Ym = X * mw[:, None]
    return Ym / Ym.sum(axis=0, keepdims=True)


def make(name: str, ncells: Optional[int] = None, seed: Optional[int] = None) -> Batch:
    """Build a named workload (optionally with fewer cells, same distributions)."""
    cfg = WORKLOADS[name]
    n = int(ncells if ncells is not None else cfg["ncells"])
    sd = int(seed if seed is not None else cfg["seed"])
    rng = np.random.default_rng(sd)
    kind = cfg["kind"]
    if kind == "h2":
        T = rng.uniform(1000.0, 1500.0, n)
        phi = rng.uniform(0.5, 2.0, n)
        P = np.full(n, ATM)
        Y = premixed_Y("h2o2", "H2", phi)
        mech = "h2o2"
    elif kind == "gri":
        T = rng.uniform(cfg["T"][0], cfg["T"][1], n)
        phi = rng.uniform(cfg["phi"][0], cfg["phi"][1], n)
        P = rng.uniform(cfg["P_atm"][0], cfg["P_atm"][1], n) * ATM
        Y = premixed_Y("gri30", "CH4", phi)
        mech = "gri30"
    elif kind == "h2_grid":
        # the reference's H2 dataset layout: a 100 x 100 grid of T (outer) and
        # phi (inner) at 1 atm; n < 10,000 takes evenly spaced grid points
        Tg, pg = np.meshgrid(np.linspace(1000.0, 2100.0, 100), np.linspace(0.5, 3.5, 100), indexing="ij")
        pick = np.linspace(0, Tg.size - 1, n).round().astype(int) if n <= Tg.size else np.arange(n) % Tg.size
        T = Tg.ravel()[pick].copy()
        phi = pg.ravel()[pick].copy()
        P = np.full(n, cfg["P"])
        Y = premixed_Y("h2_li_2004", "H2", phi)
        mech = "h2_li_2004"
    elif kind == "ndodecane":
        T = rng.uniform(cfg["T"][0], cfg["T"][1], n)
        phi = rng.uniform(cfg["phi"][0], cfg["phi"][1], n)
        P = rng.uniform(cfg["P_atm"][0], cfg["P_atm"][1], n) * ATM
        Y = premixed_Y("nDodecane_Reitz", "C12H26", phi)
        mech = "nDodecane_Reitz"
    elif kind == "kerosene":
        T = rng.uniform(cfg["T"][0], cfg["T"][1], n)
        phi = rng.uniform(cfg["phi"][0], cfg["phi"][1], n)
        P = rng.uniform(cfg["P_atm"][0], cfg["P_atm"][1], n) * ATM
        Y = premixed_Y(ESTIMATE, "kerosene", phi)
        mech = ESTIMATE
    elif kind == "gri_bimodal":
        cold = rng.uniform(0.0, 1.0, n) < 0.7
        T = np.where(cold, rng.uniform(300.0, 900.0, n), rng.uniform(1100.0, 2200.0, n))
        phi = np.exp(rng.uniform(np.log(0.3), np.log(3.0), n))
        P = np.full(n, ATM)
        Y = premixed_Y("gri30", "CH4", phi)
        mech = "gri30"
    else:
        raise ValueError(kind)
    return Batch(mech, T, Y, P, float(cfg["dt"]), sd, name)


WORKLOADS = {
    "h2_1024": dict(kind="h2", ncells=1024, dt=1e-3, seed=1),
    "gri_32k": dict(kind="gri", ncells=32768, dt=1e-4, seed=2, T=(1000.0, 1800.0),
                    phi=(0.5, 1.5), P_atm=(1.0, 10.0)),
    "gri_bimodal": dict(kind="gri_bimodal", ncells=262144, dt=1e-4, seed=3),
    "gri_1m": dict(kind="gri", ncells=1048576, dt=1e-4, seed=5, T=(900.0, 2400.0),
                   phi=(0.4, 2.5), P_atm=(1.0, 40.0)),
    # the reference's H2 dataset grid with its Li et al. (2004) mechanism (9 species, 21 reactions)
    "h2li_grid": dict(kind="h2_grid", ncells=10000, dt=1e-3, seed=7, P=101325.15),
    # larger mechanism (100 species, 553 reactions): diesel-like n-dodecane/air
    "nc12_8k": dict(kind="ndodecane", ncells=8192, dt=1e-4, seed=6, T=(800.0, 1600.0),
                    phi=(0.5, 2.0), P_atm=(10.0, 60.0)),
    # largest mechanism (214 species, 1,558 reactions with PLOG and lumped
    # steps): kerosene-surrogate/air at gas-turbine pressures
    "kero_2k": dict(kind="kerosene", ncells=2048, dt=1e-4, seed=8, T=(900.0, 1800.0),
                    phi=(0.5, 2.0), P_atm=(5.0, 40.0)),
}
RTOL, ATOL = 1e-6, 1e-10


def serving_requests(n_requests: int, seed: int = 4, min_cells: int = 1024, max_cells: int = 262144):
    """The serving workload: requests of log-uniform size in [min_cells,
    max_cells], drawn 60 % from the H2 distributions (h2_1024) and 40 % from the
    GRI distributions (gri_32k), each with dt uniform in {1e-5, 1e-4} s.
    Deterministic for a seed; yields Batch objects."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(min_cells), np.log(max_cells)
    for i in range(n_requests):
        n = int(np.exp(rng.uniform(lo, hi)))
        wl = "h2_1024" if rng.random() < 0.6 else "gri_32k"
        dt = float(rng.choice([1e-5, 1e-4]))
        b = make(wl, n, seed=seed * 1_000_003 + i)
        b.dt = dt
        b.name = f"serve[{i}]:{wl}:{n}:{dt:g}"
        yield b

