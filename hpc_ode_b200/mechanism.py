"""Cantera-YAML mechanism parser and table generator.

The reference builds its chemistry from pyJac-generated C/CUDA
(``pyJac_mechanism_generator.sh:3-4`` runs pyJac on ``gri30.cti``; the output
lives in ``src/Mechanism/CPU`` and ``src/Mechanism/GPU``).  pyJac is not part of
the reference tree, so this module restates the pyJac conventions that decide
the numbers it produces, checked against the compiled reference kernels:

* SI-kmol units: ``R = 8314.4621 J/kmol/K`` (``src/Mechanism/CPU/chem_utils.c:71``),
  pre-exponentials converted from (cm^3/mol)^(n-1)/s, activation energies
  from cal/mol with 4.184 J/cal (``rxn_rates.c:37``: ``Ea/R = 3150.154...``
  for ``O + H2 <=> H + OH``).
* State ``y = [T, Y_0 .. Y_{n-2}]``; the last species closes the mass balance
  (``mechanism.h:5`` ``last_spec 52``, ``chem_utils.c:7-13``).
* A species that appears on both sides of an elementary reaction (a
  "catalyst", e.g. ``H + 2 O2 <=> HO2 + O2``) is removed from both sides and
  becomes the sole third body of the reaction, with the third-body
  concentration written as ``m - sum_{k != s} C_k``
  (``rxn_rates_pres_mod.c:38-39`` reaction 33, ``rxn_rates.c:404-414``).
* Third-body concentration ``m + sum_k (eff_k - 1) C_k`` in species-index
  order (``rxn_rates_pres_mod.c:22``); Lindemann ``Pr/(1+Pr)`` and Troe
  blending (``rxn_rates_pres_mod.c:28-33,65-73``); for falloff reactions the
  forward rate uses the high-pressure limit and ``pres_mod`` carries the
  blending (``spec_rates.c``).
* Equilibrium constants from NASA-7 Gibbs functions with each species' own
  mid temperature (``rxn_rates.c:2803-2807``).

``Mechanism.emit_header`` writes the tables as a C header that the CPU oracle
(``oracle/chem_oracle.c``) and the CUDA library both include.
"""
from __future__ import annotations

import math
import os
import re
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import yaml


class _MechLoader(yaml.SafeLoader):
    """YAML 1.1 loader that keeps ``NO``/``ON``/``Y``... as strings (species names)."""


_MechLoader.yaml_implicit_resolvers = {
    k: [(tag, rx) for tag, rx in v if tag != "tag:yaml.org,2002:bool"]
    for k, v in yaml.SafeLoader.yaml_implicit_resolvers.items()
}
_MechLoader.add_implicit_resolver(
    "tag:yaml.org,2002:bool", re.compile(r"^(?:true|True|TRUE|false|False|FALSE)$"),
    list("tTfF"))

RU = 8314.4621            # J / kmol / K  (pyJac chem_utilities.RU)
RU_CAL = 8.3144621 / 4.184  # cal / mol / K
PA_ATM = 101325.0

# Atomic weights used by pyJac/Cantera for the mechanisms in the reference
# (checked against the printed molecular weights in src/Mechanism/CPU/dydt.c).
ELEMENT_WEIGHTS = {
    "H": 1.008, "O": 15.999, "C": 12.011, "N": 14.007, "Ar": 39.95, "AR": 39.95,
    "He": 4.002602, "HE": 4.002602, "E": 5.48579909e-4,
}

T_ELEMENTARY, T_THIRD_BODY, T_LINDEMANN, T_TROE, T_PLOG = 0, 1, 2, 3, 4
TYPE_NAMES = {T_ELEMENTARY: "elementary", T_THIRD_BODY: "three-body",
              T_LINDEMANN: "lindemann", T_TROE: "troe", T_PLOG: "plog"}


@dataclass
class Species:
    name: str
    mw: float
    tmid: float
    lo: List[float]
    hi: List[float]


@dataclass
class Reaction:
    index: int
    equation: str
    rtype: int
    reversible: bool
    reac: List[Tuple[int, int]]          # (species, stoich) in equation order
    prod: List[Tuple[int, float]]        # fractional only in irreversible reactions
    A: float = 0.0                       # SI kmol units; high-P limit for falloff
    b: float = 0.0
    EaR: float = 0.0                     # activation temperature [K]
    A0: float = 0.0                      # low-P limit (falloff only)
    b0: float = 0.0
    EaR0: float = 0.0
    troe: Tuple[float, float, float, float] = (0.0, 0.0, 0.0, 0.0)
    troe_has_T2: bool = False
    tb: List[Tuple[int, float]] = field(default_factory=list)  # (species, eff-1)
    catalyst: Optional[int] = None       # species made the sole third body
    # pressure-dependent Arrhenius (PLOG): levels sorted by pressure, each
    # (P [Pa], [(A [SI kmol units], b, Ea/R [K]), ...]) -- the rate at a level
    # is the sum of its terms
    plog: List[Tuple[float, List[Tuple[float, float, float]]]] = field(default_factory=list)

    @property
    def has_third_body(self) -> bool:
        return self.rtype != T_ELEMENTARY

    def net_stoich(self, nsp: int) -> Dict[int, float]:
        d: Dict[int, float] = {}
        for s, nu in self.reac:
            d[s] = d.get(s, 0) - nu
        for s, nu in self.prod:
            d[s] = d.get(s, 0) + nu
        return {k: v for k, v in d.items() if v != 0}


def _nu(v: float):
    """A stoichiometric coefficient: int when integral, else float."""
    return int(v) if v == int(v) else float(v)


def _parse_side(side: str) -> List[Tuple[str, float]]:
    out: List[Tuple[str, float]] = []
    for tok in side.split(" + "):
        tok = tok.strip()
        if not tok:
            continue
        m = re.match(r"^(\d+(?:\.\d+)?)\s+(\S+)$", tok)
        if m:
            out.append((m.group(2), _nu(float(m.group(1)))))
        else:
            out.append((tok, 1))
    return out


def _merge(side: List[Tuple[str, float]]) -> List[Tuple[str, float]]:
    order: List[str] = []
    cnt: Dict[str, float] = {}
    for name, nu in side:
        if name not in cnt:
            order.append(name)
            cnt[name] = 0
        cnt[name] += nu
    return [(n, cnt[n]) for n in order]


class Mechanism:
    """Species + reactions of a gas mechanism with pyJac conventions applied."""

    def __init__(self, name: str, species: List[Species], reactions: List[Reaction]):
        self.name = name
        self.species = species
        self.reactions = reactions
        self.nsp = len(species)
        self.nrxn = len(reactions)
        self.n_unknowns = self.nsp  # T + (nsp - 1) mass fractions

    # ------------------------------------------------------------------ parse
    @classmethod
    def from_yaml(cls, path: str, name: Optional[str] = None) -> "Mechanism":
        with open(path) as f:
            d = yaml.load(f, Loader=_MechLoader)
        units = d.get("units", {})
        length = units.get("length", "m")
        quantity = units.get("quantity", "kmol")
        ea_unit = units.get("activation-energy", "J/kmol")
        if length != "cm" or quantity != "mol" or ea_unit != "cal/mol":
            raise NotImplementedError(f"unsupported unit system {units}")
        phase = d["phases"][0]
        sp_names = phase["species"]
        sp_by_name = {s["name"]: s for s in d["species"]}
        species: List[Species] = []
        for nm in sp_names:
            s = sp_by_name[nm]
            mw = sum(ELEMENT_WEIGHTS[el] * n for el, n in s["composition"].items())
            th = s["thermo"]
            if th["model"] != "NASA7":
                raise NotImplementedError(f"thermo model {th['model']}")
            tr = th["temperature-ranges"]
            data = th["data"]
            if len(tr) == 2:
                lo = hi = list(map(float, data[0]))
                tmid = tr[1]
            else:
                lo, hi = list(map(float, data[0])), list(map(float, data[1]))
                tmid = tr[1]
            species.append(Species(nm, mw, float(tmid), lo, hi))
        idx = {s.name: i for i, s in enumerate(species)}

        def conv_A(A: float, order: int) -> float:
            # (cm^3/mol)^(order-1) / s  ->  (m^3/kmol)^(order-1) / s
            return A * (1e-3) ** (order - 1)

        def conv_Ea(Ea: float) -> float:
            return Ea * 4.184 / 8.3144621

        reactions: List[Reaction] = []
        for i, r in enumerate(d["reactions"]):
            eq = r["equation"]
            rtype_s = r.get("type", "elementary")
            if "<=>" in eq:
                lhs, rhs = eq.split("<=>")
                rev = True
            elif "=>" in eq:
                lhs, rhs = eq.split("=>")
                rev = False
            elif " = " in eq:
                lhs, rhs = eq.split(" = ")
                rev = True
            else:
                raise ValueError(eq)
            lhs, rhs = lhs.strip(), rhs.strip()
            falloff_m = None
            for side_name in ("lhs", "rhs"):
                s = lhs if side_name == "lhs" else rhs
                m = re.search(r"\s*\(\+\s*([^)]+)\)\s*$", s)
                if m:
                    falloff_m = m.group(1).strip()
                    s = s[: m.start()].strip()
                if side_name == "lhs":
                    lhs = s
                else:
                    rhs = s
            L = _merge(_parse_side(lhs))
            R = _merge(_parse_side(rhs))
            has_M = any(n == "M" for n, _ in L)
            L = [(n, nu) for n, nu in L if n != "M"]
            R = [(n, nu) for n, nu in R if n != "M"]
            if r.get("orders") or r.get("negative-A"):
                raise NotImplementedError(f"reaction {i}: non-standard orders / negative A")

            def rate(which: str, order: int, r=r):
                rc = r["rate-constant"] if which == "rate" else r[which]
                return conv_A(float(rc["A"]), order), float(rc["b"]), conv_Ea(float(rc["Ea"]))

            troe = None
            if "Troe" in r:
                t = r["Troe"]
                troe = (float(t["A"]), float(t["T3"]), float(t["T1"]), float(t.get("T2", 0.0)), "T2" in t)
            if "SRI" in r:
                raise NotImplementedError(f"reaction {i}: SRI falloff")
            if rtype_s == "three-body" or (has_M and rtype_s == "elementary"):
                kind = "three-body"
            elif rtype_s in ("elementary", "falloff"):
                kind = rtype_s
            else:
                raise NotImplementedError(f"reaction {i}: type {rtype_s}")
            reactions.append(cls._make_reaction(
                i, eq, rev, kind, L, R, falloff_m, rate, "rate", "high-P-rate-constant",
                "low-P-rate-constant", troe, r.get("efficiencies", {}),
                float(r.get("default-efficiency", 1.0)), idx, len(species)))
        nm = name or os.path.splitext(os.path.basename(path))[0]
        return cls(nm, species, reactions)

    @classmethod
    def from_ctml(cls, path: str, name: Optional[str] = None) -> "Mechanism":
        """Parse a Cantera CTML (XML) mechanism: NASA-7 species, Arrhenius,
        three-body, Lindemann/Troe falloff and pressure-dependent Arrhenius
        (``type="plog"``) reactions, fractional product coefficients in
        irreversible reactions.  CTML stores A in SI kmol units and names E's
        (and P's) unit on each element."""
        import xml.etree.ElementTree as ET
        root = ET.parse(path).getroot()
        phase = root.find("phase")
        sp_names = phase.find("speciesArray").text.split()
        sp_el = {e.get("name"): e for e in root.iter("species")}
        species: List[Species] = []
        for nm in sp_names:
            e = sp_el[nm]
            comp = {}
            for tok in (e.find("atomArray").text or "").split():
                el, n = tok.split(":")
                comp[el] = float(n)
            mw = sum(ELEMENT_WEIGHTS[el] * n for el, n in comp.items())
            polys = sorted(e.find("thermo").findall("NASA"), key=lambda x: float(x.get("Tmin")))
            coeffs = [[float(v) for v in p.find("floatArray").text.replace(",", " ").split()] for p in polys]
            if len(polys) == 1:
                lo = hi = coeffs[0]
                tmid = float(polys[0].get("Tmax"))
            elif len(polys) == 2:
                lo, hi = coeffs
                tmid = float(polys[0].get("Tmax"))
            else:
                raise NotImplementedError(f"species {nm}: {len(polys)} NASA ranges")
            species.append(Species(nm, mw, tmid, lo, hi))
        idx = {s.name: i for i, s in enumerate(species)}
        e_to_K = {"cal/mol": 4.184 / 8.3144621, "kcal/mol": 4184.0 / 8.3144621, "J/mol": 1.0 / 8.3144621,
                  "kJ/mol": 1000.0 / 8.3144621, "J/kmol": 1.0 / 8314.4621, "K": 1.0}

        p_to_Pa = {"atm": PA_ATM, "Pa": 1.0, "bar": 1.0e5}

        def side(text: str) -> List[Tuple[str, float]]:
            out = []
            for tok in (text or "").split():
                nm, nu = tok.rsplit(":", 1)
                out.append((nm, _nu(float(nu))))
            return _merge(out)

        reactions: List[Reaction] = []
        for i, rxn in enumerate(root.iter("reaction")):
            eq = rxn.find("equation").text
            rev = rxn.get("reversible", "yes") == "yes"
            t = rxn.get("type", "elementary")
            rc = rxn.find("rateCoeff")
            if rxn.find("order") is not None or rc.find("Arrhenius") is None or \
                    rc.find("Arrhenius").get("type") == "stick":
                raise NotImplementedError(f"reaction {i}: unsupported rate form")
            arr = {a.get("name", "rate"): a for a in rc.findall("Arrhenius")}

            def arrhenius(a):
                A = float(a.find("A").text)
                if A < 0:
                    raise NotImplementedError("negative A")
                Ee = a.find("E")
                return A, float(a.find("b").text), float(Ee.text) * e_to_K[Ee.get("units", "cal/mol")]

            def rate(which: str, order: int, arr=arr, rc=rc):
                if which == "plog":
                    levels: Dict[float, List[Tuple[float, float, float]]] = {}
                    for a in rc.findall("Arrhenius"):
                        pe = a.find("P")
                        levels.setdefault(float(pe.text) * p_to_Pa[pe.get("units", "Pa")], []).append(arrhenius(a))
                    return sorted(levels.items())
                return arrhenius(arr["k0" if which == "low" else "rate"])

            troe = None
            fo = rc.find("falloff")
            if fo is not None:
                if fo.get("type") == "Troe":
                    v = [float(x) for x in fo.text.split()]
                    troe = (v[0], v[1], v[2], v[3] if len(v) > 3 else 0.0, len(v) > 3)
                elif fo.get("type") != "Lindemann":
                    raise NotImplementedError(f"reaction {i}: falloff {fo.get('type')}")
            effs, default_eff = {}, 1.0
            ef = rc.find("efficiencies")
            if ef is not None:
                default_eff = float(ef.get("default", "1.0"))
                for tok in (ef.text or "").split():
                    nm, v = tok.rsplit(":", 1)
                    effs[nm] = float(v)
            if t == "threeBody":
                kind = "three-body"
            elif t == "falloff":
                kind = "falloff"
            elif t == "elementary":
                kind = "elementary"
            elif t == "plog":
                kind = "plog"
            else:
                raise NotImplementedError(f"reaction {i}: type {t}")
            L, R = side(rxn.find("reactants").text), side(rxn.find("products").text)
            reactions.append(cls._make_reaction(
                i, eq, rev, kind, L, R, "M" if kind == "falloff" else None, rate, "rate", "rate", "low",
                troe, effs, default_eff, idx, len(species)))
        nm = name or os.path.splitext(os.path.basename(path))[0]
        return cls(nm, species, reactions)

    @classmethod
    def _make_reaction(cls, i, eq, rev, kind, L, R, falloff_m, rate, k_elem, k_hi, k_lo, troe, effs,
                       default_eff, idx, nsp) -> Reaction:
        """One reaction with pyJac's conventions.  rate(key, order) gives
        (A [SI kmol units], b, Ea/R [K]) for the rate expression named key."""
        order = sum(nu for _, nu in L)
        if any(nu != int(nu) for _, nu in L) or (rev and any(nu != int(nu) for _, nu in R)):
            raise NotImplementedError(f"reaction {i}: fractional stoichiometry outside the products "
                                      f"of an irreversible reaction")
        rx = Reaction(index=i, equation=eq, rtype=T_ELEMENTARY, reversible=rev, reac=[], prod=[])
        if kind == "plog":
            # k(T, P): ln k interpolated linearly in ln P between the bracketing
            # levels, clamped to the end levels (Cantera's PlogRate)
            rx.rtype = T_PLOG
            rx.plog = [(p, list(terms)) for p, terms in rate("plog", order)]
            rx.A, rx.b, rx.EaR = rx.plog[0][1][0]
        elif kind == "elementary":
            rx.A, rx.b, rx.EaR = rate(k_elem, order)
            # pyJac: in a termolecular step (three molecules on either
            # side) a species found on both sides becomes the sole third
            # body; bimolecular steps such as H + CH3O <=> H + CH2OH stay
            # elementary (rxn_rates.c:764-766 vs rxn_rates_pres_mod.c:38).
            lnames = {n for n, _ in L}
            common = [n for n, _ in R if n in lnames]
            termolecular = max(sum(nu for _, nu in L), sum(nu for _, nu in R)) >= 3
            integral = all(nu == int(nu) for _, nu in R)   # lumped steps with fractional
            if common and termolecular and integral:         # products stay elementary
                if len(common) != 1:
                    raise NotImplementedError(f"reaction {i}: several catalysts")
                c = common[0]
                nl = dict(L)[c]
                nr = dict(R)[c]
                k = min(nl, nr)
                L = [(n, nu - (k if n == c else 0)) for n, nu in L]
                R = [(n, nu - (k if n == c else 0)) for n, nu in R]
                L = [(n, nu) for n, nu in L if nu > 0]
                R = [(n, nu) for n, nu in R if nu > 0]
                if k != 1:
                    raise NotImplementedError(f"reaction {i}: catalyst count {k}")
                rx.rtype = T_THIRD_BODY
                rx.catalyst = idx[c]
                ci = idx[c]
                rx.tb = [(j, -1.0) for j in range(nsp) if j != ci]
        elif kind == "three-body":
            rx.A, rx.b, rx.EaR = rate(k_elem, order + 1)
            rx.rtype = T_THIRD_BODY
            rx.tb = cls._tb_list(effs, default_eff, idx, nsp)
        elif kind == "falloff":
            if falloff_m not in (None, "M"):
                raise NotImplementedError(f"reaction {i}: falloff with (+{falloff_m})")
            rx.A, rx.b, rx.EaR = rate(k_hi, order)
            rx.A0, rx.b0, rx.EaR0 = rate(k_lo, order + 1)
            rx.tb = cls._tb_list(effs, default_eff, idx, nsp)
            if troe is not None:
                rx.rtype = T_TROE
                rx.troe = troe[:4]
                rx.troe_has_T2 = troe[4]
            else:
                rx.rtype = T_LINDEMANN
        else:
            raise NotImplementedError(f"reaction {i}: type {kind}")
        rx.reac = [(idx[n], nu) for n, nu in L]
        rx.prod = [(idx[n], nu) for n, nu in R]
        return rx

    @staticmethod
    def _tb_list(effs, default_eff, idx, nsp) -> List[Tuple[int, float]]:
        if default_eff != 1.0:
            raise NotImplementedError("default-efficiency != 1")
        out = []
        eff_by_idx = {idx[n]: float(e) for n, e in effs.items() if n in idx}
        for j in sorted(eff_by_idx):
            a = eff_by_idx[j] - 1.0
            if a != 0.0:
                out.append((j, a))
        return out

    # ------------------------------------------------------------- summaries
    def counts(self) -> Dict[str, int]:
        c = {"species": self.nsp, "reactions": self.nrxn,
             "reversible": sum(r.reversible for r in self.reactions),
             "pres_mod": sum(r.has_third_body for r in self.reactions)}
        for t, n in TYPE_NAMES.items():
            c[n] = sum(r.rtype == t for r in self.reactions)
        c["catalyst_converted"] = sum(r.catalyst is not None for r in self.reactions)
        return c

    def max_participants(self) -> int:
        return max(max(len(r.reac), len(r.prod)) for r in self.reactions)

    # ------------------------------------------------------------------ emit
    def emit_header(self, path: str) -> None:
        """Write the mechanism tables as a C header (plain C99, no CUDA)."""
        n, nr = self.nsp, self.nrxn
        P = self.max_participants()
        pfx = "MECH_" + re.sub(r"[^A-Za-z0-9]", "_", self.name).upper()
        tag = re.sub(r"[^A-Za-z0-9]", "_", self.name).lower()

        def fa(vals) -> str:
            return ", ".join(repr(float(v)) if not math.isinf(v) else "0.0" for v in vals)

        def ia(vals) -> str:
            return ", ".join(str(int(v)) for v in vals)

        reac_sp, reac_nu, prod_sp, prod_nu = [], [], [], []
        for r in self.reactions:
            rs = r.reac + [(-1, 0)] * (P - len(r.reac))
            ps = r.prod + [(-1, 0)] * (P - len(r.prod))
            reac_sp += [s for s, _ in rs]
            reac_nu += [v for _, v in rs]
            prod_sp += [s for s, _ in ps]
            prod_nu += [v for _, v in ps]
        tb_off = [0]
        tb_sp: List[int] = []
        tb_al: List[float] = []
        for r in self.reactions:
            for s, a in r.tb:
                tb_sp.append(s)
                tb_al.append(a)
            tb_off.append(len(tb_sp))
        if not tb_sp:
            tb_sp, tb_al = [0], [0.0]
        logA = [math.log(r.A) if r.A > 0 else 0.0 for r in self.reactions]
        logA0 = [math.log(r.A0) if r.A0 > 0 else 0.0 for r in self.reactions]
        # denominator that makes every product coefficient integral (kernels
        # encode nu * NU_DEN in small integer fields)
        nu_den = next((d for d in (1, 2, 4) if all(abs(v * d - round(v * d)) < 1e-12
                                                   for r in self.reactions for _, v in r.prod)), None)
        if nu_den is None:
            raise NotImplementedError("product coefficients need a denominator above 4")
        # PLOG tables: reaction r's levels are plog_off[r] .. plog_off[r+1]-1;
        # level l's Arrhenius terms are plog_term_off[l] .. plog_term_off[l+1]-1
        plog_off, plog_lnP, plog_toff = [0], [], [0]
        plog_A, plog_b, plog_EaR = [], [], []
        for r in self.reactions:
            for P_, terms in r.plog:
                plog_lnP.append(math.log(P_))
                for A_, b_, E_ in terms:
                    plog_A.append(A_)
                    plog_b.append(b_)
                    plog_EaR.append(E_)
                plog_toff.append(len(plog_A))
            plog_off.append(len(plog_lnP))
        nlev, nterm = max(len(plog_lnP), 1), max(len(plog_A), 1)
        if not plog_lnP:
            plog_lnP, plog_A, plog_b, plog_EaR = [0.0], [0.0], [0.0], [0.0]
            plog_toff = [0, 0]
        plog_logA = [math.log(a) if a > 0 else 0.0 for a in plog_A]
        # units of the kernels' balanced species gather: each species' (reaction,
        # net coefficient) entries cut into runs of at most 24 (kGatherUnit in
        # csrc/mech_dev.h); sizes the per-warp shared scratch exactly
        entries = [0] * n
        for r in self.reactions:
            for k in r.net_stoich(n):
                entries[k] += 1
        n_units = sum(-(-e // 24) for e in entries)
        lines = []
        w = lines.append
        w(f"/* Generated by hpc_ode_b200/mechanism.py from {self.name} -- do not edit. */")
        w(f"#ifndef {pfx}_H")
        w(f"#define {pfx}_H")
        w(f"/* {self.counts()} */")
        w(f"#define {pfx}_NSP {n}")
        w(f"#define {pfx}_NRXN {nr}")
        w(f"#define {pfx}_MAXP {P}")
        w(f"#define {pfx}_NTB {len(tb_sp)}")
        w(f"#define {pfx}_NU_DEN {nu_den}")
        w(f"#define {pfx}_NUNITS {n_units}")
        w(f"#define {pfx}_NPLOG {sum(r.rtype == T_PLOG for r in self.reactions)}")
        w(f"#define {pfx}_NPLOGLEV {nlev}")
        w(f"#define {pfx}_NPLOGTERM {nterm}")
        w(f"static const char* const {tag}_species_names[{n}] = {{{', '.join(chr(34)+s.name+chr(34) for s in self.species)}}};")
        w(f"static const double {tag}_mw[{n}] = {{{fa(s.mw for s in self.species)}}};")
        w(f"static const double {tag}_tmid[{n}] = {{{fa(s.tmid for s in self.species)}}};")
        w(f"static const double {tag}_nasa_lo[{n * 7}] = {{{fa(v for s in self.species for v in s.lo)}}};")
        w(f"static const double {tag}_nasa_hi[{n * 7}] = {{{fa(v for s in self.species for v in s.hi)}}};")
        w(f"static const int {tag}_rxn_type[{nr}] = {{{ia(r.rtype for r in self.reactions)}}};")
        w(f"static const int {tag}_rxn_rev[{nr}] = {{{ia(int(r.reversible) for r in self.reactions)}}};")
        w(f"static const double {tag}_rxn_A[{nr}] = {{{fa(r.A for r in self.reactions)}}};")
        w(f"static const double {tag}_rxn_logA[{nr}] = {{{fa(logA)}}};")
        w(f"static const double {tag}_rxn_b[{nr}] = {{{fa(r.b for r in self.reactions)}}};")
        w(f"static const double {tag}_rxn_EaR[{nr}] = {{{fa(r.EaR for r in self.reactions)}}};")
        w(f"static const double {tag}_rxn_A0[{nr}] = {{{fa(r.A0 for r in self.reactions)}}};")
        w(f"static const double {tag}_rxn_logA0[{nr}] = {{{fa(logA0)}}};")
        w(f"static const double {tag}_rxn_b0[{nr}] = {{{fa(r.b0 for r in self.reactions)}}};")
        w(f"static const double {tag}_rxn_EaR0[{nr}] = {{{fa(r.EaR0 for r in self.reactions)}}};")
        w(f"static const double {tag}_rxn_troe[{nr * 4}] = {{{fa(v for r in self.reactions for v in r.troe)}}};")
        w(f"static const int {tag}_rxn_troe_T2[{nr}] = {{{ia(int(r.troe_has_T2) for r in self.reactions)}}};")
        w(f"static const int {tag}_rxn_reac_sp[{nr * P}] = {{{ia(reac_sp)}}};")
        w(f"static const int {tag}_rxn_reac_nu[{nr * P}] = {{{ia(reac_nu)}}};")
        w(f"static const int {tag}_rxn_prod_sp[{nr * P}] = {{{ia(prod_sp)}}};")
        w(f"static const double {tag}_rxn_prod_nu[{nr * P}] = {{{fa(prod_nu)}}};")
        w(f"static const int {tag}_rxn_tb_off[{nr + 1}] = {{{ia(tb_off)}}};")
        w(f"static const int {tag}_tb_sp[{len(tb_sp)}] = {{{ia(tb_sp)}}};")
        w(f"static const double {tag}_tb_alpha[{len(tb_al)}] = {{{fa(tb_al)}}};")
        w(f"static const int {tag}_plog_off[{nr + 1}] = {{{ia(plog_off)}}};")
        w(f"static const double {tag}_plog_lnP[{nlev}] = {{{fa(plog_lnP)}}};")
        w(f"static const int {tag}_plog_term_off[{nlev + 1}] = {{{ia(plog_toff)}}};")
        w(f"static const double {tag}_plog_A[{nterm}] = {{{fa(plog_A)}}};")
        w(f"static const double {tag}_plog_logA[{nterm}] = {{{fa(plog_logA)}}};")
        w(f"static const double {tag}_plog_b[{nterm}] = {{{fa(plog_b)}}};")
        w(f"static const double {tag}_plog_EaR[{nterm}] = {{{fa(plog_EaR)}}};")
        w(f"#endif /* {pfx}_H */")
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            f.write("\n".join(lines) + "\n")
        # sidecar with what host code needs without parsing C
        import json
        rx = []
        for r in self.reactions:
            net = r.net_stoich(n)
            rx.append({"type": r.rtype, "rev": int(r.reversible),
                       "nf": sum(v for _, v in r.reac), "np": sum(v for _, v in r.prod),
                       "tb": len(r.tb), "nrow": len(net),
                       "constk": int(r.b == 0.0 and r.EaR == 0.0), "T2": int(r.troe_has_T2)})
        side = {"name": self.name, "nsp": n, "nrxn": nr,
                "species": [s.name for s in self.species],
                "mw": [s.mw for s in self.species], "counts": self.counts(), "reactions": rx}
        with open(os.path.splitext(path)[0] + ".json", "w") as f:
            json.dump(side, f, indent=1)


# Directory holding the Cantera YAML inputs (the reference's
# ``resources/mechanisms``).  Only table generation reads it; the generated
# headers under ``csrc/mech`` are committed, so builds do not need it.
MECH_DIR_ENV = "HPC_ODE_MECH_DIR"


def load(name: str, mech_dir: Optional[str] = None) -> Mechanism:
    """Parse ``<mech_dir>/<name>.yaml``, or ``<name>.xml`` (CTML) when there is
    no YAML file (``gri30``, ``h2o2``, ``nDodecane_Reitz``, ``h2_li_2004``,
    ``ESTiMatE-Mech_04042022``)."""
    base = os.path.splitext(name)[0] if name.endswith((".yaml", ".xml")) else name
    mech_dir = mech_dir or os.environ.get(MECH_DIR_ENV)
    if not mech_dir:
        raise RuntimeError(f"set {MECH_DIR_ENV} to the directory holding {base}.yaml")
    yml = os.path.join(mech_dir, base + ".yaml")
    if os.path.exists(yml):
        return Mechanism.from_yaml(yml, base)
    return Mechanism.from_ctml(os.path.join(mech_dir, base + ".xml"), base)


def generate_all(mech_dir: Optional[str] = None, out_dir: Optional[str] = None) -> List[str]:
    out_dir = out_dir or os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "mech")
    paths = []
    for nm in ("gri30", "h2o2", "nDodecane_Reitz", "h2_li_2004", "ESTiMatE-Mech_04042022"):
        m = load(nm, mech_dir)
        p = os.path.join(out_dir, f"{nm}_mech.h")
        m.emit_header(p)
        paths.append(p)
    return paths


if __name__ == "__main__":
    import sys
    for p in generate_all(sys.argv[1] if len(sys.argv) > 1 else None):
        print("wrote", p)
