"""Mechanism table generation (hpc_ode_b200/mechanism.py), on the CPU.

Reads the reference's mechanism files where they lie (skipped when the
reference checkout is absent): the committed tables must be what the generator
produces, and the CTML (XML) reader must give the same mechanism as the YAML
reader for the mechanisms the reference ships in both forms."""
import os

import numpy as np
import pytest

from hpc_ode_b200 import mechanism as M
from hpc_ode_b200 import workloads as W

from oracle.refpath import reference_subdir  # noqa: E402

REF_MECH = reference_subdir("resources", "mechanisms") or ""
REF_DATA = reference_subdir("ref_data") or ""
needs_ref = pytest.mark.skipif(not os.path.isdir(REF_MECH), reason="reference mechanisms not present")


@needs_ref
@pytest.mark.parametrize("name", ["gri30", "h2o2", "nDodecane_Reitz", "h2_li_2004", "ESTiMatE-Mech_04042022"])
def test_committed_tables_are_generated(tmp_path, name):
    m = M.load(name, REF_MECH)
    out = tmp_path / f"{name}_mech.h"
    m.emit_header(str(out))
    committed = os.path.join(os.path.dirname(M.__file__), "csrc", "mech", f"{name}_mech.h")
    assert open(out).read() == open(committed).read()


@needs_ref
@pytest.mark.parametrize("name", ["gri30", "nDodecane_Reitz"])
def test_ctml_reader_matches_yaml_reader(name):
    a = M.Mechanism.from_yaml(os.path.join(REF_MECH, name + ".yaml"), name)
    b = M.Mechanism.from_ctml(os.path.join(REF_MECH, name + ".xml"), name)
    assert a.counts() == b.counts()
    assert [s.name for s in a.species] == [s.name for s in b.species]
    for sa, sb in zip(a.species, b.species):
        assert sa.tmid == sb.tmid and sa.lo == sb.lo and sa.hi == sb.hi
        assert abs(sa.mw - sb.mw) <= 1e-12 * sa.mw
    for ra, rb in zip(a.reactions, b.reactions):
        assert (ra.reac, ra.prod, ra.rtype, ra.reversible, ra.tb, ra.troe_has_T2) == \
               (rb.reac, rb.prod, rb.rtype, rb.reversible, rb.tb, rb.troe_has_T2), ra.equation
        for f in ("A", "b", "EaR", "A0", "b0", "EaR0"):
            x, y = getattr(ra, f), getattr(rb, f)
            assert abs(x - y) <= 1e-15 * max(abs(x), abs(y)), (ra.equation, f, x, y)


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_DATA, "res_h2.csv")), reason="reference data not present")
def test_h2_grid_workload_reproduces_reference_dataset():
    ref = np.genfromtxt(os.path.join(REF_DATA, "res_h2.csv"), delimiter=",", names=True)
    b = W.make("h2li_grid")
    assert b.ncells == ref.size == 10000
    assert np.array_equal(b.T, ref["TEMPE"])
    Y = np.stack([ref[f"CO{k}"] for k in range(9)])
    assert np.abs(b.Y - Y).max() <= 1e-15


def _ctml(tmp_path, rxn_type, rev, reac, prod):
    p = tmp_path / "m.xml"
    p.write_text(f"""<ctml><phase id="gas"><speciesArray>A B</speciesArray></phase>
<speciesData><species name="A"><atomArray>H:1</atomArray><thermo>
<NASA Tmin="300" Tmax="1000"><floatArray>1,0,0,0,0,0,0</floatArray></NASA>
<NASA Tmin="1000" Tmax="5000"><floatArray>1,0,0,0,0,0,0</floatArray></NASA></thermo></species>
<species name="B"><atomArray>H:2</atomArray><thermo>
<NASA Tmin="300" Tmax="1000"><floatArray>1,0,0,0,0,0,0</floatArray></NASA>
<NASA Tmin="1000" Tmax="5000"><floatArray>1,0,0,0,0,0,0</floatArray></NASA></thermo></species></speciesData>
<reactionData><reaction id="1" reversible="{rev}" type="{rxn_type}"><equation>x</equation><rateCoeff>
<Arrhenius><A>1</A><b>0</b><E units="K">0</E><P units="atm">1.0</P></Arrhenius></rateCoeff>
<reactants>{reac}</reactants><products>{prod}</products></reaction>
</reactionData></ctml>""")
    return str(p)


def test_unsupported_forms_raise(tmp_path):
    with pytest.raises(NotImplementedError):      # Chebyshev rate
        M.Mechanism.from_ctml(_ctml(tmp_path, "chebyshev", "yes", "A:2", "B:1"), "bad")
    with pytest.raises(NotImplementedError):      # fractional reactant coefficient
        M.Mechanism.from_ctml(_ctml(tmp_path, "elementary", "no", "A:1.5", "B:0.75"), "bad")
    with pytest.raises(NotImplementedError):      # fractional product of a reversible step
        M.Mechanism.from_ctml(_ctml(tmp_path, "elementary", "yes", "B:1", "A:0.5 B:0.75"), "bad")
    m = M.Mechanism.from_ctml(_ctml(tmp_path, "elementary", "no", "B:1", "A:1.5 B:0.25"), "ok")
    assert m.reactions[0].prod == [(0, 1.5), (1, 0.25)]
    out = tmp_path / "ok_mech.h"
    m.emit_header(str(out))
    assert "#define MECH_OK_NU_DEN 4" in open(out).read()


@needs_ref
def test_estimate_mechanism_forms():
    """ESTiMatE (kerosene, 214 species): PLOG levels sorted by pressure in Pa,
    lumped irreversible steps with fractional products, tables with NU_DEN 2."""
    m = M.load("ESTiMatE-Mech_04042022", REF_MECH)
    c = m.counts()
    assert (c["species"], c["reactions"], c["plog"], c["troe"], c["lindemann"]) == (214, 1558, 22, 71, 2)
    plog = [r for r in m.reactions if r.rtype == M.T_PLOG]
    assert all(r.reversible for r in plog)
    for r in plog:
        ps = [p for p, _ in r.plog]
        assert ps == sorted(ps) and len(set(ps)) == len(ps) and len(ps) >= 2
    first = plog[0]
    assert first.equation.startswith("CH3 + OH") and first.plog[0][0] == pytest.approx(0.01 * 101325.0)
    frac = [r for r in m.reactions if any(v != int(v) for _, v in r.prod)]
    assert len(frac) == 5 and not any(r.reversible for r in frac)


def test_device_table_packing(tmp_path):
    """The device-table packer (csrc/mech_dev.h, compiled with g++ here) accepts
    every compiled mechanism; its gather-unit count equals the generated
    NUNITS the kernels size their shared scratch by, its gather words
    reproduce each net stoichiometric coefficient (fractional ones included),
    PLOG slots and inert species agree with the tables, and every index the
    kernels read from the tables (factor species, third-body lists, catalysts,
    Jacobian rows, gather slots and units, PLOG levels and terms) lies inside
    the array it indexes."""
    import subprocess
    here = os.path.dirname(os.path.abspath(__file__))
    exe = tmp_path / "pack_check"
    subprocess.run(["g++", "-O1", "-std=c++17", "-o", str(exe), os.path.join(here, "cpp", "pack_check.cpp")],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout
    lines = out.stdout.strip().splitlines()
    assert len(lines) == 5 and all(l.startswith("ok ") and "indices in range" in l for l in lines)
    est = [l for l in lines if "estimate" in l][0]
    assert "plog 22" in est and "nu_den 2" in est
