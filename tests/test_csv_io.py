"""The parallel cell-CSV reader/writer (include/b200ode_io.h), on the CPU:
exact round trips, thread-count independence, the reference's own data files
read the same as numpy reads them, and malformed input reported by line."""
import os
import time

import numpy as np
import pytest

from hpc_ode_b200 import build, io
from oracle.refpath import reference_subdir

REF_DATA = reference_subdir("ref_data") or ""


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


@pytest.mark.parametrize("with_h,with_xyz", [(False, False), (True, False), (True, True)])
def test_round_trip_is_exact(tmp_path, with_h, with_xyz):
    rng = np.random.default_rng(3)
    n, nsp = 1001, 53
    T = rng.uniform(300, 2500, n)
    Y = rng.dirichlet(np.ones(nsp), n).T * rng.choice([1.0, 1e-30, 1e-300], (nsp, n))
    H = rng.normal(0, 1e6, n) if with_h else None
    X = rng.normal(0, 1, (3, n)) if with_xyz else None
    p = str(tmp_path / "cells.csv")
    io.write_csv(p, T, Y, H, X, threads=4)
    d = io.read_csv(p, threads=3)
    assert np.array_equal(d["T"], T) and np.array_equal(d["Y"], Y)
    assert (d["ENTHA"] is None) == (H is None) and (H is None or np.array_equal(d["ENTHA"], H))
    assert (d["XYZ"] is None) == (X is None) and (X is None or np.array_equal(d["XYZ"], X))
    p1 = str(tmp_path / "one.csv")
    io.write_csv(p1, T, Y, H, X, threads=1)
    assert open(p, "rb").read() == open(p1, "rb").read()


@pytest.mark.skipif(not os.path.isdir(REF_DATA), reason="reference data not present")
@pytest.mark.parametrize("name,nsp,fmt", [("res_h2.csv", 9, "CO{}"), ("res_gri_100.csv", 53, "CO{:03d}")])
def test_reads_reference_files_like_numpy(name, nsp, fmt):
    path = os.path.join(REF_DATA, name)
    d = io.read_csv(path, threads=8)
    ref = np.genfromtxt(path, delimiter=",", names=True)
    start = 0 if fmt == "CO{}" else 1
    Y = np.stack([ref[fmt.format(k + start)] for k in range(nsp)])
    assert np.array_equal(d["T"], ref["TEMPE"]) and np.array_equal(d["Y"], Y)
    assert np.array_equal(d["ENTHA"], ref["ENTHA"])
    if d["XYZ"] is not None:
        assert np.array_equal(d["XYZ"][0], ref["Points0"])


def test_malformed_lines_are_reported(tmp_path):
    p = tmp_path / "bad.csv"
    p.write_text("CO0,CO1,TEMPE\n0.5,0.5,300\n0.5,abc,300\n")
    with pytest.raises(ValueError, match="line 3"):
        io.read_csv(str(p))
    p.write_text("CO0,CO1,TEMPE\n0.5,0.5\n")
    with pytest.raises(ValueError, match="expected 3"):
        io.read_csv(str(p))
    p.write_text("CO0,CO1\n0.5,0.5\n")
    with pytest.raises(ValueError, match="TEMPE"):
        io.read_csv(str(p))


def test_large_file_throughput(tmp_path):
    n, nsp = 1 << 18, 53
    rng = np.random.default_rng(1)
    T = rng.uniform(300, 2500, n)
    Y = rng.random((nsp, n))
    p = str(tmp_path / "big.csv")
    t0 = time.perf_counter()
    io.write_csv(p, T, Y)
    t1 = time.perf_counter()
    d = io.read_csv(p)
    t2 = time.perf_counter()
    assert np.array_equal(d["T"], T) and np.array_equal(d["Y"], Y)
    mb = os.path.getsize(p) / 1e6
    print(f"\n{n} GRI cells, {mb:.0f} MB: write {t1 - t0:.2f} s, read {t2 - t1:.2f} s")
