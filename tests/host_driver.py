"""Builds and runs tests/cpp/integrator_driver.cpp (the C++ host integrator
through the restated reference interface) for the host-integrator tests."""
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
PKG = os.path.join(ROOT, "hpc_ode_b200")


def build(tmpdir) -> str:
    from hpc_ode_b200 import build as b
    b.build()
    exe = os.path.join(str(tmpdir), "integrator_driver")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-o", exe,
                    os.path.join(HERE, "cpp", "integrator_driver.cpp"), "-L", PKG, "-lb200ode_host",
                    "-lb200ode", f"-Wl,-rpath,{PKG}"], check=True)
    return exe


def run(exe, tmpdir, itype, mech, T, Y_rows, dt, P, options=()):
    """T[n], Y_rows[n, nsp] (cell-major, as the reference's Mesh). Returns
    (returncode, stdout, T_out, Y_out, status) with outputs None on failure."""
    n, nsp = Y_rows.shape
    fin = os.path.join(str(tmpdir), "in.bin")
    fout = os.path.join(str(tmpdir), "out.bin")
    with open(fin, "wb") as f:
        f.write(np.array([n, nsp], dtype=np.int32).tobytes())
        f.write(np.array([dt, P], dtype=np.float64).tobytes())
        f.write(np.ascontiguousarray(T, dtype=np.float64).tobytes())
        f.write(np.ascontiguousarray(Y_rows, dtype=np.float64).tobytes())
    r = subprocess.run([exe, itype, mech, fin, fout, *options], capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        return r.returncode, r.stdout, None, None, None
    raw = open(fout, "rb").read()
    off = 24
    To = np.frombuffer(raw, np.float64, n, off); off += 8 * n
    Yo = np.frombuffer(raw, np.float64, n * nsp, off).reshape(n, nsp); off += 8 * n * nsp
    st = np.frombuffer(raw, np.int32, n, off); off += 4 * n
    run.enthalpy = np.frombuffer(raw, np.float64, n, off).copy()
    return 0, r.stdout, To.copy(), Yo.copy(), st.copy()
