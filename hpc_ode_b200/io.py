"""ctypes binding of include/b200ode_io.h (libb200ode_host.so): the parallel
reader/writer for the reference's cell CSV files, into and out of
structure-of-arrays numpy buffers (T[n], Y[nsp, n], ENTHA[n], XYZ[3, n])."""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
HOST_LIB_PATH = os.path.join(PKG, "libb200ode_host.so")
_dp = C.POINTER(C.c_double)
_lib: Optional[C.CDLL] = None


class CsvInfo(C.Structure):
    _fields_ = [("n_cells", C.c_int64), ("n_species", C.c_int32), ("has_enthalpy", C.c_int32),
                ("has_coordinates", C.c_int32)]


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(HOST_LIB_PATH):
            raise RuntimeError(f"{HOST_LIB_PATH} is missing: build it with `python -m hpc_ode_b200.build`")
        lib = C.CDLL(HOST_LIB_PATH)
        lib.b200ode_csv_inspect.argtypes = [C.c_char_p, C.POINTER(CsvInfo)]
        lib.b200ode_csv_read.argtypes = [C.c_char_p, C.c_int32, _dp, _dp, _dp, _dp]
        lib.b200ode_csv_write.argtypes = [C.c_char_p, C.c_int64, C.c_int32, _dp, _dp, _dp, _dp, C.c_int32]
        lib.b200ode_io_last_error.restype = C.c_char_p
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(_dp) if a is not None else C.cast(None, _dp)


def _check(rc: int):
    if rc != 0:
        raise ValueError(load().b200ode_io_last_error().decode())


def read_csv(path: str, threads: int = 0) -> dict:
    """Cells of a CSV file: {'T': [n], 'Y': [nsp, n], 'ENTHA': [n] or None, 'XYZ': [3, n] or None}."""
    lib = load()
    info = CsvInfo()
    _check(lib.b200ode_csv_inspect(path.encode(), C.byref(info)))
    n, nsp = info.n_cells, info.n_species
    T = np.empty(n)
    Y = np.empty((nsp, n))
    H = np.empty(n) if info.has_enthalpy else None
    X = np.empty((3, n)) if info.has_coordinates else None
    _check(lib.b200ode_csv_read(path.encode(), int(threads), _p(T), _p(Y), _p(H), _p(X)))
    return {"T": T, "Y": Y, "ENTHA": H, "XYZ": X}


def write_csv(path: str, T: np.ndarray, Y: np.ndarray, enthalpy: Optional[np.ndarray] = None,
              xyz: Optional[np.ndarray] = None, threads: int = 0) -> None:
    """Write cells (T[n], Y[nsp, n], optional ENTHA[n], XYZ[3, n]) in the reference's column order."""
    T = np.ascontiguousarray(T, dtype=np.float64)
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    H = None if enthalpy is None else np.ascontiguousarray(enthalpy, dtype=np.float64)
    X = None if xyz is None else np.ascontiguousarray(xyz, dtype=np.float64)
    _check(load().b200ode_csv_write(path.encode(), T.size, Y.shape[0], _p(T), _p(Y), _p(H), _p(X), int(threads)))
