"""ctypes bindings for the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
legs import this module, to check results.  It loads ``oracle/liboracle.so``
(restated chemistry + CVODE-semantics BDF, built by ``oracle/Makefile``) and,
when present, ``oracle/_ref/libpyjac_gri30.so`` (the reference's own pyJac C
kernels compiled from their sources; ``src/Mechanism/CPU``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libpyjac_gri30.so")

_dptr = C.POINTER(C.c_double)
RHS_FN = C.CFUNCTYPE(None, C.c_double, C.c_double, _dptr, _dptr)


class BdfOpts(C.Structure):
    _fields_ = [("rtol", C.c_double), ("atol", C.c_double),
                ("max_steps", C.c_int), ("max_order", C.c_int)]


class BdfStats(C.Structure):
    _fields_ = [("status", C.c_int), ("nst", C.c_int), ("nfe", C.c_int), ("nje", C.c_int),
                ("nsetups", C.c_int), ("nni", C.c_int), ("ncfn", C.c_int), ("netf", C.c_int),
                ("qlast", C.c_int), ("hlast", C.c_double)]


STATS_FIELDS = [f for f, _ in BdfStats._fields_]
STATS_DTYPE = np.dtype([("status", "i4"), ("nst", "i4"), ("nfe", "i4"), ("nje", "i4"),
                        ("nsetups", "i4"), ("nni", "i4"), ("ncfn", "i4"), ("netf", "i4"),
                        ("qlast", "i4"), ("pad", "i4"), ("hlast", "f8")])
assert STATS_DTYPE.itemsize == C.sizeof(BdfStats)

MECH_IDS = {"gri30": 0, "h2o2": 1, "nDodecane_Reitz": 2, "h2_li_2004": 3, "ESTiMatE-Mech_04042022": 4}


def build(force: bool = False) -> None:
    """Compile liboracle.so (and the reference pyJac .so when its sources exist)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE], check=True)


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dptr)


class Oracle:
    def __init__(self, lib_path: str = LIB_PATH):
        if not os.path.exists(lib_path):
            build()
        self.lib = C.CDLL(lib_path)
        L = self.lib
        L.oracle_mech_nsp.restype = C.c_int
        L.oracle_mech_nsp.argtypes = [C.c_int]
        for nm in ("oracle_dydt", "oracle_jacob", "oracle_dydt_scale", "oracle_dydt_conv",
                   "oracle_jacob_conv", "oracle_dydt_scale_conv"):
            getattr(L, nm).argtypes = [C.c_int, C.c_double, _dptr, _dptr]
            getattr(L, nm).restype = None
        L.oracle_density.argtypes = [C.c_int, C.c_double, _dptr]
        L.oracle_density.restype = C.c_double
        L.oracle_kf.argtypes = [C.c_int, C.c_double, C.c_double, _dptr]
        L.oracle_kf.restype = None
        L.oracle_bdf_batch_mech.restype = C.c_long
        L.oracle_bdf_batch_mech.argtypes = [C.c_int, C.c_long, _dptr, C.c_double, _dptr, C.c_double,
                                            C.c_double, C.POINTER(BdfOpts), C.c_void_p, C.c_int]
        L.oracle_bdf_batch_mech_conv.restype = C.c_long
        L.oracle_bdf_batch_mech_conv.argtypes = L.oracle_bdf_batch_mech.argtypes
        L.oracle_bdf_batch.restype = C.c_long
        L.oracle_bdf_batch.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_long, _dptr, C.c_double,
                                       _dptr, C.c_double, C.c_double, C.POINTER(BdfOpts),
                                       C.c_void_p, C.c_int]
        self.ref = C.CDLL(REF_PATH) if os.path.exists(REF_PATH) else None

    # ------------------------------------------------------------ chemistry
    def nsp(self, mech: str) -> int:
        return self.lib.oracle_mech_nsp(MECH_IDS[mech])

    def dydt(self, mech: str, pres: float, y: np.ndarray) -> np.ndarray:
        y = np.ascontiguousarray(y, dtype=np.float64)
        out = np.zeros_like(y)
        self.lib.oracle_dydt(MECH_IDS[mech], float(pres), _p(y), _p(out))
        return out

    def dydt_scale(self, mech: str, pres: float, y: np.ndarray) -> np.ndarray:
        y = np.ascontiguousarray(y, dtype=np.float64)
        out = np.zeros_like(y)
        self.lib.oracle_dydt_scale(MECH_IDS[mech], float(pres), _p(y), _p(out))
        return out

    # constant-volume forms: rho is the cell's fixed density
    def dydt_conv(self, mech: str, rho: float, y: np.ndarray) -> np.ndarray:
        y = np.ascontiguousarray(y, dtype=np.float64)
        out = np.zeros_like(y)
        self.lib.oracle_dydt_conv(MECH_IDS[mech], float(rho), _p(y), _p(out))
        return out

    def dydt_scale_conv(self, mech: str, rho: float, y: np.ndarray) -> np.ndarray:
        y = np.ascontiguousarray(y, dtype=np.float64)
        out = np.zeros_like(y)
        self.lib.oracle_dydt_scale_conv(MECH_IDS[mech], float(rho), _p(y), _p(out))
        return out

    def jacob_conv(self, mech: str, rho: float, y: np.ndarray) -> np.ndarray:
        y = np.ascontiguousarray(y, dtype=np.float64)
        n = y.size
        out = np.zeros(n * n)
        self.lib.oracle_jacob_conv(MECH_IDS[mech], float(rho), _p(y), _p(out))
        return out.reshape(n, n).T.copy()

    def density(self, mech: str, pres: float, y: np.ndarray) -> float:
        y = np.ascontiguousarray(y, dtype=np.float64)
        return float(self.lib.oracle_density(MECH_IDS[mech], float(pres), _p(y)))

    def kf(self, mech: str, pres: float, T: float, nrxn: int) -> np.ndarray:
        """Forward rate coefficient of every reaction at (T, P)."""
        out = np.zeros(nrxn)
        self.lib.oracle_kf(MECH_IDS[mech], float(pres), float(T), _p(out))
        return out

    def jacob(self, mech: str, pres: float, y: np.ndarray) -> np.ndarray:
        """Column-major n x n as a numpy array J[i, j] = d f_i / d y_j."""
        y = np.ascontiguousarray(y, dtype=np.float64)
        n = y.size
        out = np.zeros(n * n)
        self.lib.oracle_jacob(MECH_IDS[mech], float(pres), _p(y), _p(out))
        return out.reshape(n, n).T.copy()

    # ------------------------------------------------- reference pyJac (GRI)
    def has_ref(self) -> bool:
        return self.ref is not None

    def ref_dydt(self, pres: float, y: np.ndarray) -> np.ndarray:
        y = np.ascontiguousarray(y, dtype=np.float64)
        out = np.zeros_like(y)
        self.ref.dydt(C.c_double(0.0), C.c_double(pres), _p(y), _p(out))
        return out

    def ref_jacob(self, pres: float, y: np.ndarray) -> np.ndarray:
        y = np.ascontiguousarray(y, dtype=np.float64)
        n = y.size
        out = np.zeros(n * n)
        self.ref.eval_jacob(C.c_double(0.0), C.c_double(pres), _p(y), _p(out))
        return out.reshape(n, n).T.copy()

    # ------------------------------------------------------------------ BDF
    def bdf(self, mech: str, y: np.ndarray, pres, t1: float, rtol: float = 1e-6,
            atol: float = 1e-10, max_steps: int = 10000, threads: int = 1,
            use_ref_kernels: bool = False, max_order: int = 5, conv: bool = False):
        """Integrate cell-major states y[ncells, n] from 0 to t1 in place-copy.
        conv: constant volume (pres = each cell's initial pressure).

        Returns (y_out, stats structured array)."""
        y = np.array(y, dtype=np.float64, order="C", copy=True)
        if y.ndim == 1:
            y = y[None, :]
        ncells, n = y.shape
        opts = BdfOpts(rtol, atol, max_steps, max_order)
        stats = np.zeros(ncells, dtype=STATS_DTYPE)
        if np.ndim(pres) == 0:
            parr = None
            pscal = float(pres)
        else:
            parr = np.ascontiguousarray(pres, dtype=np.float64)
            pscal = 0.0
        pp = _p(parr) if parr is not None else C.cast(None, _dptr)
        if use_ref_kernels:
            if mech != "gri30" or self.ref is None:
                raise RuntimeError("reference pyJac kernels are only available for gri30")
            f = C.cast(self.ref.dydt, C.c_void_p)
            J = C.cast(self.ref.eval_jacob, C.c_void_p)
            self.lib.oracle_bdf_batch(f, J, n, ncells, pp, pscal, _p(y), 0.0, float(t1),
                                      C.byref(opts), stats.ctypes.data_as(C.c_void_p), threads)
        else:
            fn = self.lib.oracle_bdf_batch_mech_conv if conv else self.lib.oracle_bdf_batch_mech
            fn(MECH_IDS[mech], ncells, pp, pscal, _p(y), 0.0, float(t1), C.byref(opts),
               stats.ctypes.data_as(C.c_void_p), threads)
        return y, stats


_ORACLE: Optional[Oracle] = None


def get() -> Oracle:
    global _ORACLE
    if _ORACLE is None:
        _ORACLE = Oracle()
    return _ORACLE
