"""ctypes binding of the C ABI in ``include/b200ode.h``.

Loading fails loudly (``NativeLibraryError``) when ``libb200ode.so`` is absent:
there is no CPU fallback on the product path.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libb200ode.so")

B200ODE_OK = 0
B200ODE_FP64 = 0
B200ODE_MIXED = 1
B200ODE_CONP = 0
B200ODE_CONV = 1
STATUS_NAMES = {0: "OK", 1: "ERR_INVALID", 2: "ERR_MECHANISM", 3: "ERR_CUDA", 4: "ERR_ALLOC",
                5: "ERR_NO_DEVICE", 6: "ERR_BUSY", 7: "ERR_NOT_READY"}
CELL_STATUS = {0: "CV_SUCCESS", -1: "CV_TOO_MUCH_WORK", -2: "CV_TOO_MUCH_ACC", -22: "CV_ILL_INPUT",
               -3: "CV_ERR_FAILURE", -4: "CV_CONV_FAILURE", -27: "CV_TOO_CLOSE"}

# Every symbol include/b200ode.h declares.
EXPORTED = ["b200ode_default_options", "b200ode_create", "b200ode_destroy", "b200ode_num_species",
            "b200ode_mechanism_species",
            "b200ode_integrate", "b200ode_integrate_device", "b200ode_integrate_device_noalloc",
            "b200ode_eval_rhs",
            "b200ode_eval_jacobian", "b200ode_eval_enthalpy", "b200ode_eval_enthalpy_device",
            "b200ode_autotune", "b200ode_get_options", "b200ode_fp64_peak", "b200ode_fp32_peak",
            "b200ode_default_server_options", "b200ode_server_create", "b200ode_server_destroy",
            "b200ode_submit", "b200ode_poll", "b200ode_server_get_report",
            "b200ode_last_error", "b200ode_version"]


class NativeLibraryError(RuntimeError):
    pass


class B200Error(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class Options(C.Structure):
    _fields_ = [("reltol", C.c_double), ("abstol", C.c_double), ("max_steps", C.c_int32),
                ("max_order", C.c_int32), ("precision", C.c_int32), ("refine", C.c_int32),
                ("persistent", C.c_int32), ("warps_per_block", C.c_int32),
                ("blocks_per_sm", C.c_int32), ("queue_chunk", C.c_int32),
                ("use_graph", C.c_int32), ("device", C.c_int32), ("profile_phases", C.c_int32),
                ("formulation", C.c_int32), ("cta_helpers", C.c_int32),
                ("helper_join_cycles", C.c_int64), ("helper_drain_cycles", C.c_int64),
                ("helper_idle_cycles", C.c_int64), ("max_cells_per_launch", C.c_int64)]


_i32p = C.POINTER(C.c_int32)


class Stats(C.Structure):
    _fields_ = [("nst", _i32p), ("nfe", _i32p), ("nje", _i32p), ("nsetups", _i32p),
                ("nni", _i32p), ("ncfn", _i32p), ("netf", _i32p),
                ("total_nst", C.c_int64), ("total_nfe", C.c_int64), ("total_nje", C.c_int64),
                ("total_nsetups", C.c_int64), ("total_nni", C.c_int64),
                ("total_ncfn", C.c_int64), ("total_netf", C.c_int64), ("n_failed", C.c_int64),
                ("h2d_ms", C.c_double), ("kernel_ms", C.c_double), ("d2h_ms", C.c_double),
                ("gpu_launches", C.c_int32), ("phase_cycles", C.c_int64 * 5)]


class ServerOptions(C.Structure):
    _fields_ = [("solver", Options), ("hbm_budget_bytes", C.c_int64), ("max_inflight", C.c_int32),
                ("max_queued", C.c_int32), ("chunk_cells", C.c_int32)]


class RequestInfo(C.Structure):
    _fields_ = [("n_cells", C.c_int64), ("n_failed", C.c_int64), ("total_nst", C.c_int64),
                ("total_nni", C.c_int64), ("footprint_bytes", C.c_int64), ("queue_ms", C.c_double),
                ("device_ms", C.c_double), ("latency_ms", C.c_double)]


class ServerReport(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed_requests", C.c_int64),
                ("cells_completed", C.c_int64), ("p50_latency_ms", C.c_double),
                ("p99_latency_ms", C.c_double), ("max_latency_ms", C.c_double),
                ("mean_queue_ms", C.c_double), ("cells_per_sec", C.c_double),
                ("max_concurrent", C.c_int32), ("budget_bytes", C.c_int64), ("peak_bytes", C.c_int64)]


COUNTERS = ["nst", "nfe", "nje", "nsetups", "nni", "ncfn", "netf"]
_dp = C.POINTER(C.c_double)
_lib: Optional[C.CDLL] = None


def load(path: str = LIB_PATH) -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise NativeLibraryError(
            f"{path} is missing: build it with `python -m hpc_ode_b200.build` (nvcc, sm_100a)")
    lib = C.CDLL(path)
    lib.b200ode_default_options.argtypes = [C.POINTER(Options)]
    lib.b200ode_default_options.restype = None
    lib.b200ode_create.argtypes = [C.c_char_p, C.POINTER(Options), C.POINTER(C.c_void_p)]
    lib.b200ode_create.restype = C.c_int
    lib.b200ode_destroy.argtypes = [C.c_void_p]
    lib.b200ode_destroy.restype = None
    lib.b200ode_num_species.argtypes = [C.c_void_p]
    lib.b200ode_num_species.restype = C.c_int32
    lib.b200ode_mechanism_species.argtypes = [C.c_char_p]
    lib.b200ode_mechanism_species.restype = C.c_int32
    lib.b200ode_integrate.argtypes = [C.c_void_p, C.c_int64, _dp, C.c_double, _dp, _dp, C.c_double,
                                      C.c_double, _i32p, C.POINTER(Stats)]
    lib.b200ode_integrate.restype = C.c_int
    lib.b200ode_integrate_device.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_double,
                                             C.c_void_p, C.c_void_p, C.c_double, C.c_double,
                                             C.c_void_p, C.POINTER(Stats), C.c_void_p]
    lib.b200ode_integrate_device.restype = C.c_int
    lib.b200ode_integrate_device_noalloc.argtypes = lib.b200ode_integrate_device.argtypes
    lib.b200ode_integrate_device_noalloc.restype = C.c_int
    lib.b200ode_eval_rhs.argtypes = [C.c_void_p, C.c_int64, _dp, C.c_double, _dp, _dp, _dp, _dp]
    lib.b200ode_eval_rhs.restype = C.c_int
    lib.b200ode_eval_jacobian.argtypes = [C.c_void_p, C.c_int64, _dp, C.c_double, _dp, _dp, _dp]
    lib.b200ode_eval_jacobian.restype = C.c_int
    lib.b200ode_eval_enthalpy.argtypes = [C.c_void_p, C.c_int64, _dp, _dp, _dp]
    lib.b200ode_eval_enthalpy.restype = C.c_int
    lib.b200ode_eval_enthalpy_device.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                                 C.c_void_p]
    lib.b200ode_eval_enthalpy_device.restype = C.c_int
    lib.b200ode_autotune.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p,
                                     C.c_double, C.c_double, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    lib.b200ode_autotune.restype = C.c_int
    lib.b200ode_fp64_peak.argtypes = [C.c_int32, C.POINTER(C.c_double)]
    lib.b200ode_fp64_peak.restype = C.c_int
    lib.b200ode_fp32_peak.argtypes = [C.c_int32, C.POINTER(C.c_double)]
    lib.b200ode_fp32_peak.restype = C.c_int
    lib.b200ode_get_options.argtypes = [C.c_void_p, C.POINTER(Options)]
    lib.b200ode_get_options.restype = C.c_int
    lib.b200ode_default_server_options.argtypes = [C.POINTER(ServerOptions)]
    lib.b200ode_default_server_options.restype = None
    lib.b200ode_server_create.argtypes = [C.POINTER(ServerOptions), C.POINTER(C.c_void_p)]
    lib.b200ode_server_create.restype = C.c_int
    lib.b200ode_server_destroy.argtypes = [C.c_void_p]
    lib.b200ode_server_destroy.restype = None
    lib.b200ode_submit.argtypes = [C.c_void_p, C.c_char_p, C.c_int64, _dp, C.c_double, _dp, _dp,
                                   C.c_double, C.c_double, _i32p, C.POINTER(C.c_uint64)]
    lib.b200ode_submit.restype = C.c_int
    lib.b200ode_poll.argtypes = [C.c_void_p, C.c_uint64, C.c_int32, C.POINTER(RequestInfo)]
    lib.b200ode_poll.restype = C.c_int
    lib.b200ode_server_get_report.argtypes = [C.c_void_p, C.POINTER(ServerReport)]
    lib.b200ode_server_get_report.restype = C.c_int
    lib.b200ode_last_error.argtypes = []
    lib.b200ode_last_error.restype = C.c_char_p
    lib.b200ode_version.argtypes = []
    lib.b200ode_version.restype = C.c_char_p
    _lib = lib
    return lib


def default_options(**kw) -> Options:
    o = Options()
    load().b200ode_default_options(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


def last_error() -> str:
    return load().b200ode_last_error().decode()


def _check(rc: int):
    if rc != B200ODE_OK:
        raise B200Error(rc, last_error())


def _ptr(a: Optional[np.ndarray]):
    return a.ctypes.data_as(_dp) if a is not None else C.cast(None, _dp)


class Solver:
    """One handle of the C ABI (one mechanism, one set of options)."""

    def __init__(self, mech: str, opts: Optional[Options] = None, **kw):
        self.lib = load()
        self.opts = opts if opts is not None else default_options(**kw)
        h = C.c_void_p()
        _check(self.lib.b200ode_create(mech.encode(), C.byref(self.opts), C.byref(h)))
        self.h = h
        self.nsp = self.lib.b200ode_num_species(h)
        self.last_stats: Optional[Stats] = None

    def close(self):
        if getattr(self, "h", None):
            self.lib.b200ode_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def integrate(self, T: np.ndarray, Y: np.ndarray, P, t1: float, t0: float = 0.0,
                  counters: bool = False):
        """Host-buffer integration.  T[n], Y[nsp, n] (SoA) are updated in place.

        Returns (status[n], stats dict, per-cell counters dict or None)."""
        n = T.size
        assert T.dtype == np.float64 and T.flags.c_contiguous
        assert Y.dtype == np.float64 and Y.flags.c_contiguous and Y.shape == (self.nsp, n)
        if np.ndim(P) == 0:
            parr, ps = None, float(P)
        else:
            parr, ps = np.ascontiguousarray(P, dtype=np.float64), 0.0
        status = np.zeros(n, dtype=np.int32)
        st = Stats()
        cnt = None
        if counters:
            cnt = {k: np.zeros(n, dtype=np.int32) for k in COUNTERS}
            for k in COUNTERS:
                setattr(st, k, cnt[k].ctypes.data_as(_i32p))
        _check(self.lib.b200ode_integrate(self.h, n, _ptr(parr), ps, _ptr(T), _ptr(Y), float(t0),
                                          float(t1), status.ctypes.data_as(_i32p), C.byref(st)))
        self.last_stats = st
        return status, stats_dict(st), cnt

    def eval_rhs(self, T: np.ndarray, Y: np.ndarray, P):
        """dy/dt for cells (T[n], Y[nsp, n]); returns (dTdt[n], dYdt[nsp-1, n])."""
        n = T.size
        T = np.ascontiguousarray(T, dtype=np.float64)
        Y = np.ascontiguousarray(Y, dtype=np.float64)
        parr, ps = (None, float(P)) if np.ndim(P) == 0 else (np.ascontiguousarray(P, dtype=np.float64), 0.0)
        dT = np.zeros(n)
        dY = np.zeros((self.nsp - 1, n))
        _check(self.lib.b200ode_eval_rhs(self.h, n, _ptr(parr), ps, _ptr(T), _ptr(Y), _ptr(dT), _ptr(dY)))
        return dT, dY

    def eval_enthalpy(self, T: np.ndarray, Y: np.ndarray) -> np.ndarray:
        """Mixture specific enthalpy [J/kg] of cells (T[n], Y[nsp, n])."""
        n = T.size
        T = np.ascontiguousarray(T, dtype=np.float64)
        Y = np.ascontiguousarray(Y, dtype=np.float64)
        out = np.zeros(n)
        _check(self.lib.b200ode_eval_enthalpy(self.h, n, _ptr(T), _ptr(Y), _ptr(out)))
        return out

    def eval_jacobian(self, T: np.ndarray, Y: np.ndarray, P) -> np.ndarray:
        """Analytic Jacobians [n, nsp, nsp] with J[c, i, j] = d f_i / d y_j (reference order)."""
        n = T.size
        T = np.ascontiguousarray(T, dtype=np.float64)
        Y = np.ascontiguousarray(Y, dtype=np.float64)
        parr, ps = (None, float(P)) if np.ndim(P) == 0 else (np.ascontiguousarray(P, dtype=np.float64), 0.0)
        out = np.zeros(n * self.nsp * self.nsp)
        _check(self.lib.b200ode_eval_jacobian(self.h, n, _ptr(parr), ps, _ptr(T), _ptr(Y), _ptr(out)))
        return out.reshape(n, self.nsp, self.nsp).transpose(0, 2, 1).copy()

    def integrate_device(self, n: int, dP: int, P_scalar: float, dT: int, dY: int, t1: float,
                         t0: float = 0.0, dstatus: int = 0, stream: int = 0, want_stats=True):
        """Device-pointer integration (pointers as ints, e.g. torch tensor.data_ptr())."""
        st = Stats() if want_stats else None
        _check(self.lib.b200ode_integrate_device(
            self.h, n, C.c_void_p(dP or None), float(P_scalar), C.c_void_p(dT), C.c_void_p(dY),
            float(t0), float(t1), C.c_void_p(dstatus or None),
            C.byref(st) if st is not None else None, C.c_void_p(stream or None)))
        self.last_stats = st
        return stats_dict(st) if st is not None else None

    def autotune(self, n: int, dP: int, P_scalar: float, dT: int, dY: int, t1: float, t0: float = 0.0):
        """Pick the fastest launch shape on a sample of these device-resident
        cells (left unmodified); later calls on this solver use it.  Returns
        (warps per CTA, blocks-per-SM setting)."""
        w, b = C.c_int32(), C.c_int32()
        _check(self.lib.b200ode_autotune(self.h, n, C.c_void_p(dP or None), float(P_scalar), C.c_void_p(dT),
                                         C.c_void_p(dY), float(t0), float(t1), C.byref(w), C.byref(b)))
        self.opts = self.options()
        return w.value, b.value

    def options(self) -> Options:
        """The options the handle uses now (defaults resolved, autotuned choices)."""
        o = Options()
        _check(self.lib.b200ode_get_options(self.h, C.byref(o)))
        return o

    def integrate_device_noalloc(self, n: int, dP: int, P_scalar: float, dT: int, dY: int, t1: float,
                                 t0: float = 0.0, dstatus: int = 0, stream: int = 0, want_stats=True):
        """As integrate_device, through the entry point that allocates no device
        memory (its scratch is one static array per device, shared by every call)."""
        st = Stats() if want_stats else None
        _check(self.lib.b200ode_integrate_device_noalloc(
            self.h, n, C.c_void_p(dP or None), float(P_scalar), C.c_void_p(dT), C.c_void_p(dY),
            float(t0), float(t1), C.c_void_p(dstatus or None),
            C.byref(st) if st is not None else None, C.c_void_p(stream or None)))
        self.last_stats = st
        return stats_dict(st) if st is not None else None


B200ODE_ERR_NOT_READY = 7


class Server:
    """The request loop of the C ABI (b200ode_server_*): submit batches of cells,
    poll for their results; continuous batching on one GPU."""

    def __init__(self, hbm_budget_bytes: int = 0, max_inflight: int = 4, max_queued: int = 4096,
                 chunk_cells: int = 32768, **solver_kw):
        self.lib = load()
        o = ServerOptions()
        self.lib.b200ode_default_server_options(C.byref(o))
        for k, v in solver_kw.items():
            if not hasattr(o.solver, k):
                raise KeyError(k)
            setattr(o.solver, k, v)
        o.hbm_budget_bytes = int(hbm_budget_bytes)
        o.max_inflight = int(max_inflight)
        o.max_queued = int(max_queued)
        o.chunk_cells = int(chunk_cells)
        h = C.c_void_p()
        _check(self.lib.b200ode_server_create(C.byref(o), C.byref(h)))
        self.h = h
        self._live = {}   # request id -> buffers the library writes into

    def submit(self, mech: str, T: np.ndarray, Y: np.ndarray, P, t1: float, t0: float = 0.0) -> int:
        """Queue cells (T[n], Y[nsp, n] SoA, updated in place when done)."""
        n = T.size
        assert T.dtype == np.float64 and T.flags.c_contiguous
        assert Y.dtype == np.float64 and Y.flags.c_contiguous and Y.shape[1] == n
        parr, ps = (None, float(P)) if np.ndim(P) == 0 else (np.ascontiguousarray(P, dtype=np.float64), 0.0)
        status = np.full(n, 99, dtype=np.int32)
        rid = C.c_uint64()
        _check(self.lib.b200ode_submit(self.h, mech.encode(), n, _ptr(parr), ps, _ptr(T), _ptr(Y), float(t0),
                                       float(t1), status.ctypes.data_as(_i32p), C.byref(rid)))
        self._live[rid.value] = (T, Y, parr, status)
        return rid.value

    def poll(self, rid: int, wait_ms: int = -1):
        """(status[n], info dict) when done, None if still in flight after wait_ms."""
        info = RequestInfo()
        rc = self.lib.b200ode_poll(self.h, rid, int(wait_ms), C.byref(info))
        if rc == B200ODE_ERR_NOT_READY:
            return None
        bufs = self._live.pop(rid, None)
        _check(rc)
        return bufs[3], {f: getattr(info, f) for f, _ in RequestInfo._fields_}

    def report(self) -> dict:
        r = ServerReport()
        _check(self.lib.b200ode_server_get_report(self.h, C.byref(r)))
        return {f: getattr(r, f) for f, _ in ServerReport._fields_}

    def close(self):
        if getattr(self, "h", None):
            self.lib.b200ode_server_destroy(self.h)
            self.h = None
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fp64_peak_gflops(device: int = -1) -> float:
    """Measured FP64 FMA throughput of the device (GFLOP/s)."""
    g = C.c_double()
    _check(load().b200ode_fp64_peak(int(device), C.byref(g)))
    return g.value


def fp32_peak_gflops(device: int = -1) -> float:
    """Measured FP32 FMA throughput of the device (GFLOP/s)."""
    g = C.c_double()
    _check(load().b200ode_fp32_peak(int(device), C.byref(g)))
    return g.value


def algorithmic_flops(mech: str, stats: dict) -> float:
    from .roofline import algorithmic_flops as _af
    return _af(mech, stats)


PHASES = ["rhs", "jac", "lu", "solve", "total"]


def stats_dict(st: Stats) -> dict:
    d = {f: getattr(st, f) for f, _ in Stats._fields_ if f not in COUNTERS and f != "phase_cycles"}
    d["phase_cycles"] = {k: int(st.phase_cycles[i]) for i, k in enumerate(PHASES)}
    return d
