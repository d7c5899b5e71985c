"""b200ode_integrate_device_noalloc (the entry point that allocates no device
memory) against b200ode_integrate_device, both called through the C ABI on
device buffers.

Two calls of the no-allocation entry point in a row, on different cells and cell
counts, so the second call runs on the scratch the first one left behind; each
must agree with the allocating entry point on the same cells within the
integration tolerances of the parity tests: |dT|/T <= 1e-5 and
|dY| <= max(1e-4 |Y|, 1e-10) for every entry, the same per-cell status and the
same call totals.  Collected last (file name) so it also runs after every other
test in one process.
"""
import numpy as np
import pytest

from conftest import y_ok
from hpc_ode_b200 import native, workloads as W

pytestmark = pytest.mark.gpu

GATE_T = 1e-5


def _run(solver, b, noalloc):
    import torch
    T = torch.from_numpy(b.T.copy()).cuda()
    Y = torch.from_numpy(np.ascontiguousarray(b.Y)).cuda()
    P = torch.from_numpy(np.ascontiguousarray(b.P)).cuda()
    status = torch.full((b.ncells,), 99, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    call = solver.integrate_device_noalloc if noalloc else solver.integrate_device
    stats = call(b.ncells, P.data_ptr(), 0.0, T.data_ptr(), Y.data_ptr(), b.dt,
                 dstatus=status.data_ptr())
    torch.cuda.synchronize()
    return T.cpu().numpy(), Y.cpu().numpy(), status.cpu().numpy(), stats


def _check_same(a, b):
    Ta, Ya, sa, sta = a
    Tb, Yb, sb, stb = b
    assert np.array_equal(sa, sb)
    assert (sa == 0).all()
    assert (np.abs(Ta - Tb) / Tb).max() <= GATE_T
    assert y_ok(Ya, Yb).all()
    for k in ("total_nst", "total_nfe", "total_nje", "total_nsetups", "total_nni", "n_failed"):
        assert sta[k] == stb[k], k


@pytest.mark.parametrize("mech,wl,precision,sizes", [
    ("gri30", "gri_32k", native.B200ODE_MIXED, (300, 77)),
    ("h2o2", "h2_1024", native.B200ODE_FP64, (257, 1024)),
])
def test_noalloc_matches_integrate_device_two_calls(mech, wl, precision, sizes):
    s = native.Solver(mech, precision=precision)
    try:
        for i, n in enumerate(sizes):
            b = W.make(wl, n, seed=21 + i)
            ref = _run(s, b, noalloc=False)
            got = _run(s, b, noalloc=True)
            _check_same(got, ref)
    finally:
        s.close()


def test_noalloc_rejects_bad_arguments():
    s = native.Solver("gri30")
    try:
        with pytest.raises(native.B200Error):
            s.integrate_device_noalloc(4, 0, 101325.0, 0, 0, 1e-4)
        with pytest.raises(native.B200Error):
            s.integrate_device_noalloc(-1, 0, 101325.0, 0, 0, 1e-4)
    finally:
        s.close()


def test_noalloc_refuses_a_launch_larger_than_its_scratch():
    """n-dodecane in FP64 keeps about 89 KB of scratch per resident warp; its
    default launch (2 resident warps on each SM) needs more than the 24 MiB
    array, so the call is refused with a message that gives the numbers, and the
    allocating entry point still integrates the same cells."""
    import torch
    b = W.make("nc12_8k", 600, seed=3)
    s = native.Solver("nDodecane_Reitz", precision=native.B200ODE_FP64)
    try:
        T = torch.from_numpy(b.T.copy()).cuda()
        Y = torch.from_numpy(np.ascontiguousarray(b.Y)).cuda()
        P = torch.from_numpy(np.ascontiguousarray(b.P)).cuda()
        with pytest.raises(native.B200Error) as e:
            s.integrate_device_noalloc(b.ncells, P.data_ptr(), 0.0, T.data_ptr(), Y.data_ptr(), b.dt)
        assert e.value.code == 1 and "static scratch holds" in str(e.value)
        torch.cuda.synchronize()
        assert torch.equal(T, torch.from_numpy(b.T).cuda())     # nothing ran
        stats = s.integrate_device(b.ncells, P.data_ptr(), 0.0, T.data_ptr(), Y.data_ptr(), b.dt)
        assert stats["n_failed"] == 0
    finally:
        s.close()
