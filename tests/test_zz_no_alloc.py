"""b200ode_integrate_device_noalloc (the entry point that allocates no device
memory) against b200ode_integrate_device, both called through the C ABI on
device buffers.

Two calls of the no-allocation entry point in a row, on different cells and cell
counts, so the second call runs on the scratch the first one left behind.  Both
entry points launch the same kernel on the same grid, so each call must return
bitwise the results, per-cell statuses and call totals of the allocating entry
point on the same cells; and the device's free memory must not move across the
second no-allocation call.  Collected last (file name) so it also runs after
every other test in one process.
"""
import numpy as np
import pytest

from hpc_ode_b200 import native, workloads as W

pytestmark = pytest.mark.gpu


def _run(solver, b, noalloc):
    """One call on fresh device copies of the batch; returns the results, the
    totals and the device's free bytes just before and just after the call."""
    import torch
    T = torch.from_numpy(b.T.copy()).cuda()
    Y = torch.from_numpy(np.ascontiguousarray(b.Y)).cuda()
    P = torch.from_numpy(np.ascontiguousarray(b.P)).cuda()
    status = torch.full((b.ncells,), 99, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    call = solver.integrate_device_noalloc if noalloc else solver.integrate_device
    stats = call(b.ncells, P.data_ptr(), 0.0, T.data_ptr(), Y.data_ptr(), b.dt,
                 dstatus=status.data_ptr())
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    return T.cpu().numpy(), Y.cpu().numpy(), status.cpu().numpy(), stats, (free0, free1)


def _check_same(a, b):
    Ta, Ya, sa, sta, _ = a
    Tb, Yb, sb, stb, _ = b
    assert (sa == 0).all()
    assert np.array_equal(sa, sb)
    assert np.array_equal(Ta, Tb)
    assert np.array_equal(Ya, Yb)
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
            if i == 1:
                free0, free1 = got[4]
                assert free1 == free0, (free0, free1)
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
