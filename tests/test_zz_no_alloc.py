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


@pytest.mark.parametrize("mech,wl,precision,ncells", [
    ("gri30", "gri_32k", native.B200ODE_MIXED, 148 * 16),
    ("gri30", "gri_32k", native.B200ODE_FP64, 148 * 16),
    ("h2o2", "h2_1024", native.B200ODE_MIXED, 148 * 16),
    ("nDodecane_Reitz", "nc12_8k", native.B200ODE_MIXED, 148 * 16),
    ("nDodecane_Reitz", "nc12_8k", native.B200ODE_FP64, 148 * 16),
    (W.ESTIMATE, "kero_2k", native.B200ODE_MIXED, 148),
])
def test_noalloc_takes_every_default_full_launch(mech, wl, precision, ncells):
    """With enough cells for every resident warp of every SM (at most 16 per SM;
    one CTA per cell for the kerosene mechanism) the default launch of each
    compiled-in mechanism needs its largest scratch, and it fits the static
    array: the call is not refused and integrates every cell (a short interval:
    the launch shape does not depend on it)."""
    import torch
    b = W.make(wl, ncells, seed=5)
    s = native.Solver(mech, precision=precision)
    try:
        T = torch.from_numpy(b.T.copy()).cuda()
        Y = torch.from_numpy(np.ascontiguousarray(b.Y)).cuda()
        P = torch.from_numpy(np.ascontiguousarray(b.P)).cuda()
        stats = s.integrate_device_noalloc(b.ncells, P.data_ptr(), 0.0, T.data_ptr(), Y.data_ptr(), 1e-7)
        assert stats["n_failed"] == 0
        assert torch.isfinite(T).all()
    finally:
        s.close()
