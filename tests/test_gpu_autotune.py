"""The autotuner (b200ode_autotune): it leaves the sample cells untouched,
picks one of its candidates (warps per CTA, register variant, threads per cell
for the widest mechanism, work-queue chunk), and integration results do not
depend on the launch shape (bitwise)."""
import numpy as np
import pytest

from hpc_ode_b200 import native, workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [native.B200ODE_MIXED, native.B200ODE_FP64])
def test_autotune_picks_a_shape_and_results_do_not_change(precision):
    import torch
    b = W.make("gri_32k", 3000, seed=17)
    T = torch.from_numpy(b.T.copy()).cuda()
    Y = torch.from_numpy(np.ascontiguousarray(b.Y)).cuda()
    P = torch.from_numpy(b.P.copy()).cuda()
    T0, Y0 = T.clone(), Y.clone()
    s = native.Solver("gri30", precision=precision)
    wpb, bps = s.autotune(b.ncells, P.data_ptr(), 0.0, T.data_ptr(), Y.data_ptr(), b.dt)
    torch.cuda.synchronize()
    assert (wpb, bps) in {(4, 0), (2, 0), (1, 0), (4, 3), (2, 6), (1, 12)}
    o = s.options()
    assert o.queue_chunk in (1, 2, 8)
    assert (o.warps_per_block, o.blocks_per_sm) == (wpb, bps)
    assert torch.equal(T, T0) and torch.equal(Y, Y0)          # sample left untouched
    st = torch.zeros(b.ncells, dtype=torch.int32, device="cuda")
    s.integrate_device(b.ncells, P.data_ptr(), 0.0, T.data_ptr(), Y.data_ptr(), b.dt, dstatus=st.data_ptr())
    s.close()
    ref = native.Solver("gri30", precision=precision, warps_per_block=4)
    T2, Y2 = T0.clone(), Y0.clone()
    ref.integrate_device(b.ncells, P.data_ptr(), 0.0, T2.data_ptr(), Y2.data_ptr(), b.dt)
    ref.close()
    torch.cuda.synchronize()
    assert (st == 0).all()
    assert torch.equal(T, T2) and torch.equal(Y, Y2)


def test_autotune_skips_shapes_that_do_not_fit():
    """The 214-species mechanism fits one warp per CTA (its Newton matrix fills
    the shared memory): the autotuner times only the shapes that fit and keeps
    one of them."""
    import torch
    b = W.make("kero_2k", 148, seed=18)
    T = torch.from_numpy(b.T.copy()).cuda()
    Y = torch.from_numpy(np.ascontiguousarray(b.Y)).cuda()
    P = torch.from_numpy(b.P.copy()).cuda()
    T0, Y0 = T.clone(), Y.clone()
    s = native.Solver(b.mech)
    wpb, bps = s.autotune(b.ncells, P.data_ptr(), 0.0, T.data_ptr(), Y.data_ptr(), b.dt)
    torch.cuda.synchronize()
    assert wpb == 1 and bps in (0, 12)
    assert s.options().cta_helpers in (0, 1)
    assert torch.equal(T, T0) and torch.equal(Y, Y0)
    s.integrate_device(b.ncells, P.data_ptr(), 0.0, T.data_ptr(), Y.data_ptr(), b.dt)
    s.close()
    ref = native.Solver(b.mech)
    T2, Y2 = T0.clone(), Y0.clone()
    ref.integrate_device(b.ncells, P.data_ptr(), 0.0, T2.data_ptr(), Y2.data_ptr(), b.dt)
    ref.close()
    torch.cuda.synchronize()
    assert torch.equal(T, T2) and torch.equal(Y, Y2)


def test_autotune_h2_keeps_results_bitwise():
    """The 10-species H2 mechanism: whichever shape and queue chunk the
    autotuner keeps, the integration equals the default launch bitwise."""
    import torch
    b = W.make("h2_1024", 4096, seed=19)
    T = torch.from_numpy(b.T.copy()).cuda()
    Y = torch.from_numpy(np.ascontiguousarray(b.Y)).cuda()
    P = torch.from_numpy(b.P.copy()).cuda()
    T0, Y0 = T.clone(), Y.clone()
    s = native.Solver(b.mech)
    s.autotune(b.ncells, P.data_ptr(), 0.0, T.data_ptr(), Y.data_ptr(), b.dt)
    assert s.options().queue_chunk in (1, 2, 8)
    st = torch.zeros(b.ncells, dtype=torch.int32, device="cuda")
    s.integrate_device(b.ncells, P.data_ptr(), 0.0, T.data_ptr(), Y.data_ptr(), b.dt, dstatus=st.data_ptr())
    s.close()
    ref = native.Solver(b.mech)
    T2, Y2 = T0.clone(), Y0.clone()
    ref.integrate_device(b.ncells, P.data_ptr(), 0.0, T2.data_ptr(), Y2.data_ptr(), b.dt)
    ref.close()
    torch.cuda.synchronize()
    assert (st == 0).all()
    assert torch.equal(T, T2) and torch.equal(Y, Y2)
