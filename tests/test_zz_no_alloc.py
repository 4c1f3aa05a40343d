"""The allocation-free FP32 hydro step (trg_hydro_step_fp32_noalloc), called
through the C ABI on caller-owned device buffers, against the regular FP32
full step of a context (trg_full_step) for the same state and time step, on
two calls in a row.

Callers of this entry point may not allocate device memory while they run
(their device memory is reserved up front by their own allocator, or
cudaMalloc's implicit synchronisation is not allowed on their stepping path);
the second call is also checked to leave the device's free memory unchanged.
Collected last (file name) so that a run stopping at the first failure has
already run every other test; it needs nothing from the other tests.
"""
import ctypes as C

import numpy as np
import pytest

import common
import torch_b200
from torch_b200 import workloads

pytestmark = pytest.mark.gpu

TOL = 1e-5  # the FP32 tests' bound for the Sedov blast


def test_noalloc_step_matches_full_step_two_calls():
    import torch
    tp, ic = workloads.sedov(n=32)
    ref = torch_b200.Torch(tp, ic, precision=torch_b200.PRECISION_FP32)
    ref.run_steps(1)  # the reference's dt_max * 1e-20 start step
    dev_in = torch.from_numpy(ref.state().U.copy()).cuda()
    dev_out = torch.empty_like(dev_in)
    torch.cuda.synchronize()
    lib = ref.lib
    for call in range(2):
        dt = ref.full_step()
        expected = ref.state().U
        free_before = torch.cuda.mem_get_info()[0]
        rc = lib.trg_hydro_step_fp32_noalloc(ref.ctx, C.c_void_p(dev_in.data_ptr()),
                                             C.c_void_p(dev_out.data_ptr()), dt, None, None)
        assert rc == 0, lib.trg_last_error(ref.ctx).decode()
        if call == 1:
            assert torch.cuda.mem_get_info()[0] == free_before
        got = dev_out.cpu().numpy()
        for f in range(7):
            assert common.rel_l1(got[f], expected[f]) <= TOL, (call, f)
        dev_in.copy_(dev_out)
    ref.close()


def test_noalloc_step_in_place_at_the_size_limit_on_a_side_stream():
    """64^3 = TRG_NOALLOC_MAX_CELLS cells (the scratch's intermediate state
    fully used), stepped in place (U_in == U_out) on a non-default stream; the
    time step each call reports for the next one is the one trg_full_step
    takes next."""
    import torch
    tp, ic = workloads.sedov(n=64)
    ref = torch_b200.Torch(tp, ic, precision=torch_b200.PRECISION_FP32)
    ref.run_steps(1)
    buf = torch.from_numpy(ref.state().U.copy()).cuda()
    side = torch.cuda.Stream()
    torch.cuda.synchronize()
    lib = ref.lib
    dt_next = C.c_double(0.0)
    prev_next = None
    for call in range(2):
        dt = ref.full_step()
        if prev_next is not None:
            assert dt == prev_next
        rc = lib.trg_hydro_step_fp32_noalloc(ref.ctx, C.c_void_p(buf.data_ptr()), C.c_void_p(buf.data_ptr()), dt,
                                             C.byref(dt_next), C.c_void_p(side.cuda_stream))
        assert rc == 0, lib.trg_last_error(ref.ctx).decode()
        assert dt_next.value > 0
        prev_next = dt_next.value
        expected = ref.state().U
        got = buf.cpu().numpy()
        for f in range(7):
            assert common.rel_l1(got[f], expected[f]) <= TOL, (call, f)
    ref.close()


def test_noalloc_step_rejects_radiation_contexts_and_bad_dt():
    import torch
    tp, ic = workloads.hii_region(n=12, seed=3)
    sim = torch_b200.Torch(tp, ic, precision=torch_b200.PRECISION_FP32)
    buf = torch.zeros((7, 12 ** 3), dtype=torch.float64, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    assert sim.lib.trg_hydro_step_fp32_noalloc(sim.ctx, p, p, 1e-3, None, None) == 1
    assert "hydrodynamics only" in sim.lib.trg_last_error(sim.ctx).decode()
    sim.close()
    tp, ic = workloads.sedov(n=16)
    sim = torch_b200.Torch(tp, ic, precision=torch_b200.PRECISION_FP32)
    buf = torch.zeros((7, 16 ** 3), dtype=torch.float64, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    for dt in (0.0, -1.0, float("nan"), float("inf")):
        assert sim.lib.trg_hydro_step_fp32_noalloc(sim.ctx, p, p, dt, None, None) == 1
    sim.close()


def test_noalloc_step_rejects_grids_above_the_limit():
    import torch
    tp, ic = workloads.sedov(n=65)  # 274625 cells > TRG_NOALLOC_MAX_CELLS
    sim = torch_b200.Torch(tp, ic, precision=torch_b200.PRECISION_FP32)
    buf = torch.zeros((7, 65 ** 3), dtype=torch.float64, device="cuda")
    rc = sim.lib.trg_hydro_step_fp32_noalloc(sim.ctx, C.c_void_p(buf.data_ptr()), C.c_void_p(buf.data_ptr()),
                                             1e-3, None, None)
    assert rc == 1
    assert "exceeds the limit of 262144 cells" in sim.lib.trg_last_error(sim.ctx).decode()
    sim.close()
