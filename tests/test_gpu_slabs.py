"""x-slab decomposition of hydrodynamics-only runs (torch_b200.slabs): every
slab of a run in one process on one GPU, each stepped by its own host thread,
halos copied between the slabs' buffers by the exchange hook.  The state
assembled from the slabs must equal the undecomposed run's bit for bit: a
face between two slabs gets the same flux from both (the ghost layers are the
neighbour's cells), and the time step is the minimum over the slabs."""
import dataclasses

import numpy as np
import pytest

import torch_b200
from torch_b200 import slabs, workloads

pytestmark = pytest.mark.gpu


def whole_and_slabs(tp, ic, nslabs, steps, precision=torch_b200.PRECISION_FP64):
    whole = torch_b200.Torch(tp, ic, precision=precision)
    whole.run_steps(steps)
    ref = whole.state()
    whole.close()
    ls = slabs.LocalSlabs(tp, ic, nslabs, precision=precision)
    ls.run_steps(steps)
    U, Q, times = ls.state()
    ls.close()
    return ref, U, Q, times


@pytest.mark.parametrize("nslabs", [2, 3])
def test_fp64_sedov_slabs_bitwise(nslabs):
    tp, ic = workloads.sedov(n=24)
    ref, U, Q, times = whole_and_slabs(tp, ic, nslabs, 12)
    assert np.array_equal(U, ref.U)
    assert all(t == ref.time for t in times)


def test_fp64_periodic_slabs_bitwise():
    """Periodic x: the two ends of the grid are neighbours (the reference's
    PERIODIC_MSG between the first and the last rank, Grid.cpp:823-826)."""
    tp, ic = workloads.sedov(n=20, nd=2)
    tp = dataclasses.replace(tp, leftBC=("periodic", "outflow", "outflow"), rightBC=("periodic", "outflow", "outflow"))
    ref, U, Q, times = whole_and_slabs(tp, ic, 3, 15)
    assert np.array_equal(U, ref.U)


def test_fp64_cylindrical_slabs_bitwise():
    """The shipped 2-D cylindrical setup with hydrodynamics only: the slabs'
    cell volumes, face areas and the P/r source use global radii."""
    tp, ic = workloads.blister()
    tp = dataclasses.replace(tp, radiation_on=False, cooling_on=False, star_on=False)
    ref, U, Q, times = whole_and_slabs(tp, ic, 4, 10)
    assert np.array_equal(U, ref.U)


def test_fp32_sedov_slabs_bitwise():
    """The hydro-only FP32 form (one fused kernel per RK2 stage): with the
    whole grid's reference density and pressure in every slab, and the
    partition ghost layers staged from the halo, the slabs give the
    undecomposed FP32 run's state bit for bit."""
    tp, ic = workloads.sedov(n=32)
    ref, U, Q, times = whole_and_slabs(tp, ic, 2, 10, precision=torch_b200.PRECISION_FP32)
    assert np.array_equal(U, ref.U)


def test_slab_needs_its_exchange_hook_and_a_hydro_only_run():
    tp, ic = workloads.sedov(n=16)
    s = torch_b200.Torch(tp, ic, slab=(0, 8, None))
    with pytest.raises(torch_b200.TrgError):
        s.run_steps(1)
    s.close()
    tp2, ic2 = workloads.hii_region(n=16, seed=2)
    with pytest.raises(torch_b200.TrgError):
        torch_b200.Torch(tp2, ic2, slab=(0, 8, None))
