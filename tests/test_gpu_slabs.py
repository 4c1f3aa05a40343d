"""x-slab decomposition (torch_b200.slabs): every slab of a run in one
process on one GPU, each stepped by its own host thread, halos and sweep
boundary layers copied between the slabs' buffers by the exchange hook.  The
state assembled from the slabs must equal the undecomposed run's bit for bit:
a face between two slabs gets the same flux from both (the ghost layers are
the neighbour's cells), a cell whose upwind neighbours lie in the star-side
slab reads their optical depths and column densities from that slab's
boundary layer, and the time step is the minimum over the slabs."""
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


def test_slab_needs_its_exchange_hooks_the_fp64_form_with_a_star_and_no_wind():
    tp, ic = workloads.sedov(n=16)
    s = torch_b200.Torch(tp, ic, slab=(0, 8, None))
    with pytest.raises(torch_b200.TrgError):
        s.run_steps(1)
    s.close()
    tp2, ic2 = workloads.hii_region(n=16, seed=2)
    with pytest.raises(torch_b200.TrgError):  # radiation slabs take the FP64 form
        torch_b200.Torch(tp2, ic2, precision=torch_b200.PRECISION_FP32, slab=(0, 8, None))
    with pytest.raises(torch_b200.TrgError):  # no stellar wind
        torch_b200.Torch(dataclasses.replace(tp2, windCellRadius=2, massLossRate=1e-6), ic2, slab=(0, 8, None))
    s = torch_b200.Torch(tp2, ic2, slab=(0, 8, None))
    assert s.lib.trg_slab_star_side(s.ctx) == 2  # the star (cell 8) lies at higher x
    with pytest.raises(torch_b200.TrgError):  # no hook and no sweep buffers yet
        s.run_steps(1)
    s.close()


def rad_whole_and_slabs(tp, ic, nslabs, steps):
    whole = torch_b200.Torch(tp, ic)
    whole.run_steps(steps)
    ref = whole.state()
    whole.close()
    ls = slabs.LocalSlabs(tp, ic, nslabs)
    ls.run_steps(steps)
    U, Q, R, T, sts = ls.full_state()
    ls.close()
    return ref, U, R, T, sts


def assert_rad_bitwise(ref, U, R, T, sts):
    assert np.array_equal(U, ref.U)
    assert np.array_equal(R, ref.R)
    assert np.array_equal(T, ref.T)
    for st in sts:
        assert np.array_equal(st.dts, ref.dts) and st.time == ref.time


# K1 = 0: the reference gives each rank's first causal cell the one-off form
# of the recombination time step (a function-local static per process,
# Radiation.cpp:300-316), so a decomposed run with K1 != 0 takes different
# time steps from an undecomposed one by design; with K1 = 0 they agree.
@pytest.mark.parametrize("nslabs,star,scheme", [(2, (8, 8, 8), "implicit"), (3, (8, 8, 8), "implicit"),
                                                (3, (2, 9, 6), "implicit"), (4, (13, 4, 9), "implicit2")])
def test_fp64_hii_region_slabs_bitwise(nslabs, star, scheme):
    """3-D HII region with radiation, cooling and hydrodynamics: the slab
    holding the star sweeps first and each other slab after its star-side
    neighbour; state, optical depths, column densities and time steps equal
    the undecomposed run's bit for bit."""
    tp, ic = workloads.hii_region(n=16, seed=3)
    tp = dataclasses.replace(tp, K1=0.0, star_position=star, rt_scheme=scheme)
    assert_rad_bitwise(*rad_whole_and_slabs(tp, ic, nslabs, 12))


def test_fp64_blister_slabs_bitwise():
    """The shipped 2-D cylindrical blister (radiation, cooling, hydrodynamics;
    the star on the axis, in the first slab; wind off), three slabs."""
    tp, ic = workloads.blister()
    tp = dataclasses.replace(tp, K1=0.0, windCellRadius=0, massLossRate=0.0)
    assert_rad_bitwise(*rad_whole_and_slabs(tp, ic, 3, 10))


def test_fp64_hii_region_slabs_with_per_slab_one_off_time_step():
    """With K1 != 0 every slab's first causal non-wind cell takes the one-off
    recombination time step, as every rank's does in the reference: the first
    step (dt_max) and its state agree with the undecomposed run; the second
    step is at most the undecomposed one, since the slabs' one-off cells add
    candidates to the minimum."""
    tp, ic = workloads.hii_region(n=16, seed=3)
    tp = dataclasses.replace(tp, star_position=(8, 8, 8))
    whole = torch_b200.Torch(tp, ic)
    whole.run_steps(1)
    ref1 = whole.state()
    whole.run_steps(1)
    ref2 = whole.state()
    whole.close()
    ls = slabs.LocalSlabs(tp, ic, 3)
    ls.run_steps(1)
    U1, _, R1, _, _ = ls.full_state()
    ls.run_steps(1)
    _, _, _, _, sts = ls.full_state()
    ls.close()
    assert np.array_equal(U1, ref1.U) and np.array_equal(R1, ref1.R)
    for st in sts:
        assert st.dts[0] == ref2.dts[0] and st.dts[1] <= ref2.dts[1]
        assert np.all(np.isfinite(st.U))
