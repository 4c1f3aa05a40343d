"""Global FP64 mass and energy sums (trg_conservation_*): exact against the
oracle's rational-arithmetic sums of the same state, conserved to rounding in
a periodic box, and the per-step record (formed inside the time-step
reduction) equal to the on-demand sums of the same states."""
import dataclasses

import numpy as np
import pytest

import common
import oracle
import torch_b200
from torch_b200 import workloads

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["sedov3d_small", "blister_small", "sedov2d_mixed_bc"])
def test_sums_equal_exact_oracle_sums_on_golden(name):
    """The FP64 form is bit-exact with the reference on the golden cases, so
    its sums must be the exact sums of the reference's final state, rounded
    once (cartesian and cylindrical volumes)."""
    tp, ic, steps, ref = common.load_golden(name)
    t = torch_b200.Torch(tp, ic)
    t.run_steps(steps)
    m, e = t.conservation_sums()
    U = t.state().U
    t.close()
    o = oracle.Oracle(tp, ic)
    vol = o.cell_volumes()
    o.close()
    m_ref, e_ref = oracle.conservation_sums(U, vol)
    print(f"{name}: mass {m!r} vs {m_ref!r}, energy {e!r} vs {e_ref!r}")
    assert m == m_ref and e == e_ref
    # and the reference's own final state has the same sums to the parity bar
    m_g, e_g = oracle.conservation_sums(ref["U"], vol)
    assert abs(m / m_g - 1) <= 1e-10 and abs(e / e_g - 1) <= 1e-10


def test_periodic_sedov_conserves_mass_and_energy():
    """A periodic 3-D Sedov box, FP64 form: every face flux leaves one cell
    and enters another, so total mass and energy change only by rounding
    (relative drift <= 1e-13 over 40 steps)."""
    tp, ic = workloads.sedov(n=24)
    tp = dataclasses.replace(tp, leftBC=("periodic",) * 3, rightBC=("periodic",) * 3)
    t = torch_b200.Torch(tp, ic)
    t.conservation_enable(True)
    t.run_steps(40)
    h = t.conservation_history()
    m1, e1 = t.conservation_sums()
    t.close()
    assert h.shape == (40, 2)
    m0, e0 = h[0]
    dm = max(abs(h[:, 0] / m0 - 1).max(), abs(m1 / m0 - 1))
    de = max(abs(h[:, 1] / e0 - 1).max(), abs(e1 / e0 - 1))
    print(f"periodic sedov24 40 steps: mass drift {dm:.2e}, energy drift {de:.2e}")
    assert dm <= 1e-13 and de <= 1e-13


def test_periodic_sedov_fp32_form_conserves_to_fp32_rounding():
    tp, ic = workloads.sedov(n=24)
    tp = dataclasses.replace(tp, leftBC=("periodic",) * 3, rightBC=("periodic",) * 3)
    t = torch_b200.Torch(tp, ic, precision=torch_b200.PRECISION_FP32)
    t.conservation_enable(True)
    t.run_steps(40)
    h = t.conservation_history()
    t.close()
    dm = abs(h[:, 0] / h[0, 0] - 1).max()
    de = abs(h[:, 1] / h[0, 1] - 1).max()
    print(f"periodic sedov24 FP32 form 40 steps: mass drift {dm:.2e}, energy drift {de:.2e}")
    assert dm <= 1e-6 and de <= 1e-6


@pytest.mark.parametrize("precision", [torch_b200.PRECISION_FP64, torch_b200.PRECISION_FP32])
def test_record_equals_on_demand_sums(precision):
    """Record k (formed by the time-step reduction of step k, or by a pass
    of its own where none runs) is bitwise the on-demand sum of the state
    after k steps; radiation-hydro HII region in both forms."""
    tp, ic = workloads.hii_region(n=20, seed=4)
    t = torch_b200.Torch(tp, ic, precision=precision)
    t.conservation_enable(True)
    demand = [t.conservation_sums()]
    for _ in range(6):
        t.full_step()
        demand.append(t.conservation_sums())
    h = t.conservation_history()
    t.close()
    assert h.shape == (6, 2)
    for k in range(6):
        assert tuple(h[k]) == demand[k], (k, tuple(h[k]), demand[k])
