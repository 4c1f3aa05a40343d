"""Known answers through the C ABI on the GPU: the Sod shock tube against
its exact solution in the FP64 form (1-D, also bit for bit the oracle) and
the FP32 form (2-D, the fused hydro kernel), and the D-type expansion of an
HII region against Spitzer's law in the FP64 form (1-D spherical, I-front
within half a cell of the oracle's)."""
import dataclasses

import numpy as np
import pytest

import known_answers as ka
import oracle
import torch_b200
from test_known_answers import run_to, sod_errors, spitzer_track

pytestmark = pytest.mark.gpu


def test_fp64_sod_matches_exact_solution_and_oracle():
    n = 400
    tp, ic = ka.sod_case(n)
    t = torch_b200.Torch(tp, ic)
    st = run_to(t, tp, ka.sod_time())
    t.close()
    r, p = sod_errors(st, tp, n)
    assert r < 0.005 and p < 0.004
    o = oracle.Oracle(tp, ic)
    ref = run_to(o, tp, ka.sod_time())
    o.close()
    assert np.array_equal(st.U, ref.U)  # hydrodynamics only: no transcendental, bit for bit


def test_fp32_sod_2d_matches_exact_solution():
    """The fused FP32 hydro kernel (2-D: a tube of 400 x 4 cells, outflow in
    y): every row is the exact solution to the same bar as the FP64 form."""
    n, ny = 400, 4
    tp, ic1 = ka.sod_case(n)
    tp = dataclasses.replace(tp, nd=2, ncells=(n, ny, 1), star_position=(0, 0, 0))
    den = np.tile(ic1.den, ny)
    pre = np.tile(ic1.pre, ny)
    ic = torch_b200.config.make_initial_conditions((n, ny, 1), ic1.dx, den, pre, np.zeros(n * ny),
                                                   np.zeros((3, n * ny)))
    t = torch_b200.Torch(tp, ic, precision=torch_b200.PRECISION_FP32)
    st = run_to(t, tp, ka.sod_time())
    t.close()
    rho_e, _, p_e = ka.sod_exact_profile(n, st.time * tp.tscale)
    for row in range(ny):
        rho = st.Q[0].reshape(ny, n)[row] * tp.dscale
        p = st.Q[1].reshape(ny, n)[row] * tp.pscale
        assert np.abs(rho - rho_e).sum() / np.abs(rho_e).sum() < 0.005
        assert np.abs(p - p_e).sum() / np.abs(p_e).sum() < 0.004


def test_fp64_hii_region_follows_spitzer_expansion():
    n, side = 200, 6.0
    tp, ic = ka.spitzer_case(n, side)
    t = torch_b200.Torch(tp, ic)
    track = spitzer_track(t, tp, n, side)
    t.close()
    errs = [abs(r - s) / s for r, s in track]
    assert all(a < b for (a, _), (b, _) in zip(track, track[1:]))
    assert errs[0] < 0.045 and errs[1] < 0.03 and errs[2] < 0.025
    o = oracle.Oracle(tp, ic)
    ref = spitzer_track(o, tp, n, side)
    o.close()
    rs_cells = ka.stromgren_radius() / (side * ka.PC2CM / n)
    for (r, _), (q, _) in zip(track, ref):
        assert abs(r - q) * rs_cells < 0.5  # I-front within half a cell of the oracle's
