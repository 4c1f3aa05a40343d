"""Parity cases shared by the tests and tests/golden/make_golden.py.

Each case is (TorchParameters, InitialConditions, steps).  Initial conditions
go through the reference's text snapshot format (write + DataReader-style
read), so the grid spacing is derived exactly as the reference derives it.
"""
from __future__ import annotations

import dataclasses
import os
import tempfile

import numpy as np

from torch_b200 import config, workloads


def _through_text(ic, tmpdir=None):
    d = tmpdir or tempfile.mkdtemp(prefix="trg_case_")
    path = os.path.join(d, "ic_000.txt")
    config.write_initial_conditions(path, ic.ncells, ic.dx, ic.den, ic.pre, ic.hii, ic.vel)
    with open(path) as f:
        text = f.read()
    return config.read_initial_conditions(path), text


def blister_small():
    tp, ic = workloads.blister(ncells=(30, 40, 1), star_cell_y=22)
    tp = dataclasses.replace(tp, windCellRadius=3)
    return tp, ic, 30


def blister_full():
    tp, ic = workloads.blister()
    return tp, ic, 20


def sedov3d_small():
    tp, ic = workloads.sedov(n=12, nd=3)
    return tp, ic, 10


def sedov2d_mixed_bc():
    # 2-D, periodic x / reflecting-inflow y, HLL solver, minmod limiter
    tp, ic = workloads.sedov(n=16, nd=2, riemann="HLL", limiter="minmod")
    tp = dataclasses.replace(tp, leftBC=("periodic", "reflecting", "free"), rightBC=("periodic", "inflow", "free"))
    rng = np.random.default_rng(7)
    ic.vel[0] = rng.normal(0, 3e6, ic.den.size)
    ic.vel[1] = rng.normal(0, 3e6, ic.den.size)
    return tp, ic, 12


def sedov1d_order0():
    tp, ic = workloads.sedov(n=40, nd=1, order=0, riemann="HLLC", limiter="superbee")
    return tp, ic, 15


def sedov3d_limiters():
    tp, ic = workloads.sedov(n=10, nd=3, limiter="monotonised_central")
    rng = np.random.default_rng(11)
    for d in range(3):
        ic.vel[d] = rng.normal(0, 1e6, ic.den.size)
    return tp, ic, 6


def hii3d_small():
    tp, ic = workloads.hii_region(n=12, seed=3)
    return tp, ic, 10


def hii3d_offcentre():
    tp, ic = workloads.hii_region(n=14, seed=5)
    tp = dataclasses.replace(tp, star_position=(3, 9, 6), windCellRadius=2, massLossRate=1e18,
                             windVelocity=2e8)
    return tp, ic, 8


def hii3d_implicit2():
    """transferRadiation2 with the implicit2 scheme (Radiation.cpp:508-567)."""
    tp, ic = workloads.hii_region(n=12, seed=6)
    return dataclasses.replace(tp, rt_scheme="implicit2"), ic, 10


def blister_explicit():
    """transferRadiation2 with the explicit scheme, shipped 2-D setup at 30x40."""
    tp, ic, steps = blister_small()
    return dataclasses.replace(tp, rt_scheme="explicit"), ic, 20


# Cases whose initial state comes from a Lua setup script (the reference's
# Torch::setUpLua path), which is also the only way gravity enters a run.
class LuaSetup:
    def __init__(self, text):
        self.text = text


GRAV2D_LUA = """-- isothermal atmosphere in a constant downward gravity, with a shear perturbation
PC2CM = 3.09e18
g = 2.0e-9
rho0 = 1.0e-20
cs2 = 1.0e10
H = cs2 / g
L = 0.5 * PC2CM

function initialise(x, y, z, xs, ys, zs)
	local den = rho0 * math.exp(-y / H)
	local pre = cs2 * den
	local v0 = 3.0e4 * math.sin(2 * math.pi * y / L)
	local v1 = 1.0e4 * math.cos(2 * math.pi * x / L)
	-- the reference's GRAV is a force density (Hydro.cpp:134-137): rho g
	return den, pre, 0, v0, v1, 0, 0, -g * den, 0
end
"""

SPH1D_LUA = """-- 1-D spherical blast: hot core of three cells in a uniform medium
PC2CM = 3.09e18
dx = 0.5 * PC2CM / 64

function initialise(x, y, z, xs, ys, zs)
	local pre = 1.0e-12
	if x < 3 * dx then
		pre = 1.0e-9
	elseif x < 4 * dx then
		pre = 1.0e-10
	end
	return 1.0e-20, pre, 0, 0, 0, 0, 0, 0, 0
end
"""


def grav2d_lua():
    """Gravity (Hydrodynamics::updateSourceTerms, Hydro.cpp:134-137), 2-D
    cartesian, periodic in x, reflecting in y."""
    tp = workloads.sedov_parameters(n=20, nd=2)
    tp = dataclasses.replace(tp, ncells=(20, 24, 1), sideLength=0.5 * workloads.PC2CM, pscale=1.0e-10,
                             tscale=1.0e11, leftBC=("periodic", "reflecting", "free"),
                             rightBC=("periodic", "reflecting", "free"))
    return tp, LuaSetup(GRAV2D_LUA), 12


def sph1d_lua():
    """Spherical geometry (Grid.cpp:846-907 volumes and areas, the P/r
    source of Hydro.cpp:145-151), 1-D."""
    tp = workloads.sedov_parameters(n=64, nd=1)
    tp = dataclasses.replace(tp, geometry="spherical", sideLength=0.5 * workloads.PC2CM, tscale=1.0e11)
    return tp, LuaSetup(SPH1D_LUA), 15


def blister_collisions():
    """Collisional ionisation on (collisions_on: the Voronov rate in the
    implicit solve, the heating and the time step), shipped 2-D setup at
    30x40.  (The 3-D HII region at 12^3 with collisions on drives the
    reference's time step down to ~1e-45 s within a few steps, where its
    result depends on single ulps of libm; this case stays regular.)"""
    tp, ic, steps = blister_small()
    return dataclasses.replace(tp, collisions_on=True), ic, steps


def blister_tti():
    """TTI coupling of radiation and hydro (Radiation::updateSourceTerms,
    Radiation.cpp:657-671), shipped 2-D setup at 30x40.  (In the 12^3 HII
    region the first TTI step already moves the state by ~1e-6 when a single
    libm result changes by one ulp - the implicit solve's stopping test flips
    for some cell - so that case cannot carry a 1e-10 bar for a build with
    another libm; this one stays at 1e-13.)"""
    tp, ic, steps = blister_small()
    return dataclasses.replace(tp, rt_coupling="tti"), ic, steps


def _limiter_case(limiter):
    tp, ic = workloads.sedov(n=16, nd=2, limiter=limiter)
    rng = np.random.default_rng(13)
    for d in range(2):
        ic.vel[d] = rng.normal(0, 1e6, ic.den.size)
    return tp, ic, 8


def sedov2d_maxmod():
    """maxmod is compressive (it takes the larger slope), so across the blast
    the reconstructed pressure goes negative and the reference throws: a
    smooth subsonic field instead."""
    tp, ic = workloads.sedov(n=16, nd=2, limiter="maxmod")
    rng = np.random.default_rng(17)
    ic.pre[:] = 1.0e-12
    ic.den *= 1.0 + 0.1 * rng.standard_normal(ic.den.size)
    for d in range(2):
        ic.vel[d] = rng.normal(0, 3e3, ic.den.size)
    return tp, ic, 8


def sedov2d_leer():
    return _limiter_case("leer")


def sedov2d_ospre():
    return _limiter_case("ospre")


CASES = {
    "blister_small": blister_small,
    "sedov3d_small": sedov3d_small,
    "sedov2d_mixed_bc": sedov2d_mixed_bc,
    "sedov1d_order0": sedov1d_order0,
    "sedov3d_limiters": sedov3d_limiters,
    "hii3d_small": hii3d_small,
    "hii3d_offcentre": hii3d_offcentre,
    "hii3d_implicit2": hii3d_implicit2,
    "blister_explicit": blister_explicit,
    "grav2d_lua": grav2d_lua,
    "sph1d_lua": sph1d_lua,
    "blister_collisions": blister_collisions,
    "blister_tti": blister_tti,
    "sedov2d_maxmod": sedov2d_maxmod,
    "sedov2d_leer": sedov2d_leer,
    "sedov2d_ospre": sedov2d_ospre,
}


def build(name, tmpdir=None):
    """Returns (tp, ic_through_text, ic_text, steps); for a Lua-setup case
    (tp, LuaSetup, None, steps)."""
    tp, ic, steps = (CASES[name] if name in CASES else globals()[name])()
    if isinstance(ic, LuaSetup):
        return tp, ic, None, steps
    ic2, text = _through_text(ic, tmpdir)
    return tp, ic2, text, steps
