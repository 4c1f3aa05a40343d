"""Named workloads: run parameters plus seeded initial conditions.

* ``blister``   - the reference's shipped 2-D cylindrical HII-region setup
                  (config/torch-config.lua + config/torch-setup.lua): 150x200,
                  0.5 pc, rotated HLLC, albada, radiation + cooling + stellar
                  wind, star face-snapped at cell (0, 110).
* ``sedov``     - hydro-only Sedov blast: uniform rho = 1e-20 g/cm^3,
                  P = 1e-12 dyn/cm^2, 1e51 erg in a 3-cell-radius sphere at the
                  centre, outflow boundaries, albada-limited piecewise-linear
                  reconstruction (the reference's spatial_order = 1), RK2.
* ``hii_region``- 3-D HII-region expansion: lognormal density (mean 1e3 cm^-3,
                  sigma_ln 0.5, P(k) ~ k^-11/3, seeded), T = 100 K, star of
                  1e49 photons/s at the centre, radiation + cooling, wind off.
* ``blister_batch`` - many independent 2-D cylindrical HII-region grids of
                  uneven sizes (64-256 x 64-320), photon rates and cloud
                  profiles, for batched stepping.

Each returns ``(TorchParameters, InitialConditions)``.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import setups
from .config import TorchParameters, make_initial_conditions

PC2CM = 3.09e18
YR2S = 3.15569e7


def blister_parameters(ncells=(150, 200, 1)) -> TorchParameters:
    """The values of the shipped config/torch-config.lua."""
    return TorchParameters(
        dscale=1.0e-20, pscale=1.0e-28, tscale=1.0e11, spatialOrder=1, temporalOrder=2,
        tmax=5.0e4 * YR2S, radiation_on=True, cooling_on=True, debug=False, outputDirectory="tmp",
        initialConditions="", ncheckpoints=100, nd=2, ncells=tuple(ncells), geometry="cylindrical",
        sideLength=0.5 * PC2CM, leftBC=("reflecting", "outflow", "reflecting"),
        rightBC=("outflow", "outflow", "outlfow"), heatCapacityRatio=1.67, dfloor=1.0e-30,
        pfloor=1.0e-22, tfloor=0.1, riemannSolver="RotatedHLLC", slopeLimiter="albada",
        K1=0.2, K2=0.0, K3=0.0, K4=0.0, photoIonCrossSection=6.3e-18, alphaB=2.59e-13, tau0=0.6,
        minX=0.0, THI=300.0, THII=10000.0, massFractionH=1.0, rt_scheme="implicit",
        collisions_on=False, rt_coupling="neq", heatingAmplification=1.0, thermoHII_Switch=1e-2,
        thermoSubcycling=True, minTempInitialState=True, star_on=True, star_position=(0, 110, 0),
        faceSnap=(True, False, False), photonEnergy=2.976e-11, photonRate=4.9e48,
        windCellRadius=10, massLossRate=9.79e18, windVelocity=311000000.0, windTemperature=10000.0)


def blister(ncells=(150, 200, 1), star_cell_y=None, side=None):
    nx, ny, _ = ncells
    tp = blister_parameters(ncells)
    if star_cell_y is None:
        star_cell_y = int(round(110 * ny / 200))
    side = 0.5 * PC2CM * nx / 150 if side is None else side
    tp = dataclasses.replace(tp, star_position=(0, star_cell_y, 0), sideLength=side)
    g = setups.blister_profile(ncells=ncells, side=side, star_cell=(0, star_cell_y))
    return tp, make_initial_conditions(ncells, g["dx"], g["den"], g["pre"], g["hii"], g["vel"])


def sedov_parameters(n=256, nd=3, order=1, riemann="RotatedHLLC", limiter="albada", side=2 * PC2CM):
    ncells = (n, n if nd > 1 else 1, n if nd > 2 else 1)
    return TorchParameters(
        dscale=1.0e-20, pscale=1.0e-12, tscale=3.0e11, spatialOrder=order, temporalOrder=2,
        tmax=1.0e13, radiation_on=False, cooling_on=False, debug=False, ncheckpoints=100,
        nd=nd, ncells=ncells, geometry="cartesian", sideLength=side,
        leftBC=("outflow",) * 3, rightBC=("outflow",) * 3, heatCapacityRatio=1.67,
        dfloor=1.0e-30, pfloor=1.0e-22, tfloor=0.1, riemannSolver=riemann, slopeLimiter=limiter,
        massFractionH=1.0, star_on=False, star_position=(n // 2, n // 2 if nd > 1 else 0, n // 2 if nd > 2 else 0),
        thermoHII_Switch=1e-2, minTempInitialState=False)


def sedov(n=256, nd=3, order=1, riemann="RotatedHLLC", limiter="albada", side=2 * PC2CM):
    tp = sedov_parameters(n, nd, order, riemann, limiter, side)
    g = setups.sedov_blast(n=n, nd=nd, side=side)
    return tp, make_initial_conditions(g["ncells"], g["dx"], g["den"], g["pre"], g["hii"], g["vel"])


def hii_region_parameters(n=256, side=2 * PC2CM, photon_rate=1e49):
    c = n // 2
    return TorchParameters(
        dscale=1.0e-20, pscale=1.0e-10, tscale=1.0e11, spatialOrder=1, temporalOrder=2,
        tmax=3.0e4 * YR2S, radiation_on=True, cooling_on=True, debug=False, ncheckpoints=100,
        nd=3, ncells=(n, n, n), geometry="cartesian", sideLength=side,
        leftBC=("outflow",) * 3, rightBC=("outflow",) * 3, heatCapacityRatio=1.67,
        dfloor=1.0e-30, pfloor=1.0e-22, tfloor=0.1, riemannSolver="RotatedHLLC", slopeLimiter="albada",
        K1=0.2, K2=0.0, K3=0.0, K4=0.0, photoIonCrossSection=6.3e-18, alphaB=2.59e-13, tau0=0.6,
        minX=0.0, THI=300.0, THII=10000.0, massFractionH=1.0, rt_scheme="implicit",
        collisions_on=False, rt_coupling="neq", heatingAmplification=1.0, thermoHII_Switch=1e-2,
        thermoSubcycling=True, minTempInitialState=True, star_on=True, star_position=(c, c, c),
        faceSnap=(False, False, False), photonEnergy=2.976e-11, photonRate=photon_rate,
        windCellRadius=0, massLossRate=0.0, windVelocity=0.0, windTemperature=10000.0)


def hii_region(n=256, seed=12345, side=2 * PC2CM, photon_rate=1e49):
    tp = hii_region_parameters(n, side, photon_rate)
    g = setups.lognormal_cloud(n=n, side=side, seed=seed)
    return tp, make_initial_conditions(g["ncells"], g["dx"], g["den"], g["pre"], g["hii"], g["vel"])


def blister_batch(G=256, seed=2024, nx_range=(64, 256), ny_range=(64, 320), q_range=(1e47, 1e49),
                  alpha_range=(0.0, 2.0), rc_pc_range=(0.005, 0.05)):
    """Independent 2-D cylindrical HII-region grids of uneven sizes: nx, ny
    uniform in the ranges, photon rate log-uniform, cloud n(R) = n0 (1 +
    R^2/rc^2)^-alpha with alpha and rc uniform (the shipped setup's profile,
    nHI = 32000 cm^-3 at the star, star offset 0.35 pc, T = 300 K), the
    shipped cell size (0.5 pc / 150), star on the axis at row 0.55 ny,
    radiation and cooling on, wind off.  Returns a list of (params, initial
    conditions)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(G):
        nx = int(rng.integers(nx_range[0], nx_range[1] + 1))
        ny = int(rng.integers(ny_range[0], ny_range[1] + 1))
        q = float(10 ** rng.uniform(np.log10(q_range[0]), np.log10(q_range[1])))
        alpha = float(rng.uniform(*alpha_range))
        rc = float(rng.uniform(*rc_pc_range))
        side = 0.5 * PC2CM * nx / 150
        star_y = int(round(0.55 * ny))
        tp = dataclasses.replace(blister_parameters((nx, ny, 1)), star_position=(0, star_y, 0), sideLength=side,
                                 photonRate=q, windCellRadius=0, massLossRate=0.0)
        g = setups.blister_profile(ncells=(nx, ny, 1), side=side, star_cell=(0, star_y), rc_pc=rc, alpha=alpha)
        out.append((tp, make_initial_conditions((nx, ny, 1), g["dx"], g["den"], g["pre"], g["hii"], g["vel"])))
    return out
