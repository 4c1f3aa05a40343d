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
}


def build(name, tmpdir=None):
    """Returns (tp, ic_through_text, ic_text, steps)."""
    tp, ic, steps = (CASES[name] if name in CASES else globals()[name])()
    ic2, text = _through_text(ic, tmpdir)
    return tp, ic2, text, steps
