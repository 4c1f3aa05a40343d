"""Seeded initial-condition generators for the benchmark and parity workloads.

The reference builds its initial state from a Lua ``initialise(x,y,z,xs,ys,zs)``
callback (src/Torch/Torch.cpp:192-228) or from a text snapshot
(src/IO/DataReader.cpp:70-125).  These generators produce the same kind of
primitive fields (cgs, interior cells, x fastest) for the workloads measured
here; the arrays are handed to the reference through the text snapshot format
and to this library through its C interface, so both see identical inputs.

* ``blister_profile``: the density profile of the shipped 2-D cylindrical
  setup (config/torch-setup.lua: n(R) = n0 (1 + R^2/rc^2)^-alpha with the star
  offset RS along the axis, uniform T), restated in numpy.
* ``sedov_blast``: uniform medium plus a thermal-energy deposit inside a sphere
  of a few cells at the grid centre.
* ``lognormal_cloud``: a seeded Gaussian random field with a power-law
  spectrum, exponentiated to a lognormal density of given mean and sigma_ln.
"""
from __future__ import annotations

import numpy as np

HYDROGEN_MASS = 1.674e-24
SPECIFIC_GAS_CONSTANT = 8.314462e7
PC2CM = 3.09e18


def cell_centres(ncells, dx):
    nx, ny, nz = ncells
    idx = np.arange(nx * ny * nz)
    return [((idx % nx) + 0.5) * dx, (((idx // nx) % ny) + 0.5) * dx, ((idx // (nx * ny)) + 0.5) * dx]


def blister_profile(ncells=(150, 200, 1), side=0.5 * PC2CM, star_cell=(0, 110), T=300.0,
                    nHI=32000.0, rc_pc=0.01, RS_pc=0.35, alpha=1.0):
    nx, ny, nz = ncells
    dx = side / nx
    x, y, _ = cell_centres(ncells, dx)
    # the star sits on the axis (face-snapped in x) at the centre of cell row star_cell[1]
    xs, ys = 0.0, (star_cell[1] + 0.5) * dx
    rc = rc_pc * PC2CM
    RS = RS_pc * PC2CM
    n0 = nHI * (1 + RS * RS / (rc * rc)) ** alpha
    dy = RS + (ys - y)
    R2 = x * x + dy * dy
    den = n0 * HYDROGEN_MASS * (1 + R2 / (rc * rc)) ** (-alpha)
    pre = np.full_like(den, SPECIFIC_GAS_CONSTANT * nHI * HYDROGEN_MASS * T)
    N = den.size
    return dict(den=den, pre=pre, hii=np.zeros(N), vel=np.zeros((3, N)), dx=dx)


def sedov_blast(n=32, side=2 * PC2CM, rho=1e-20, P=1e-12, E=1e51, radius_cells=3.0, gamma=1.67, nd=3):
    ncells = (n, n, n) if nd == 3 else ((n, n, 1) if nd == 2 else (n, 1, 1))
    dx = side / n
    cs = cell_centres(ncells, dx)
    centre = 0.5 * side
    r2 = np.zeros(int(np.prod(ncells)))
    for d in range(nd):
        r2 = r2 + (cs[d] - centre) ** 2
    inside = r2 <= (radius_cells * dx) ** 2
    N = r2.size
    den = np.full(N, rho)
    pre = np.full(N, P)
    vol = dx ** nd
    ninside = int(inside.sum())
    pre[inside] = P + (gamma - 1.0) * E / (ninside * vol)
    return dict(den=den, pre=pre, hii=np.zeros(N), vel=np.zeros((3, N)), dx=dx, ncells=ncells)


def lognormal_cloud(n=64, side=2 * PC2CM, mean_n=1e3, sigma_ln=0.5, slope=-11.0 / 3.0, T=100.0, seed=12345):
    """Lognormal number density with P(k) ~ k^slope (3-D), mean mean_n, sigma of ln n = sigma_ln."""
    rng = np.random.default_rng(seed)
    k = np.fft.fftfreq(n) * n
    kx, ky, kz = np.meshgrid(k, k, k, indexing="ij")
    kk = np.sqrt(kx * kx + ky * ky + kz * kz)
    kk[0, 0, 0] = 1.0
    amp = kk ** (slope / 2.0)
    amp[0, 0, 0] = 0.0
    noise = rng.standard_normal((n, n, n)) + 1j * rng.standard_normal((n, n, n))
    field = np.real(np.fft.ifftn(noise * amp))
    field = (field - field.mean()) / field.std() * sigma_ln
    nfield = np.exp(field)
    nfield *= mean_n / nfield.mean()
    # grid order: x fastest -> transpose (i, j, k) to flat i + n*(j + n*k)
    nflat = np.ascontiguousarray(nfield.transpose(2, 1, 0)).reshape(-1)
    den = nflat * HYDROGEN_MASS
    pre = nflat * HYDROGEN_MASS * SPECIFIC_GAS_CONSTANT * T
    N = den.size
    return dict(den=den, pre=pre, hii=np.zeros(N), vel=np.zeros((3, N)), dx=side / n, ncells=(n, n, n))
