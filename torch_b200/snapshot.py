"""Checkpoint files in the reference's formats, written from a run on the GPU.

* ``write_data2d`` - ``DataPrinter::print2D`` (src/IO/DataPrinter.cpp:139-174):
  gzip text, the time in seconds and the three cell counts on their own
  lines, then one line per cell (x fastest) with the cell centre in cm for
  each dimension, density (g/cm^3), pressure (dyn/cm^2), HII fraction and
  the velocity components (cm/s), tab separated, ``%.10e``.
* ``write_heating`` - ``DataPrinter::printHeating`` (:325-354): the same
  header, then the cell centre in cell units and the 11 heating/cooling terms
  of ``Thermodynamics::fillHeatingArrays`` in erg/cm^3/s.

The files are what ``Torch::run`` writes at a checkpoint and what the
reference's ``DataReader`` reads back as initial conditions.  Conversions
restate ``Converter`` (src/Torch/Converter.cpp:17-63) so that the numbers
round as the reference's do.
"""
from __future__ import annotations

import gzip
import math

import numpy as np

from .config import TorchParameters


class Converter:
    """Converter::set_rho_pressure_time and ::convertCodeUnits."""

    def __init__(self, dscale: float, pscale: float, tscale: float):
        M, L, T = 1.0 * 2.0e33, 14.6 * 3.09e18, 10000.0 * 3.15569e7
        rho_0 = dscale if dscale > 0 else M / (L * L * L)
        pressure_0 = pscale if pscale > 0 else rho_0 * L * L / (T * T)
        T = tscale if tscale > 0 else T
        self.M = math.sqrt((pressure_0 / rho_0) * pressure_0 * pressure_0) * T * T * T
        self.L = math.sqrt(pressure_0 / rho_0) * T
        self.T = T

    def _convert(self, val, mi, li, ti, to_code):
        MM = self.M if mi >= 0 else 1.0 / self.M
        LL = self.L if li >= 0 else 1.0 / self.L
        TT = self.T if ti >= 0 else 1.0 / self.T
        if to_code:
            MM, LL, TT = 1.0 / MM, 1.0 / LL, 1.0 / TT
        im, il, it = int(abs(mi)), int(abs(li)), int(abs(ti))
        result = np.asarray(val, dtype=np.float64)
        while im >= 1 or il >= 1 or it >= 1:
            if im >= 1:
                result = result * MM
            im -= 1
            if il >= 1:
                result = result * LL
            il -= 1
            if it >= 1:
                result = result * TT
            it -= 1
        return result

    def to_code(self, val, mi, li, ti):
        return self._convert(val, mi, li, ti, True)

    def from_code(self, val, mi, li, ti):
        return self._convert(val, mi, li, ti, False)


def _cells(ncells, nd):
    nx, ny, nz = ncells
    idx = np.arange(nx * ny * nz)
    ijk = [idx % nx, (idx // nx) % ny, idx // (nx * ny)]
    return [ijk[d] + 0.5 for d in range(nd)]


def _header(f, conv, time_code, ncells):
    f.write(f"{float(conv.from_code(time_code, 0, 0, 1)):.10e}\n{ncells[0]}\n{ncells[1]}\n{ncells[2]}\n")


def _table(f, cols):
    np.savetxt(f, np.stack(cols, axis=1), fmt="%.10e", delimiter="\t")


def write_data2d(path: str, tp: TorchParameters, ncells, Q: np.ndarray, time_code: float):
    """DataPrinter::print2D of the primitives Q [7][N] (code units) at time
    `time_code` (code units)."""
    conv = Converter(tp.dscale, tp.pscale, tp.tscale)
    nd = 1 if ncells[1] == 1 else (2 if ncells[2] == 1 else 3)
    side = float(conv.to_code(tp.sideLength, 0, 1, 0))
    dx = side / ncells[0]  # Grid.cpp:470-471: every dimension uses ncells[0]
    cols = [conv.from_code(xc * dx, 0, 1, 0) for xc in _cells(ncells, nd)]
    cols += [conv.from_code(Q[0], 1, -3, 0), conv.from_code(Q[1], 1, -1, -2), np.asarray(Q[2], dtype=np.float64)]
    cols += [conv.from_code(Q[4 + d], 0, 1, -1) for d in range(nd)]
    with gzip.open(path, "wt") as f:
        _header(f, conv, time_code, ncells)
        _table(f, cols)


def write_heating(path: str, tp: TorchParameters, ncells, H: np.ndarray, time_code: float):
    """DataPrinter::printHeating of the heating terms H [11][N] (code units)."""
    conv = Converter(tp.dscale, tp.pscale, tp.tscale)
    nd = 1 if ncells[1] == 1 else (2 if ncells[2] == 1 else 3)
    cols = list(_cells(ncells, nd)) + [conv.from_code(H[i], 1, -1, -3) for i in range(H.shape[0])]
    with gzip.open(path, "wt") as f:
        _header(f, conv, time_code, ncells)
        _table(f, cols)


def write_checkpoint(directory: str, sim, tp: TorchParameters, ncells, suffix: str = "final"):
    """What Torch::run writes at a checkpoint (src/Torch/Torch.cpp:270-281):
    heating_<suffix>.txt.gz and data2D_<suffix>.txt.gz.  `sim` is a
    torch_b200.Torch run with heating_enable() on since its first step."""
    H = sim.heating()
    s = sim.state()
    write_heating(f"{directory}/heating_{suffix}.txt.gz", tp, ncells, H, s.time)
    write_data2d(f"{directory}/data2D_{suffix}.txt.gz", tp, ncells, s.Q, s.time)


def read_table(path: str):
    """(time_s, ncells, rows[N][ncol]) of a print2D / printHeating file."""
    opener = gzip.open if path.endswith(".gz") else open
    with opener(path, "rt") as f:
        lines = f.read().split("\n")
    t = float(lines[0])
    ncells = (int(lines[1]), int(lines[2]), int(lines[3]))
    rows = [ln.split("\t") for ln in lines[4:] if ln.strip()]
    vals = np.array([[float(v) for v in r] for r in rows], dtype=np.float64)
    return t, ncells, vals
