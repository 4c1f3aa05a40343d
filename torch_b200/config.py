"""Lua configuration and initial-condition front end.

Mirrors the reference's configuration interface so that the same files drive
both:

* ``parse_parameters`` restates ``parseParameters`` (src/main.cpp:126-208):
  every ``Parameters.<Section>.<key>`` it reads, with the ``TorchParameters``
  defaults of src/Torch/Parameters.hpp:25-97 for keys that are absent
  (``parseLuaVariable`` keeps the default and warns, src/IO/ParseLua.hpp:28-34).
* ``read_initial_conditions`` restates ``DataReader::readDataParameters`` and
  ``DataReader::readGrid`` (src/IO/DataReader.cpp:18-125): the text snapshot
  format written by ``DataPrinter::print2D`` (src/IO/DataPrinter.cpp:139-174).
* The string-to-enum maps follow ``Constants::Constants`` (src/Torch/
  Constants.cpp:3-25): unknown strings fall back to ``"default"``.

Only the table-literal subset of Lua that TORCH configs use is accepted:
global numeric assignments, nested ``{ key = value }`` tables, numbers,
strings, booleans and ``+ - * /`` arithmetic on earlier globals.
"""
from __future__ import annotations

import dataclasses
import math
import re
from typing import Any, Dict, List, Optional, Tuple

import numpy as np

GEOMETRY = {"cartesian": 0, "cylindrical": 1, "spherical": 2, "default": 0}
CONDITION = {"free": 0, "reflecting": 1, "outflow": 2, "inflow": 3, "periodic": 4, "default": 0}
COUPLING = {"tti": 0, "neq": 1, "off": 2, "default": 2}
SCHEME = {"implicit": 0, "implicit2": 1, "explicit": 2, "default": 0}
# RiemannSolverFactory::create (src/Integrators/Riemann.cpp:246-257)
RIEMANN = {"HLLC": 0, "RotatedHLLC": 1, "HLL": 2, "default": 1}
# SlopeLimiterFactory::create (src/Integrators/SlopeLimiter.cpp:56-75)
LIMITER = {"monotonised_central": 0, "superbee": 1, "minmod": 2, "maxmod": 3,
           "leer": 4, "ospre": 5, "albada": 6, "default": 6}


def enum_value(table: Dict[str, int], key: str, default_key: str = "default") -> int:
    """EnumParser::parseEnum (src/Torch/Constants.hpp:31-41)."""
    if key in table:
        return table[key]
    return table[default_key]


# --------------------------------------------------------------------------
# Lua table-literal subset
# --------------------------------------------------------------------------
_TOKEN = re.compile(r"""
    (?P<ws>\s+) |
    (?P<comment>--[^\n]*) |
    (?P<num>(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?) |
    (?P<str>"(?:[^"\\]|\\.)*"|'(?:[^'\\]|\\.)*') |
    (?P<name>[A-Za-z_][A-Za-z_0-9]*) |
    (?P<op>[{}=,;+\-*/()^.\[\]])
""", re.VERBOSE)


class LuaSubsetError(ValueError):
    pass


def _tokenize(text: str) -> List[Tuple[str, str]]:
    out, pos = [], 0
    while pos < len(text):
        m = _TOKEN.match(text, pos)
        if not m:
            raise LuaSubsetError(f"unsupported Lua near: {text[pos:pos + 30]!r}")
        pos = m.end()
        kind = m.lastgroup
        if kind in ("ws", "comment"):
            continue
        out.append((kind, m.group()))
    return out


class _Parser:
    def __init__(self, tokens, env):
        self.t, self.i, self.env = tokens, 0, env

    def peek(self, k=0):
        j = self.i + k
        return self.t[j] if j < len(self.t) else ("eof", "")

    def take(self, val=None):
        tok = self.peek()
        if val is not None and tok[1] != val:
            raise LuaSubsetError(f"expected {val!r}, got {tok[1]!r}")
        self.i += 1
        return tok

    def chunk(self):
        while self.peek()[0] != "eof":
            if self.peek()[1] == "local":
                self.take()
            kind, name = self.take()
            if kind != "name":
                raise LuaSubsetError(f"expected a global name, got {name!r}")
            if self.peek()[1] == "(" or name == "function":
                raise LuaSubsetError("functions are not part of the config subset")
            self.take("=")
            self.env[name] = self.expr()
            if self.peek()[1] == ";":
                self.take()

    def expr(self):
        v = self.term()
        while self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            r = self.term()
            v = v + r if op == "+" else v - r
        return v

    def term(self):
        v = self.unary()
        while self.peek()[1] in ("*", "/"):
            op = self.take()[1]
            r = self.unary()
            v = v * r if op == "*" else v / r
        return v

    def unary(self):
        if self.peek()[1] == "-":
            self.take()
            return -self.unary()
        return self.atom()

    def atom(self):
        kind, val = self.take()
        if kind == "num":
            return float(val)
        if kind == "str":
            return bytes(val[1:-1], "utf-8").decode("unicode_escape")
        if kind == "name":
            if val == "true":
                return True
            if val == "false":
                return False
            if val == "nil":
                return None
            if val not in self.env:
                raise LuaSubsetError(f"undefined name {val!r}")
            return self.env[val]
        if val == "(":
            v = self.expr()
            self.take(")")
            return v
        if val == "{":
            return self.table()
        raise LuaSubsetError(f"unexpected token {val!r}")

    def table(self):
        out: Dict[Any, Any] = {}
        n = 1
        while self.peek()[1] != "}":
            if self.peek()[0] == "name" and self.peek(1)[1] == "=":
                key = self.take()[1]
                self.take("=")
                out[key] = self.expr()
            elif self.peek()[1] == "[":
                self.take("[")
                key = self.expr()
                self.take("]")
                self.take("=")
                out[key] = self.expr()
            else:
                out[n] = self.expr()
                n += 1
            if self.peek()[1] in (",", ";"):
                self.take()
        self.take("}")
        return out


def load_lua_tables(text: str) -> Dict[str, Any]:
    env: Dict[str, Any] = {}
    p = _Parser(_tokenize(text), env)
    p.chunk()
    return env


# --------------------------------------------------------------------------
# TorchParameters
# --------------------------------------------------------------------------
@dataclasses.dataclass
class TorchParameters:
    """Raw run parameters with the defaults of src/Torch/Parameters.hpp:25-97."""
    setupFile: str = ""
    initialConditions: str = ""
    nd: int = 0
    sideLength: float = 0.0
    ncells: Tuple[int, int, int] = (0, 0, 0)
    leftBC: Tuple[str, str, str] = ("free", "free", "free")
    rightBC: Tuple[str, str, str] = ("free", "free", "free")
    geometry: str = "cartesian"
    riemannSolver: str = "hll"
    slopeLimiter: str = "falle"
    rt_scheme: str = "implicit"
    rt_coupling: str = "off"
    spatialOrder: int = 0
    temporalOrder: int = 0
    tmax: float = 0.0
    radiation_on: bool = False
    cooling_on: bool = False
    debug: bool = True
    outputDirectory: str = "tmp/"
    ncheckpoints: int = 100
    dfloor: float = 0.0
    pfloor: float = 0.0
    tfloor: float = 0.0
    dscale: float = 0.0
    pscale: float = 0.0
    tscale: float = 0.0
    K1: float = 0.0
    K2: float = 0.0
    K3: float = 0.0
    K4: float = 0.0
    photoIonCrossSection: float = 0.0
    alphaB: float = 0.0
    tau0: float = 0.0
    minX: float = 0.0
    THI: float = 0.0
    THII: float = 0.0
    collisions_on: bool = False
    star_on: bool = False
    star_position: Tuple[int, int, int] = (0, 0, 0)
    faceSnap: Tuple[bool, bool, bool] = (False, False, False)
    photonEnergy: float = 0.0
    photonRate: float = 0.0
    massLossRate: float = 0.0
    windVelocity: float = 0.0
    windTemperature: float = 0.0
    windCellRadius: int = 0
    thermoHII_Switch: float = 0.0
    heatingAmplification: float = 1.0
    thermoSubcycling: bool = True
    minTempInitialState: bool = False
    massFractionH: float = 0.0
    heatCapacityRatio: float = 0.0

    def riemann_id(self) -> int:
        # An unknown name makes the factory throw; Torch::initialise then keeps
        # the default RotatedHLLC (src/Torch/Torch.cpp:66-70, Hydro.cpp:25-29).
        return RIEMANN.get(self.riemannSolver, RIEMANN["default"])

    def limiter_id(self) -> int:
        return LIMITER.get(self.slopeLimiter, LIMITER["default"])

    def coupling_id(self) -> int:
        # Radiation::initialise compares against "neq"/"tti" only (Radiation.cpp:44-49).
        return {"neq": 1, "tti": 0}.get(self.rt_coupling, 2)

    def scheme_id(self) -> int:
        return {"implicit2": 1, "explicit": 2}.get(self.rt_scheme, 0)


# (section, key, attribute, kind, index) in the order of src/main.cpp:134-204
_KEYS = [
    ("Integration", "density_scale", "dscale", float, None),
    ("Integration", "pressure_scale", "pscale", float, None),
    ("Integration", "time_scale", "tscale", float, None),
    ("Integration", "spatial_order", "spatialOrder", int, None),
    ("Integration", "temporal_order", "temporalOrder", int, None),
    ("Integration", "simulation_time", "tmax", float, None),
    ("Integration", "radiation_on", "radiation_on", bool, None),
    ("Integration", "cooling_on", "cooling_on", bool, None),
    ("Integration", "debug", "debug", bool, None),
    ("Integration", "initial_conditions", "initialConditions", str, None),
    ("Integration", "ncheckpoints", "ncheckpoints", int, None),
    ("Integration", "output_directory", "outputDirectory", str, None),
    ("Grid", "no_dimensions", "nd", int, None),
    ("Grid", "no_cells_x", "ncells", int, 0),
    ("Grid", "no_cells_y", "ncells", int, 1),
    ("Grid", "no_cells_z", "ncells", int, 2),
    ("Grid", "side_length", "sideLength", float, None),
    ("Grid", "geometry", "geometry", str, None),
    ("Grid", "left_boundary_condition_x", "leftBC", str, 0),
    ("Grid", "left_boundary_condition_y", "leftBC", str, 1),
    ("Grid", "left_boundary_condition_z", "leftBC", str, 2),
    ("Grid", "right_boundary_condition_x", "rightBC", str, 0),
    ("Grid", "right_boundary_condition_y", "rightBC", str, 1),
    ("Grid", "right_boundary_condition_z", "rightBC", str, 2),
    ("Hydrodynamics", "gamma", "heatCapacityRatio", float, None),
    ("Hydrodynamics", "density_floor", "dfloor", float, None),
    ("Hydrodynamics", "pressure_floor", "pfloor", float, None),
    ("Hydrodynamics", "temperature_floor", "tfloor", float, None),
    ("Hydrodynamics", "riemann_solver", "riemannSolver", str, None),
    ("Hydrodynamics", "slope_limiter", "slopeLimiter", str, None),
    ("Radiation", "K1", "K1", float, None),
    ("Radiation", "K2", "K2", float, None),
    ("Radiation", "K3", "K3", float, None),
    ("Radiation", "K4", "K4", float, None),
    ("Radiation", "photoion_cross_section", "photoIonCrossSection", float, None),
    ("Radiation", "case_b_recombination_coeff", "alphaB", float, None),
    ("Radiation", "tau_0", "tau0", float, None),
    ("Radiation", "minimum_hii_fraction", "minX", float, None),
    ("Radiation", "temperature_hi", "THI", float, None),
    ("Radiation", "temperature_hii", "THII", float, None),
    ("Radiation", "mass_fraction_hydrogen", "massFractionH", float, None),
    ("Radiation", "collisions_on", "collisions_on", bool, None),
    ("Radiation", "coupling", "rt_coupling", str, None),
    ("Radiation", "integration_scheme", "rt_scheme", str, None),
    ("Thermodynamics", "thermo_hii_switch", "thermoHII_Switch", float, None),
    ("Thermodynamics", "heating_amplification", "heatingAmplification", float, None),
    ("Thermodynamics", "thermo_subcycling", "thermoSubcycling", bool, None),
    ("Thermodynamics", "min_temp_initial_state", "minTempInitialState", bool, None),
    ("Star", "on", "star_on", bool, None),
    ("Star", "cell_position_x", "star_position", int, 0),
    ("Star", "cell_position_y", "star_position", int, 1),
    ("Star", "cell_position_z", "star_position", int, 2),
    ("Star", "snap_to_face_left_x", "faceSnap", bool, 0),
    ("Star", "snap_to_face_left_y", "faceSnap", bool, 1),
    ("Star", "snap_to_face_left_z", "faceSnap", bool, 2),
    ("Star", "photon_energy", "photonEnergy", float, None),
    ("Star", "photon_rate", "photonRate", float, None),
    ("Star", "wind_radius_in_cells", "windCellRadius", int, None),
    ("Star", "mass_loss_rate", "massLossRate", float, None),
    ("Star", "wind_velocity", "windVelocity", float, None),
    ("Star", "wind_temperature", "windTemperature", float, None),
]


def _convert(kind, v):
    if kind is bool:
        return bool(v)
    if kind is int:
        # Selene converts a Lua number with lua_tointeger (truncation).
        return int(math.trunc(float(v)))
    if kind is float:
        return float(v)
    if isinstance(v, float) and v.is_integer():
        v = int(v)
    return str(v)


def parse_parameters(text_or_path: str, warnings: Optional[list] = None) -> TorchParameters:
    """Reads ``Parameters`` from a TORCH Lua config (src/main.cpp:126-208)."""
    text = text_or_path
    if "\n" not in text_or_path and "=" not in text_or_path:
        with open(text_or_path) as f:
            text = f.read()
    env = load_lua_tables(text)
    root = env.get("Parameters", {})
    p = TorchParameters()
    for section, key, attr, kind, idx in _KEYS:
        sec = root.get(section, {}) if isinstance(root, dict) else {}
        if not isinstance(sec, dict) or key not in sec or sec[key] is None:
            if warnings is not None:
                warnings.append(f"Parameters.{section}.{key} missing; keeping default")
            continue
        v = _convert(kind, sec[key])
        if idx is None:
            setattr(p, attr, v)
        else:
            cur = list(getattr(p, attr))
            cur[idx] = v
            setattr(p, attr, tuple(cur))
    return p


# --------------------------------------------------------------------------
# Initial conditions in the reference's text snapshot format
# --------------------------------------------------------------------------
@dataclasses.dataclass
class InitialConditions:
    """Primitives in cgs on the interior cells, flat index i + nx*(j + ny*k)."""
    time: float
    ncells: Tuple[int, int, int]
    nd: int
    dx: float
    side_length: float
    den: np.ndarray
    pre: np.ndarray
    hii: np.ndarray
    vel: np.ndarray  # [3][N]
    grav: Optional[np.ndarray] = None  # [3][N] or None (zero); only a Lua setup provides it


def write_initial_conditions(path: str, ncells, dx_cgs: float, den, pre, hii, vel, time: float = 0.0):
    """Writes the DataPrinter::print2D layout (one cell per line, x fastest) at
    full double precision, so that both implementations read identical
    primitives.  Cell centres are written as (index + 0.5) * dx."""
    nx, ny, nz = ncells
    nd = 1 if ny == 1 else (2 if nz == 1 else 3)
    N = nx * ny * nz
    idx = np.arange(N)
    coords = [((idx % nx) + 0.5) * dx_cgs, (((idx // nx) % ny) + 0.5) * dx_cgs, ((idx // (nx * ny)) + 0.5) * dx_cgs]
    cols = coords[:nd] + [np.asarray(den, float), np.asarray(pre, float), np.asarray(hii, float)]
    cols += [np.asarray(vel[d], float) for d in range(nd)]
    table = np.stack(cols, axis=1)
    with open(path, "w") as f:
        f.write(f"{time!r}\n{nx}\n{ny}\n{nz}\n")
        np.savetxt(f, table, fmt="%.17g", delimiter="\t")


def read_initial_conditions(path: str) -> InitialConditions:
    """DataReader::readDataParameters + readGrid (src/IO/DataReader.cpp:18-125)."""
    with open(path) as f:
        toks = f.read().split()
    t = float(toks[0])
    ncells = (int(toks[1]), int(toks[2]), int(toks[3]))
    nd = 1 if ncells[1] == 1 else (2 if ncells[2] == 1 else 3)
    ncol = nd + 3 + nd
    body = np.array(toks[4:], dtype=np.float64)
    N = ncells[0] * ncells[1] * ncells[2]
    rows = body[: N * ncol].reshape(N, ncol)
    x0 = [0.0, 0.0, 0.0]
    x1 = [0.0, 0.0, 0.0]
    for d in range(nd):
        x0[d] = rows[0, d]
        x1[d] = rows[1, d] if N > 1 else rows[0, d]
    dxs = [abs(x1[d] - x0[d]) for d in range(nd) if abs(x1[d] - x0[d]) > np.finfo(np.float64).tiny]
    dx = min(dxs)
    side = dx * ncells[0]
    den = np.zeros(N); pre = np.zeros(N); hii = np.zeros(N); vel = np.zeros((3, N))
    # readGrid: coordinates truncate x/dx to a cell index; Grid::locate places the values.
    xi = np.zeros((N, 3), dtype=np.int64)
    for d in range(nd):
        xi[:, d] = np.trunc(rows[:, d] / dx).astype(np.int64)
    ok = (xi[:, 0] >= 0) & (xi[:, 0] < ncells[0]) & (xi[:, 1] >= 0) & (xi[:, 1] < ncells[1]) \
        & (xi[:, 2] >= 0) & (xi[:, 2] < ncells[2])
    flat = xi[:, 0] + ncells[0] * (xi[:, 1] + ncells[1] * xi[:, 2])
    den[flat[ok]] = rows[ok, nd]
    pre[flat[ok]] = rows[ok, nd + 1]
    hii[flat[ok]] = rows[ok, nd + 2]
    for d in range(nd):
        vel[d, flat[ok]] = rows[ok, nd + 3 + d]
    return InitialConditions(t, ncells, nd, dx, side, den, pre, hii, vel)


def to_lua(tp: TorchParameters) -> str:
    """Writes the Parameters table that parse_parameters reads back (and that
    the reference's own parseParameters reads, src/main.cpp:126-208)."""
    def lit(v):
        if isinstance(v, bool):
            return "true" if v else "false"
        if isinstance(v, str):
            return '"' + v.replace('"', '\\"') + '"'
        if isinstance(v, int):
            return str(v)
        return repr(float(v))

    sections: Dict[str, List[str]] = {}
    for section, key, attr, kind, idx in _KEYS:
        v = getattr(tp, attr)
        if idx is not None:
            v = v[idx]
        sections.setdefault(section, []).append(f"\t\t{key} = {lit(v)},")
    out = ["Parameters = {"]
    for section, lines in sections.items():
        out.append(f"\t{section} = {{")
        out.extend(lines)
        out.append("\t},")
    out.append("}")
    return "\n".join(out) + "\n"


def make_initial_conditions(ncells, dx: float, den, pre, hii, vel, time: float = 0.0) -> InitialConditions:
    """In-memory initial conditions with side_length = dx * ncells[0]."""
    nx, ny, nz = ncells
    nd = 1 if ny == 1 else (2 if nz == 1 else 3)
    vel = np.asarray(vel, dtype=np.float64)
    return InitialConditions(time, tuple(ncells), nd, dx, dx * nx, np.asarray(den, np.float64),
                             np.asarray(pre, np.float64), np.asarray(hii, np.float64), vel)
