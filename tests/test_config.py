"""Host-side front end: Lua config subset, initial-condition text format."""
import os
import tempfile

import numpy as np
import pytest

from torch_b200 import config, workloads


def test_lua_round_trip():
    tp, _ = workloads.blister()
    assert config.parse_parameters(config.to_lua(tp)) == tp


def test_lua_defaults_and_unknown_enums():
    text = 'X = 2\nParameters = { Grid = { no_cells_x = X * 8, geometry = "weird" } }\n'
    warnings = []
    tp = config.parse_parameters(text, warnings)
    assert tp.ncells == (16, 0, 0)
    assert tp.riemannSolver == "hll" and tp.riemann_id() == config.RIEMANN["default"]
    assert tp.limiter_id() == config.LIMITER["albada"]
    assert config.enum_value(config.GEOMETRY, tp.geometry) == 0
    assert any("density_scale" in w for w in warnings)


def test_lua_rejects_functions():
    with pytest.raises(config.LuaSubsetError):
        config.parse_parameters("Parameters = { } function f() end\n")


def test_initial_conditions_round_trip():
    rng = np.random.default_rng(0)
    n = (5, 4, 3)
    N = 60
    den, pre, hii = rng.random(N), rng.random(N), rng.random(N)
    vel = rng.normal(size=(3, N))
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "ic_000.txt")
        config.write_initial_conditions(p, n, 3.7e16, den, pre, hii, vel)
        ic = config.read_initial_conditions(p)
    assert ic.nd == 3 and ic.ncells == n
    assert np.array_equal(ic.den, den) and np.array_equal(ic.vel, vel)
    assert abs(ic.side_length / (3.7e16 * 5) - 1) < 1e-12
