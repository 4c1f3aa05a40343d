"""The Lua setup interface (Torch::setUpLua, src/Torch/Torch.cpp:196-228):
the library's evaluator of setup scripts against the reference's own Lua.

* golden Lua-setup cases (tests/golden/*_lua.npz): the nine values per cell
  that the reference's Lua 5.2 returned for the script, reproduced bit for
  bit from the positions the library computes (trg_setup_positions);
* the shipped config/torch-setup.lua, evaluated by the reference build in
  this container when the reference tree is present;
* the language subset itself (precedence, multiple results, control flow,
  Lua's arithmetic corner cases).
"""
import math
import os
import subprocess
import tempfile

import numpy as np
import pytest

import common
import oracle
import torch_b200
from torch_b200 import config, lua_setup

LUA_GOLDEN = [n for n in common.golden_names() if n.endswith("_lua")]


def _eval_golden(name):
    z = np.load(os.path.join(common.GOLDEN, f"{name}.npz"))
    tp = config.parse_parameters(str(z["params_lua"]))
    ic = torch_b200.initial_conditions_from_lua(tp, lua_setup.LuaScript(str(z["setup_lua"])))
    ours = np.vstack([ic.den, ic.pre, ic.hii, ic.vel, ic.grav])
    return ours, z["setup_vals"]


@pytest.mark.parametrize("name", LUA_GOLDEN)
def test_evaluator_matches_reference_lua_bitwise(name):
    ours, ref = _eval_golden(name)
    assert ours.shape == ref.shape
    assert np.array_equal(ours, ref)


def test_shipped_setup_matches_reference_lua_bitwise():
    setup = os.path.join(oracle.REF_TREE, "config", "torch-setup.lua")
    params = os.path.join(oracle.REF_TREE, "config", "torch-config.lua")
    binp = oracle.build_reference() if os.path.exists(setup) else None
    if binp is None:
        pytest.skip("reference tree or build unavailable")
    with tempfile.TemporaryDirectory() as d:
        dump = os.path.join(d, "setup.bin")
        subprocess.run([binp, f"--params={params}", f"--setup={setup}", "--steps=0", f"--out={d}/o.bin",
                        f"--setup-dump={dump}"], cwd=d, check=True, capture_output=True, timeout=300)
        ref = np.fromfile(dump).reshape(9, -1)
    tp = config.parse_parameters(open(params).read())
    ic = torch_b200.initial_conditions_from_lua(tp, setup)
    assert np.array_equal(np.vstack([ic.den, ic.pre, ic.hii, ic.vel, ic.grav]), ref)


def run(src, *args, fn="f"):
    return lua_setup.LuaScript(src).call_global(fn, *args)


def test_language_subset():
    assert run("function f(a, b) return a + b * 2 ^ 2, -a ^ 2 end", 1.0, 3.0) == [13.0, -1.0]
    assert run("function f() return 2 ^ 3 ^ 2 end") == [512.0]  # right associative
    assert run("function f(x) if x < 0 then return -1 elseif x == 0 then return 0 else return 1 end end",
               0.0) == [0.0]
    assert run("function f() local s = 0 for i = 1, 10, 3 do s = s + i end return s end") == [22.0]
    assert run("function f() local i, s = 0, 0 while i < 5 do i = i + 1 if i == 4 then break end s = s + i end "
               "return s end") == [6.0]
    assert run("local function g(a) return a, a * 2 end function f() return g(3) end") == [3.0, 6.0]
    assert run("local function g(a) return a, a * 2 end function f() return g(3), 1 end") == [3.0, 1.0]
    assert run("function f() local a = nil return a or 5, false and 1, not nil end") == [5.0, False, True]
    assert run("k = 3 function f() return k * 2 end") == [6.0]
    assert run("function f() return 5 % -3, -5 % 3, 5.5 % 2 end") == [-1.0, 1.0, 1.5]
    assert run("function f() return 1 / 0, -1 / 0 end") == [math.inf, -math.inf]
    assert math.isnan(run("function f() return 0 / 0 end")[0])
    assert run("function f() return math.log(100, 10), math.max(1, 7, 3), math.floor(-1.5) end") == \
        [2.0, 7.0, -2.0]
    assert run("function f() return 0x10, 1e2, .5 end") == [16.0, 100.0, 0.5]
    assert run("-- comment\n--[[ block\ncomment ]] function f() return 'a' .. 1 end") == ["a1"]


def test_unsupported_syntax_is_refused():
    for src in ("t = {1, 2}", "function f(...) end", "for k, v in pairs(x) do end", "goto x"):
        with pytest.raises(lua_setup.LuaError):
            lua_setup.LuaScript(src)
    with pytest.raises(lua_setup.LuaError):
        run("function f() return nil + 1 end")


def test_setup_positions_cover_the_grid():
    """Cell centres at (index + 1/2) dx for the dimensions in use, 0 beyond;
    the star face-snapped to x = 0 (Star.cpp:13-25)."""
    z = np.load(os.path.join(common.GOLDEN, "blister_small.npz"))
    tp = config.parse_parameters(str(z["params_lua"]))
    x, y, zz, star = torch_b200.setup_positions(tp)
    nx, ny, _ = tp.ncells
    assert x.shape == (nx * ny,) and np.all(zz == 0)
    dx = x[1] - x[0]
    assert np.allclose(x[:nx], (np.arange(nx) + 0.5) * dx, rtol=1e-12)
    assert np.allclose(y[::nx], (np.arange(ny) + 0.5) * dx, rtol=1e-12)
    assert star[0] == 0.0 and star[2] == 0.0 and abs(star[1] / dx - (tp.star_position[1] + 0.5)) < 1e-9
