"""Generates the golden fixtures in tests/golden/ by running the reference.

Usage (needs the reference tree and oracle/_ref/torch_ref, i.e. this build
container):  python tests/golden/make_golden.py

For each case of tests/cases.py it writes <case>.npz holding the exact Lua
parameter text and initial-condition text the reference read, the number of
full steps, and the reference's final U, Q, R, T, T_min and dt history.  A
case set up by a Lua script (cases.LuaSetup: the reference's Torch::setUpLua
path, the only one that carries gravity) keeps the script text and the nine
values per cell that the reference's own Lua evaluation of it returned
(setup_vals [9][N]) instead of an initial-condition text.  For
the cases of CHECKPOINT_CASES it also keeps the reference's own checkpoint
files of the final state (DataPrinter::print2D and ::printHeating after
fillHeatingArrays) as ckpt_<case>_data2D.txt.gz and ckpt_<case>_heating.txt.gz.
"""
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import cases  # noqa: E402
import oracle  # noqa: E402
from torch_b200 import config  # noqa: E402


CHECKPOINT_CASES = ("blister_small", "hii3d_small")


def make(name):
    extra = {}
    with tempfile.TemporaryDirectory() as d:
        tp, ic, text, steps = cases.build(name, d)
        params = config.to_lua(tp)
        ppath = os.path.join(d, "params.lua")
        with open(ppath, "w") as f:
            f.write(params)
        if isinstance(ic, cases.LuaSetup):
            # initial state from the reference's own Lua evaluation of the setup
            spath, dump = os.path.join(d, "setup.lua"), os.path.join(d, "setup.bin")
            with open(spath, "w") as f:
                f.write(ic.text)
            ref = oracle.run_reference(ppath, None, steps, d, setup_path=spath, setup_dump=dump)
            extra = {"setup_lua": np.array(ic.text), "setup_vals": np.fromfile(dump).reshape(9, -1)}
            text = ""
        else:
            ref = oracle.run_reference(ppath, os.path.join(d, "ic_000.txt"), steps, d,
                                       print2d=d if name in CHECKPOINT_CASES else None)
        if name in CHECKPOINT_CASES:
            for kind in ("data2D", "heating"):
                shutil.copyfile(os.path.join(d, f"{kind}_final.txt.gz"),
                                os.path.join(HERE, f"ckpt_{name}_{kind}.txt.gz"))
    out = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(out, params_lua=np.array(params), ic_text=np.array(text), steps=np.array(steps),
                        U=ref.U, Q=ref.Q, R=ref.R, T=ref.T, Tmin=ref.Tmin, dts=ref.dts, time=np.array(ref.time),
                        **extra)
    print(f"{name}: {steps} steps, {ref.U.shape[1]} cells -> {os.path.relpath(out, ROOT)} "
          f"({os.path.getsize(out) // 1024} KiB)")


if __name__ == "__main__":
    for name in (sys.argv[1:] or list(cases.CASES)):
        make(name)
