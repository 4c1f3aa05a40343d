"""Helpers shared by the tests: golden fixtures and field comparisons."""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLDEN = os.path.join(HERE, "golden")
for p in (ROOT, HERE, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

from torch_b200 import config  # noqa: E402

FIELD_NAMES = {
    "U": ["den", "energy", "rho_hii", "rho_adv", "mom0", "mom1", "mom2"],
    "Q": ["den", "pre", "hii", "adv", "vel0", "vel1", "vel2"],
    "R": ["hii_avg", "tau", "tau_avg", "dtau", "dtau_avg", "heat"],
    "T": ["col_den", "dcol_den", "heat", "rate"],
}


def golden_names():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


def load_golden(name):
    """Returns (tp, ic, steps, arrays) for tests/golden/<name>.npz."""
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    tp = config.parse_parameters(str(z["params_lua"]))
    if "setup_lua" in z:
        # Lua-setup case: the reference's own evaluation of the script, cgs
        v = z["setup_vals"]
        ic = config.make_initial_conditions(tuple(tp.ncells), tp.sideLength / tp.ncells[0], v[0], v[1], v[2],
                                            v[3:6].copy())
        ic.side_length = tp.sideLength
        ic.grav = v[6:9].copy()
    else:
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "ic_000.txt")
            with open(path, "w") as f:
                f.write(str(z["ic_text"]))
            ic = config.read_initial_conditions(path)
    arrays = {k: z[k] for k in ("U", "Q", "R", "T", "Tmin", "dts", "time")}
    return tp, ic, int(z["steps"]), arrays


def inplane(group: str, f: int, nd: int) -> bool:
    """Velocity/momentum components beyond nd are not part of the solution
    (the reference leaves them uninitialised in 2-D, Riemann.cpp:212-228)."""
    if group in ("U", "Q") and f >= 4:
        return f - 4 < nd
    return True


def rel_l1(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).sum()
    num = np.abs(a - b).sum()
    if den == 0:
        return 0.0 if num == 0 else float("inf")
    return float(num / den)


def compare_states(got: dict, ref: dict, nd: int, groups=("U", "Q", "R", "T")):
    """Per-field relative L1 error of got against ref: {(group, name): err}."""
    out = {}
    for g in groups:
        for f in range(ref[g].shape[0]):
            if not inplane(g, f, nd):
                continue
            out[(g, FIELD_NAMES[g][f])] = rel_l1(got[g][f], ref[g][f])
    return out


def state_dict(s):
    return {"U": s.U, "Q": s.Q, "R": s.R, "T": s.T, "Tmin": s.Tmin}


def ifront_cells(hii, n):
    """I-front distance (cells) from a star at the centre of an n^3 grid along
    +x: the first cell with HII < 0.5, linearly interpolated (the rule of the
    reference's scripts/misc/calc_if.py:43-56)."""
    x = np.asarray(hii).reshape(n, n, n)[n // 2, n // 2, n // 2:]
    for i in range(1, len(x)):
        if x[i] < 0.5:
            return (i - 1) + (x[i - 1] - 0.5) / (x[i - 1] - x[i])
    return float(len(x))
