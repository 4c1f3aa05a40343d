"""Host-side set-up of the library (runs before any CUDA call), checked on CPU:
parameter validation, wind cells, the first non-wind cell of the causal order
(the reference's one-off `once` time-step cell) and the shell order of the
sweeps, whose dependency check runs inside host_setup."""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

import common
import oracle
import torch_b200
from torch_b200 import workloads

SRC = os.path.join(common.ROOT, "torch_b200", "csrc", "setup.cpp")
HARNESS = os.path.join(common.HERE, "host_harness", "hs_check.cpp")


@pytest.fixture(scope="module")
def hs():
    d = tempfile.mkdtemp(prefix="trg_hs_")
    so = os.path.join(d, "hs.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-o", so, SRC, HARNESS],
                   check=True)
    lib = C.CDLL(so)
    lib.hs_check.restype = C.c_int
    lib.hs_check.argtypes = [C.POINTER(torch_b200.TrgParams)] + [C.c_void_p] * 6 + [C.c_char_p, C.c_int] + \
        [C.POINTER(C.c_longlong)] * 4
    return lib


def run(lib, tp, ic):
    p = torch_b200.make_params(tp, ic.side_length, ic.ncells)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (ic.den, ic.pre, ic.hii, ic.vel[0], ic.vel[1], ic.vel[2])]
    err = C.create_string_buffer(256)
    out = [C.c_longlong(0) for _ in range(4)]
    rc = lib.hs_check(C.byref(p), *[a.ctypes.data_as(C.c_void_p) for a in arrs], err, 256, *[C.byref(o) for o in out])
    return rc, err.value.decode(), [o.value for o in out]


@pytest.mark.parametrize("name", common.golden_names())
def test_sweep_order_valid_for_golden_cases(hs, name):
    tp, ic, _, _ = common.load_golden(name)
    rc, err, (ns_all, ns_nw, first, nwind) = run(hs, tp, ic)
    assert rc == 0, err
    assert ns_all >= 1 and ns_nw >= 1
    # the first non-wind cell agrees with the oracle's causal order
    o = oracle.Oracle(tp, ic)
    order = o.causal_order()
    assert first in order.tolist()


@pytest.mark.parametrize("make", [lambda: workloads.blister(), lambda: workloads.hii_region(n=64),
                                  lambda: workloads.sedov(n=48)])
def test_sweep_order_valid_for_workloads(hs, make):
    tp, ic = make()
    rc, err, (ns_all, _, first, nwind) = run(hs, tp, ic)
    assert rc == 0, err


def test_shell_count_centred_star(hs):
    tp, ic = workloads.hii_region(n=32)
    rc, err, (ns_all, ns_nw, first, nwind) = run(hs, tp, ic)
    assert rc == 0
    # centred star at cell 16: max-norm distances 0..16 cells in whole steps
    assert ns_all == 17 and nwind == 1


def test_rejects_unsupported_order(hs):
    import dataclasses
    tp, ic = workloads.sedov(n=8)
    rc, err, _ = run(hs, dataclasses.replace(tp, spatialOrder=2), ic)
    assert rc == 1 and "spatial_order" in err


def test_first_nonwind_cell_matches_oracle_config1(hs):
    tp, ic = workloads.blister()
    rc, err, (_, _, first, nwind) = run(hs, tp, ic)
    assert rc == 0
    o = oracle.Oracle(tp, ic)
    order = o.causal_order()
    # the reference's wind test (Fluid.cpp:41-53) on the causal order
    nx = ic.ncells[0]
    for cid in order:
        i, j = cid % nx, cid // nx
        d2 = (i - 0) * (i + 0.5 - 0) + (j - 110) * (j + 0.5 - 110)
        if not (d2 <= 100 or cid == 110 * nx):
            assert cid == first
            break
