"""Accuracy of the IEEE-only exp/log/log10/pow of torch_b200/csrc/trg_math.h
(the FP64 kernels' transcendentals) against the host libm."""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

import common

HDR = os.path.join(common.ROOT, "torch_b200", "csrc", "trg_math.h")
SRC = r"""
#include "%s"
double f_exp(double x) { return trg_exp(x); }
double f_log(double x) { return trg_log(x); }
double f_log10(double x) { return trg_log10(x); }
double f_pow(double x, double y) { return trg_pow(x, y); }
""" % HDR


@pytest.fixture(scope="module")
def lib():
    d = tempfile.mkdtemp(prefix="trg_math_")
    src = os.path.join(d, "m.c")
    with open(src, "w") as f:
        f.write(SRC)
    so = os.path.join(d, "m.so")
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-o", so, src], check=True)
    L = C.CDLL(so)
    for n in ("f_exp", "f_log", "f_log10"):
        getattr(L, n).restype = C.c_double
        getattr(L, n).argtypes = [C.c_double]
    L.f_pow.restype = C.c_double
    L.f_pow.argtypes = [C.c_double, C.c_double]
    return L


def ulp_err(a, b):
    b = np.asarray(b)
    return np.abs(np.asarray(a) - b) / np.abs(np.spacing(b))


def test_exp_log_accuracy(lib):
    rng = np.random.default_rng(0)
    x = rng.uniform(-700, 700, 20000)
    assert ulp_err([lib.f_exp(v) for v in x], np.exp(x)).max() <= 1.0
    y = np.exp(rng.uniform(-690, 690, 20000))
    assert ulp_err([lib.f_log(v) for v in y], np.log(y)).max() <= 2.0
    assert ulp_err([lib.f_log10(v) for v in y], np.log10(y)).max() <= 2.0
    b = rng.uniform(1e-3, 1e3, 20000)
    p = rng.uniform(-3, 3, 20000)
    assert ulp_err([lib.f_pow(u, v) for u, v in zip(b, p)], np.power(b, p)).max() <= 64.0


def test_special_values(lib):
    assert lib.f_exp(0.0) == 1.0 and lib.f_log(1.0) == 0.0
    assert lib.f_exp(-800.0) == 0.0 and np.isinf(lib.f_exp(800.0))
    assert np.isnan(lib.f_log(-1.0)) and np.isinf(lib.f_log(0.0))
    assert lib.f_pow(2.0, 0.0) == 1.0 and lib.f_pow(0.0, 1.6) == 0.0
    assert lib.f_exp(-740.0) > 0  # subnormal range
