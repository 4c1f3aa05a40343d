"""The FP64 form's exp/log/log10/pow (torch_b200/csrc/trg_math.h): correct
rounding against quad-precision values (libquadmath), and how often they
differ from the host glibc (the reference's libm) over the argument ranges
the radiation and cooling step uses."""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

import common

HDR = os.path.join(common.ROOT, "torch_b200", "csrc", "trg_math.h")
SRC = r"""
#include <quadmath.h>
#include "%s"
void v_trg(int f, const double* x, const double* y, double* out, long n) {
    for (long i = 0; i < n; ++i)
        out[i] = f == 0 ? trg_exp(x[i]) : f == 1 ? trg_log(x[i]) : f == 2 ? trg_log10(x[i]) : trg_pow(x[i], y[i]);
}
void v_libm(int f, const double* x, const double* y, double* out, long n) {
    for (long i = 0; i < n; ++i)
        out[i] = f == 0 ? exp(x[i]) : f == 1 ? log(x[i]) : f == 2 ? log10(x[i]) : pow(x[i], y[i]);
}
/* (exact value - d) in ulps of d, the exact value from quad precision */
void v_err(int f, const double* x, const double* y, const double* d, double* out, long n) {
    for (long i = 0; i < n; ++i) {
        __float128 X = x[i], Y = y[i];
        __float128 r = f == 0 ? expq(X) : f == 1 ? logq(X) : f == 2 ? log10q(X) : powq(X, Y);
        double a = fabs(d[i]);
        double u = a < 0x1p-1022 ? 0x1p-1074 : nextafter(a, INFINITY) - a;
        out[i] = (double)((r - (__float128)d[i]) / (__float128)u);
    }
}
double f1(int f, double x, double y) { double o; v_trg(f, &x, &y, &o, 1); return o; }
""" % HDR


@pytest.fixture(scope="module")
def lib():
    d = tempfile.mkdtemp(prefix="trg_math_")
    src = os.path.join(d, "m.c")
    with open(src, "w") as f:
        f.write(SRC)
    so = os.path.join(d, "m.so")
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-o", so, src, "-lquadmath", "-lm"],
                   check=True)
    L = C.CDLL(so)
    for n in ("v_trg", "v_libm"):
        getattr(L, n).argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_long]
    L.v_err.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_long]
    L.f1.restype = C.c_double
    L.f1.argtypes = [C.c_int, C.c_double, C.c_double]
    return L


def _run(L, fn, f, x, y):
    out = np.zeros(len(x))
    getattr(L, fn)(f, x.ctypes.data, y.ctypes.data, out.ctypes.data, len(x))
    return out


def _err(L, f, x, y, d):
    out = np.zeros(len(x))
    L.v_err(f, x.ctypes.data, y.ctypes.data, d.ctypes.data, out.ctypes.data, len(x))
    return out


def cases(n, seed):
    rng = np.random.default_rng(seed)
    return [
        ("exp", 0, "x in [-745, 709.7]", rng.uniform(-745, 709.7, n), None),
        ("exp", 0, "x in [-745.2, -708] (subnormal results)", rng.uniform(-745.2, -708, n), None),
        ("exp", 0, "x in [-1, 1]", rng.uniform(-1, 1, n), None),
        ("log", 1, "x log-uniform in [1e-300, 1e300]", 10 ** rng.uniform(-300, 300, n), None),
        ("log", 1, "x in [0.98, 1.02]", rng.uniform(0.98, 1.02, n), None),
        ("log10", 2, "T log-uniform in [1, 1e9] (spline abscissae)", 10 ** rng.uniform(0, 9, n), None),
        ("pow", 3, "x log-uniform in [1e-3, 1e6], y in [-3, 3]", 10 ** rng.uniform(-3, 6, n), rng.uniform(-3, 3, n)),
        ("pow", 3, "(1e-5 T)^1.63, T in [1, 1e9]", 1e-5 * 10 ** rng.uniform(0, 9, n), np.full(n, 1.63)),
    ]


def test_exp_log_pow_are_correctly_rounded(lib):
    """exp, log and pow round to nearest (error at most half an ulp of the
    quad-precision value) on every sample; log10 follows the classical
    reduction n log10(2) + log(m)/ln 10 (two roundings after the correctly
    rounded log), so it is held to its own bound of 2 ulp."""
    for name, f, what, x, y in cases(200_000, 7):
        x = np.ascontiguousarray(x)
        y = np.ascontiguousarray(np.zeros(len(x)) if y is None else y)
        a = _run(lib, "v_trg", f, x, y)
        e = np.abs(_err(lib, f, x, y, a))
        print(f"{name:6s} {what:48s} max error {e.max():.6f} ulp")
        assert e.max() <= (2.0 if name == "log10" else 0.5 + 1e-6), (name, what)


def test_where_the_math_differs_from_glibc(lib):
    """How often trg_math.h (the FP64 kernels' exp/log/log10/pow) and the host
    glibc return different doubles over the step's argument ranges, and that
    every difference is a case where glibc is not correctly rounded (its
    error above half an ulp) - i.e. the two agree wherever glibc rounds
    correctly.  The fractions are the ones quoted in the design notes; at
    this rate the reference's step (which amplifies single-ulp differences)
    stays within 1e-10 of the FP64 form for 100 steps of the shipped setup
    (tests/test_oracle.py)."""
    for name, f, what, x, y in cases(200_000, 42):
        x = np.ascontiguousarray(x)
        y = np.ascontiguousarray(np.zeros(len(x)) if y is None else y)
        a = _run(lib, "v_trg", f, x, y)
        b = _run(lib, "v_libm", f, x, y)
        diff = a != b
        frac = float(np.mean(diff))
        eb = np.abs(_err(lib, f, x, y, b))
        print(f"{name:6s} {what:48s} differing {frac:.2e}  glibc not correctly rounded {np.mean(eb > 0.5):.2e}")
        assert frac <= 2e-3, (name, what)
        if name != "log10":
            assert np.all(eb[diff] > 0.5), (name, what)


def test_special_values(lib):
    f = lib.f1
    assert f(0, 0.0, 0) == 1.0 and f(1, 1.0, 0) == 0.0 and f(2, 1.0, 0) == 0.0
    assert f(0, -800.0, 0) == 0.0 and np.isinf(f(0, 800.0, 0))
    assert f(0, -745.0, 0) == 5e-324 and f(0, -740.0, 0) > 0
    assert f(0, 709.78, 0) == np.exp(709.78) and np.isinf(f(0, 709.7828, 0))
    assert np.isnan(f(1, -1.0, 0)) and np.isinf(f(1, 0.0, 0)) and np.isinf(f(1, np.inf, 0))
    assert f(1, 5e-324, 0) == np.log(5e-324) and f(2, 1e-310, 0) == np.log10(1e-310)
    assert f(2, 1000.0, 0) == 3.0 and f(2, 1e-5, 0) == -5.0
    assert f(3, 2.0, 0.0) == 1.0 and f(3, 0.0, 1.6) == 0.0 and f(3, 4.0, 0.5) == 2.0
    assert f(3, -2.0, 3.0) == -8.0 and np.isnan(f(3, -2.0, 0.5))
    assert np.isnan(f(0, np.nan, 0)) and np.isnan(f(3, np.nan, 2.0))
