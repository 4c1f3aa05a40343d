"""Known-answer problems for the hydrodynamics and the radiation transfer
(no golden vectors exist for them in the reference; its analysis scripts
compare runs with the same closed forms):

* the Sod shock tube against the exact solution of the Riemann problem for an
  ideal gas (restated here from the published method: the star-region
  pressure is the root of f_L(p) + f_R(p) + (u_R - u_L) = 0, with the shock
  and rarefaction branches of f_K, found by Newton iteration; the solution is
  then sampled at x / t);
* the D-type expansion of an HII region in uniform gas (the reference's
  scripts/radiation-plots/spitzer-torch.py compares its runs with Spitzer's
  R(t) = R_S (1 + 7 t / (4 t_s))^(4/7) and Raga's variant with the factor
  sqrt(4/3); R_S = (3 Q / (4 pi n^2 alpha_B))^(1/3), t_s = R_S / c_i), with
  the I-front radius taken as scripts/misc/calc_if.py does: the first cell
  along the ray whose HII fraction drops below 0.5, interpolated linearly
  with the cell before it.

Used by tests/test_known_answers.py (the oracle, CPU) and
tests/test_gpu_known_answers.py (the CUDA path)."""
import dataclasses
import math

import numpy as np

from torch_b200 import config, workloads

PC2CM = workloads.PC2CM
M_H = 1.674e-24        # the reference's hydrogen mass (Constants)
R_GAS = 8.314462e7     # its specific gas constant (erg / K / mol)


# ------------------------------------------------------------------- Sod
def _f_branch(p, rho, pk, gamma):
    """Pressure function of one side and its derivative: a shock where p > pk,
    a rarefaction where p <= pk."""
    c = math.sqrt(gamma * pk / rho)
    if p > pk:
        a = 2.0 / ((gamma + 1.0) * rho)
        b = (gamma - 1.0) / (gamma + 1.0) * pk
        q = math.sqrt(a / (p + b))
        return (p - pk) * q, q * (1.0 - 0.5 * (p - pk) / (p + b))
    e = (gamma - 1.0) / (2.0 * gamma)
    return 2.0 * c / (gamma - 1.0) * ((p / pk) ** e - 1.0), (p / pk) ** (-(gamma + 1.0) / (2.0 * gamma)) / (rho * c)


def riemann_exact(left, right, gamma):
    """Star-region pressure and velocity of the Riemann problem
    left = (rho, u, p), right = (rho, u, p)."""
    (rl, ul, pl), (rr, ur, pr) = left, right
    p = 0.5 * (pl + pr)
    for _ in range(100):
        fl, dl = _f_branch(p, rl, pl, gamma)
        fr, dr = _f_branch(p, rr, pr, gamma)
        step = (fl + fr + ur - ul) / (dl + dr)
        p_new = max(p - step, 1e-12 * p)
        if abs(p_new - p) <= 1e-14 * p_new:
            p = p_new
            break
        p = p_new
    fl, _ = _f_branch(p, rl, pl, gamma)
    fr, _ = _f_branch(p, rr, pr, gamma)
    return p, 0.5 * (ul + ur) + 0.5 * (fr - fl)


def sample_exact(s, left, right, gamma):
    """(rho, u, p) of the exact solution at similarity coordinate s = x / t."""
    (rl, ul, pl), (rr, ur, pr) = left, right
    ps, us = riemann_exact(left, right, gamma)
    g1, g2 = (gamma - 1.0) / (gamma + 1.0), (gamma - 1.0) / (2.0 * gamma)
    if s <= us:  # left of the contact
        cl = math.sqrt(gamma * pl / rl)
        if ps > pl:  # left shock
            sl = ul - cl * math.sqrt((gamma + 1.0) / (2.0 * gamma) * ps / pl + g2)
            return (rl, ul, pl) if s <= sl else (rl * (ps / pl + g1) / (g1 * ps / pl + 1.0), us, ps)
        cs = cl * (ps / pl) ** g2
        if s <= ul - cl:
            return rl, ul, pl
        if s >= us - cs:
            return rl * (ps / pl) ** (1.0 / gamma), us, ps
        u = 2.0 / (gamma + 1.0) * (cl + 0.5 * (gamma - 1.0) * ul + s)
        c = 2.0 / (gamma + 1.0) * (cl + 0.5 * (gamma - 1.0) * (ul - s))
        rho = rl * (c / cl) ** (2.0 / (gamma - 1.0))
        return rho, u, pl * (c / cl) ** (2.0 * gamma / (gamma - 1.0))
    cr = math.sqrt(gamma * pr / rr)
    if ps > pr:  # right shock
        sr = ur + cr * math.sqrt((gamma + 1.0) / (2.0 * gamma) * ps / pr + g2)
        return (rr, ur, pr) if s >= sr else (rr * (ps / pr + g1) / (g1 * ps / pr + 1.0), us, ps)
    cs = cr * (ps / pr) ** g2
    if s >= ur + cr:
        return rr, ur, pr
    if s <= us + cs:
        return rr * (ps / pr) ** (1.0 / gamma), us, ps
    u = 2.0 / (gamma + 1.0) * (-cr + 0.5 * (gamma - 1.0) * ur + s)
    c = 2.0 / (gamma + 1.0) * (cr - 0.5 * (gamma - 1.0) * (ur - s))
    rho = rr * (c / cr) ** (2.0 / (gamma - 1.0))
    return rho, u, pr * (c / cr) ** (2.0 * gamma / (gamma - 1.0))


SOD_LEFT = (1.0e-20, 0.0, 1.0e-10)    # rho [g/cm^3], u [cm/s], p [dyn/cm^2]
SOD_RIGHT = (0.125e-20, 0.0, 1.0e-11)
SOD_GAMMA = 1.4


def sod_case(n: int, riemann="HLLC", limiter="albada"):
    """1-D Sod shock tube on n cells over 1 pc, the diaphragm in the middle."""
    tp = workloads.sedov_parameters(n=n, nd=1, riemann=riemann, limiter=limiter, side=PC2CM)
    tp = dataclasses.replace(tp, heatCapacityRatio=SOD_GAMMA, star_position=(0, 0, 0), tscale=1.0e11)
    dx = PC2CM / n
    left = np.arange(n) < n // 2
    den = np.where(left, SOD_LEFT[0], SOD_RIGHT[0])
    pre = np.where(left, SOD_LEFT[2], SOD_RIGHT[2])
    ic = config.make_initial_conditions((n, 1, 1), dx, den, pre, np.zeros(n), np.zeros((3, n)))
    return tp, ic


def sod_time():
    """End time of the Sod runs: 0.2 of the tube's length crossed at the left sound speed."""
    return 0.2 * PC2CM / math.sqrt(SOD_GAMMA * SOD_LEFT[2] / SOD_LEFT[0])


def sod_exact_profile(n: int, t: float):
    x = (np.arange(n) + 0.5) / n * PC2CM - 0.5 * PC2CM
    out = np.array([sample_exact(xi / t, SOD_LEFT, SOD_RIGHT, SOD_GAMMA) for xi in x])
    return out[:, 0], out[:, 1], out[:, 2]


# -------------------------------------------------------------- Spitzer
SPITZER_N = 400.0       # hydrogen number density [cm^-3]
SPITZER_Q = 1.0e49      # ionising photons per second
SPITZER_ALPHA_B = 2.59e-13
SPITZER_TI, SPITZER_TN = 8000.0, 300.0  # ionised and neutral temperatures (TTI coupling)


def stromgren_radius():
    return (3.0 * SPITZER_Q / (4.0 * math.pi * SPITZER_N ** 2 * SPITZER_ALPHA_B)) ** (1.0 / 3.0)


def ionised_sound_speed():
    """Isothermal sound speed of the ionised gas at T_i (mean mass per
    particle m_H / 2): the D-type front is driven by its pressure."""
    return math.sqrt(2.0 * R_GAS * SPITZER_TI)


def spitzer_radius(t, rs, ts):
    return rs * (1.0 + 7.0 * t / (4.0 * ts)) ** (4.0 / 7.0)


def raga_radius(t, rs, ts):
    return rs * (1.0 + 7.0 * math.sqrt(4.0 / 3.0) * t / (4.0 * ts)) ** (4.0 / 7.0)


def spitzer_case(n: int, side_pc: float):
    """1-D spherical HII region: uniform neutral hydrogen at SPITZER_N and
    SPITZER_TN, the star at the origin (face-snapped), TTI coupling between
    SPITZER_TN and SPITZER_TI, no cooling, n cells over side_pc parsecs."""
    tp = workloads.hii_region_parameters(n=n, side=side_pc * PC2CM, photon_rate=SPITZER_Q)
    tp = dataclasses.replace(tp, nd=1, ncells=(n, 1, 1), geometry="spherical", cooling_on=False,
                             rt_coupling="tti", THI=SPITZER_TN, THII=SPITZER_TI, alphaB=SPITZER_ALPHA_B,
                             star_position=(0, 0, 0), faceSnap=(True, False, False),
                             leftBC=("reflecting",) * 3, rightBC=("outflow",) * 3, tmax=1.0e15)
    dx = side_pc * PC2CM / n
    rho = SPITZER_N * M_H
    pre = rho * R_GAS * SPITZER_TN  # neutral: mean mass per particle m_H
    ic = config.make_initial_conditions((n, 1, 1), dx, np.full(n, rho), np.full(n, pre), np.zeros(n),
                                        np.zeros((3, n)))
    return tp, ic


def ifront_radius(hii: np.ndarray, dx: float) -> float:
    """I-front radius along the ray (cell centres (i + 1/2) dx from the
    star at the origin): the first cell with HII < 0.5, interpolated with the
    one before it (calc_if.py:43-56)."""
    xi = (np.arange(hii.size) + 0.5) * dx
    below = np.nonzero(hii < 0.5)[0]
    if below.size == 0 or below[0] == 0:
        return 0.0
    i = below[0]
    f = (0.5 - hii[i - 1]) / (hii[i] - hii[i - 1])
    return xi[i - 1] + f * (xi[i] - xi[i - 1])
