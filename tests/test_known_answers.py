"""Known answers on the CPU: the exact Riemann solver of the test helpers
against the published Sod star state, and the oracle (the reference's
algorithm, bit-exact with the reference build) against the exact Sod
solution and against Spitzer's expansion law of an HII region - the
comparisons the reference's own analysis scripts make
(scripts/misc/sod.py, scripts/radiation-plots/spitzer-torch.py)."""
import numpy as np

import known_answers as ka
import oracle


def run_to(sim, tp, t_end):
    """Full steps until t_end (seconds), the last one cut to land on it;
    sim is the oracle or the library's Torch."""
    t_code = t_end / tp.tscale
    now = (lambda: sim.lib.orc_time(sim.ctx)) if isinstance(sim, oracle.Oracle) else \
        (lambda: sim.lib.trg_time(sim.ctx))
    while True:
        t = now()
        if t >= t_code * (1 - 1e-12):
            return sim.state()
        sim.full_step(t_code - t)


def test_exact_riemann_solver_gives_the_sod_star_state():
    # Sod's problem in units of the left state: p* = 0.30313 p_L, u* = 0.92745 sqrt(p_L / rho_L)
    p, u = ka.riemann_exact((1.0, 0.0, 1.0), (0.125, 0.0, 0.1), 1.4)
    assert abs(p - 0.30313) < 1e-5 and abs(u - 0.92745) < 1e-5
    # a symmetric collision: no velocity in the star region
    p2, u2 = ka.riemann_exact((1.0, 1.0, 1.0), (1.0, -1.0, 1.0), 1.4)
    assert abs(u2) < 1e-12 and p2 > 1.0


def sod_errors(st, tp, n):
    rho_e, _, p_e = ka.sod_exact_profile(n, st.time * tp.tscale)
    rho, p = st.Q[0] * tp.dscale, st.Q[1] * tp.pscale
    return (np.abs(rho - rho_e).sum() / np.abs(rho_e).sum(), np.abs(p - p_e).sum() / np.abs(p_e).sum())


def test_oracle_sod_converges_to_the_exact_solution():
    errs = []
    for n in (400, 800):
        tp, ic = ka.sod_case(n)
        o = oracle.Oracle(tp, ic)
        errs.append(sod_errors(run_to(o, tp, ka.sod_time()), tp, n))
        o.close()
    (r4, p4), (r8, p8) = errs
    assert r4 < 0.005 and p4 < 0.004  # measured 0.0032, 0.0023
    assert r8 < 0.65 * r4 and p8 < 0.65 * p4  # first order across the discontinuities


def spitzer_track(sim, tp, n, side_pc, marks=(2.0, 3.0, 4.0)):
    """I-front radii (units of R_S) at the given multiples of t_s, with the
    Spitzer radii there."""
    rs, ts = ka.stromgren_radius(), ka.stromgren_radius() / ka.ionised_sound_speed()
    dx = side_pc * ka.PC2CM / n
    out = []
    for m in marks:
        st = run_to(sim, tp, m * ts)
        out.append((ka.ifront_radius(st.Q[2], dx) / rs, ka.spitzer_radius(m * ts, rs, ts) / rs))
    return out


def test_oracle_hii_region_follows_spitzer_expansion():
    """1-D spherical HII region in uniform gas (n = 400 cm^-3, Q = 1e49 s^-1,
    TTI coupling 300 K / 8000 K): after the R-type phase the I-front follows
    R_S (1 + 7 t / 4 t_s)^(4/7), the more closely the later (the analytic
    law neglects the front's early transient)."""
    n, side = 200, 6.0
    tp, ic = ka.spitzer_case(n, side)
    o = oracle.Oracle(tp, ic)
    track = spitzer_track(o, tp, n, side)
    o.close()
    errs = [abs(r - s) / s for r, s in track]
    assert all(a < b for (a, _), (b, _) in zip(track, track[1:]))
    assert errs[0] < 0.045 and errs[1] < 0.03 and errs[2] < 0.025  # measured 0.034, 0.022, 0.016
