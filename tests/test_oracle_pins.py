"""Pins of the oracle's MUSCL and HLLC paths.

The reference committed no run of its MUSCL linear-Riemann solver
(Taylor_Green_Vortex/Solver_Normalized_MUSCL_Linear_Riemann_Delta_SPS.f90) nor of
its HLLC solver (Moving_Square_Or_Cylinder_Inside_a_Rectangular_Box/
Solver_Normalized_HLLC_Riemann_Delta.f90), so their restatements are tied here
to what is pinned or published:

* MUSCL: with the reconstruction gradients forced to zero, every limiter call
  returns zero increments and the MUSCL solver's Riemann states are the
  unreconstructed ones, so its rates must equal, bit for bit, those of the
  modified linear-Riemann solver (Solver_Normalized_Modified_Linear_Riemann_Delta_SPS.f90:
  305-363), whose restatement is pinned by the reference's own Taylor-Green
  output (tests/test_oracle.py).  The limiter (Taylor_Green_Vortex/
  function_module.f90:34-80) is pinned by known answers worked out by hand from
  its source text, one per branch.
* HLLC: the pair state is compared with an independent implementation, written
  here from E. F. Toro, "Riemann Solvers and Numerical Methods for Fluid
  Dynamics" (3rd ed., Springer 2009): the acoustic (linearised) star state from
  the Riemann invariants (ch. 9), the HLLC star states rho*_K = rho_K (S_K - u_K)
  / (S_K - S*) with the tangential velocity carried across the contact and the
  four-region sampling (ch. 10), Davis' and the pressure-based wave-speed
  estimates (ch. 10), the latter with the shock factor of the Rankine-Hugoniot
  condition of the barotropic equations, (S - u_K)^2 = (rho*/rho_K)(p* - p_K) /
  (rho* - rho_K).  The comparison shows two properties of the reference's HLLC,
  both reproduced by the oracle and the GPU:
    - its contact speed weights each side's velocity with the OTHER side's
      acoustic impedance, (C_R u_L + C_L u_R + p_L - p_R)/(C_L + C_R), where the
      invariants give (C_L u_L + C_R u_R + p_L - p_R)/(C_L + C_R); the two agree
      when C_L = C_R;
    - its shock branch (:243-275) is taken only when p* > p_K and rho_K > rho*,
      which a monotone equation of state never satisfies together, so for
      states whose pressure follows their density the wave speeds are Davis'
      S_L = u_L - c_L, S_R = u_R + c_R.
"""
import math

import numpy as np
import pytest

import sph_b200 as S


# ---------------------------------------------------------------------------
# MUSCL
# ---------------------------------------------------------------------------
# (di, dj, dij) -> (li, lj), evaluated by hand from MUSCL_Limiter's source text
# (beta_lim = 1.3, diff_factor = 0.5).
LIMITER_KAT = [
    # dj > 0, lim = max(0, min(1.3di, dj), min(di, 1.3dj)) = 0.39 > dij/2, di < dj: j side gets dij/2
    ((0.3, 0.5, 0.2), (0.0, 0.1)),
    # dj > 0, lim = 0.6 > dij/2, di > dj: i side gets dij/2
    ((0.6, 0.5, 0.2), (0.1, 0.0)),
    # dj > 0, lim = 0.05 <= dij/2: both sides get lim
    ((0.05, 0.04, 1.0), (0.05, 0.05)),
    # dj <= 0, lim = min(0, max(1.3di, dj), max(di, 1.3dj)) = -0.39 < dij/2, di > dj: j side gets dij/2
    ((-0.3, -0.5, -0.2), (0.0, -0.1)),
    # dj <= 0, lim = -0.6 < dij/2, di < dj: i side gets dij/2
    ((-0.6, -0.5, -0.2), (-0.1, 0.0)),
    # dj <= 0, lim = -0.05 >= dij/2 = -0.5: both sides get lim
    ((-0.05, -0.04, -1.0), (-0.05, -0.05)),
    # opposite signs (a linear field: di = dij/2, dj = -dij/2): lim = 0, no reconstruction
    ((0.5, -0.5, 1.0), (0.0, 0.0)),
    ((-0.5, 0.5, -1.0), (0.0, 0.0)),
    # zero gradients
    ((0.0, 0.0, 0.7), (0.0, 0.0)),
]


@pytest.mark.parametrize("args,expect", LIMITER_KAT)
def test_muscl_limiter_known_answers(oracle, args, expect):
    li, lj = oracle.muscl_limiter(*args)
    assert li == pytest.approx(expect[0], abs=1e-15)
    assert lj == pytest.approx(expect[1], abs=1e-15)


@pytest.mark.parametrize("case_kw", [
    dict(n_side=64, jitter=0.1, seed=1),
    dict(n_side=48, jitter=0.1, seed=2),
])
@pytest.mark.parametrize("renorm", [0, 1])
def test_muscl_without_gradients_is_the_modified_solver(oracle, case_kw, renorm):
    """Zero reconstruction gradients: MUSCL rates == modified linear-Riemann rates, bit for bit."""
    muscl = S.make_tgv(solver=S.SOLVER_MUSCL_DELTA_SPS, **case_kw)
    modlr_cfg = muscl.cfg.copy()
    modlr_cfg.solver = S.SOLVER_MODLR_DELTA_SPS
    cfg = muscl.cfg.copy()
    cfg.renormalize = renorm
    modlr_cfg.renormalize = renorm
    args = (muscl.pos, muscl.vel, muscl.rho, muscl.mass, muscl.type)
    try:
        oracle.set_muscl_gradient_scale(0.0)
        m0 = oracle.rhs(cfg, *args)
    finally:
        oracle.set_muscl_gradient_scale(1.0)
    m1 = oracle.rhs(cfg, *args)
    ref = oracle.rhs(modlr_cfg, *args)
    for k in ("drhodt", "acc", "fs", "near", "fra_v", "binv", "tau"):
        assert np.array_equal(m0[k], ref[k]), k
    # grad rho (the delta-SPH term) is the same sum in both solvers
    assert np.array_equal(m0["grads"][:2 * muscl.n], ref["grads"][:2 * muscl.n])
    # with its gradients the MUSCL solver reconstructs: the rates differ
    assert not np.array_equal(m1["acc"], ref["acc"])
    rel = np.linalg.norm(m1["acc"] - ref["acc"]) / np.linalg.norm(ref["acc"])
    assert 1e-8 < rel < 0.5


# ---------------------------------------------------------------------------
# HLLC
# ---------------------------------------------------------------------------
def toro_hllc(vl, vr, e, rl, rr, cl, cr, pl, pr, c0sq, rho0, pb, wave_speeds="davis", contact="invariants"):
    """HLLC state sampled at x/t = the mean normal velocity, for the barotropic
    equations with the linear equation of state p = c0^2 (rho - rho0) + pb.
    wave_speeds: "davis" (S_L = u_L - c_L, S_R = u_R + c_R) or "pressure" (the
    pressure-based estimate, q_K = 1 for a rarefaction p* <= p_K, else the
    Rankine-Hugoniot factor).  contact: "invariants" (u* from the acoustic
    Riemann invariants) or "reference" (each velocity weighted with the other
    side's impedance).  Returns (v*, P*, region) with region 0..3 = L, L*, R*, R."""
    n = np.array(e, np.float64)
    t = np.array([-n[1], n[0]])
    ul, tl = float(np.dot(vl, n)), float(np.dot(vl, t))
    ur, tr = float(np.dot(vr, n)), float(np.dot(vr, t))
    Cl, Cr = rl * cl, rr * cr
    # Riemann invariants across the acoustic waves: p* + C_L u* = p_L + C_L u_L,
    # p* - C_R u* = p_R - C_R u_R
    p_star = (Cr * pl + Cl * pr + Cl * Cr * (ul - ur)) / (Cl + Cr)
    if contact == "invariants":
        u_star = (Cl * ul + Cr * ur + pl - pr) / (Cl + Cr)
    else:
        u_star = (Cr * ul + Cl * ur + pl - pr) / (Cl + Cr)
    rho_star = rho0 + (p_star - pb) / c0sq

    def q(pk, rk, ck):
        if wave_speeds == "davis" or p_star <= pk:
            return 1.0
        return math.sqrt((rho_star / rk) * (p_star - pk) / (rho_star - rk)) / ck

    sl = ul - cl * q(pl, rl, cl)
    sr = ur + cr * q(pr, rr, cr)
    xi = 0.5 * (ul + ur)
    if sl > xi:
        region, rh, un, ut = 0, rl, ul, tl
    elif u_star >= xi:
        region, rh, un, ut = 1, rl * (sl - ul) / (sl - u_star), u_star, tl
    elif sr >= xi:
        region, rh, un, ut = 2, rr * (sr - ur) / (sr - u_star), u_star, tr
    else:
        region, rh, un, ut = 3, rr, ur, tr
    v = un * n + ut * t
    return v, c0sq * (rh - rho0) + pb, region


def _ms_cfg():
    return S.moving_square_config(0.02, 4.0, 2.0, S.SOLVER_MS_HLLC_DELTA)


def _eos(cfg, rho):
    """The linear equation of state and sound speed c0 (rho/rho0)^3 of status_equation."""
    p = cfg.c0sq * (rho - cfg.rho0) + cfg.background_p
    c = math.sqrt(cfg.c0sq) * (rho / cfg.rho0) ** 3
    return p, c


def _random_pair(rng, cfg, equal_impedance, ujump, spread=0.02):
    rl, rr = cfg.rho0 * rng.uniform(1.0 - spread, 1.0 + spread, 2)
    pl, cl = _eos(cfg, rl)
    pr, cr = _eos(cfg, rr)
    if equal_impedance:
        cl = math.sqrt(cfg.c0sq) * rng.uniform(0.9, 1.1)
        cr = rl * cl / rr
    ang = rng.uniform(0, 2 * math.pi)
    e = np.array([math.cos(ang), math.sin(ang)])
    t = np.array([-e[1], e[0]])
    ul, ur = rng.uniform(-ujump, ujump, 2)
    tl, tr = rng.uniform(-2.0, 2.0, 2)
    return ul * e + tl * t, ur * e + tr * t, e, rl, rr, cl, cr, pl, pr


def _compare(oracle, cfg, args, **kw):
    vs, ps = oracle.hllc_state(cfg, *args)
    v, p, region = toro_hllc(*args, cfg.c0sq, cfg.rho0, cfg.background_p, **kw)
    scale = max(1.0, np.abs(v).max())
    return np.abs(vs - v).max() / scale, abs(ps - p) / max(1.0, abs(p)), region


def test_hllc_equal_impedance_states_match_toro(oracle):
    """C_L = C_R: the contact speeds agree; states over all four sampled regions."""
    cfg = _ms_cfg()
    rng = np.random.default_rng(11)
    hits = np.zeros(4, int)
    for _ in range(4000):
        # a wide density spread so that c_R < (u_L - u_R)/2 <= c_L (region R) occurs
        args = _random_pair(rng, cfg, equal_impedance=True, ujump=30.0, spread=0.2)
        ev, ep, region = _compare(oracle, cfg, args, wave_speeds="davis", contact="invariants")
        assert ev < 1e-13 and ep < 1e-12, (args, ev, ep)
        hits[region] += 1
    assert (hits >= 25).all(), hits


def test_hllc_rarefactions_match_toro_pressure_based_speeds(oracle):
    """Both waves rarefactions (p* <= p_L, p_R): Toro's pressure-based wave speeds
    are the acoustic ones, and the reference's state equals Toro's."""
    cfg = _ms_cfg()
    rng = np.random.default_rng(12)
    seen = 0
    for _ in range(4000):
        args = _random_pair(rng, cfg, equal_impedance=True, ujump=30.0)
        vl, vr, e, rl, rr, cl, cr, pl, pr = args
        ul, ur = np.dot(vl, e), np.dot(vr, e)
        Cl, Cr = rl * cl, rr * cr
        p_star = (Cr * pl + Cl * pr + Cl * Cr * (ul - ur)) / (Cl + Cr)
        if p_star > min(pl, pr):
            continue
        seen += 1
        ev, ep, _ = _compare(oracle, cfg, args, wave_speeds="pressure", contact="invariants")
        assert ev < 1e-13 and ep < 1e-12
    assert seen > 500


def test_hllc_contact_speed_uses_the_opposite_impedance(oracle):
    """Unequal impedances (EOS-consistent states): the reference's contact speed
    is (C_R u_L + C_L u_R + p_L - p_R)/(C_L + C_R), not the invariants' value."""
    cfg = _ms_cfg()
    rng = np.random.default_rng(13)
    max_gap = 0.0
    for _ in range(3000):
        args = _random_pair(rng, cfg, equal_impedance=False, ujump=3.0)
        ev, ep, _ = _compare(oracle, cfg, args, wave_speeds="davis", contact="reference")
        assert ev < 1e-13 and ep < 1e-12
        gv, gp, region = _compare(oracle, cfg, args, wave_speeds="davis", contact="invariants")
        if region in (1, 2):
            max_gap = max(max_gap, gv, gp)
    # the two weightings differ by (C_R - C_L)(u_L - u_R)/(C_L + C_R) in the contact speed
    assert max_gap > 1e-6


def test_hllc_shock_branch_is_unreachable_for_consistent_states(oracle):
    """Compression (p* > p_K) with the pressure following the density: the guard
    rho_K > rho* never holds, so the reference keeps q_K = 1 (Davis' speeds)
    where the Rankine-Hugoniot factor would widen the fan."""
    cfg = _ms_cfg()
    rng = np.random.default_rng(14)
    shocks = 0
    for _ in range(3000):
        args = _random_pair(rng, cfg, equal_impedance=False, ujump=3.0)
        vl, vr, e, rl, rr, cl, cr, pl, pr = args
        ul, ur = np.dot(vl, e), np.dot(vr, e)
        Cl, Cr = rl * cl, rr * cr
        p_star = (Cr * pl + Cl * pr + Cl * Cr * (ul - ur)) / (Cl + Cr)
        rho_star = cfg.rho0 + (p_star - cfg.background_p) / cfg.c0sq
        for pk, rk in ((pl, rl), (pr, rr)):
            if p_star > pk:
                shocks += 1
                assert not rk > rho_star
        ev, ep, _ = _compare(oracle, cfg, args, wave_speeds="davis", contact="reference")
        assert ev < 1e-13 and ep < 1e-12
    assert shocks > 1000
