"""The moving-square tangent-linear model (oracle/sph_tangent.cpp,
oracle_tangent_ms), the CPU reference of the moving-square adjoint: its value
path must reproduce the oracle's Euler predictor-corrector steps with ghost
assignment and a per-step body motion (final kinetic energy and the drag
impulse), with and without the particle shift after the corrector and the
density re-initialisation (orders 1, 3 and 6, every second step), and its directional derivatives must match central differences of
its own value path."""
import numpy as np
import pytest

import sph_b200 as S

NSTEPS = 5


SOLVERS = [S.SOLVER_MS_MODLR_DELTA, S.SOLVER_MS_HLLC_DELTA]


def _case(solver=S.SOLVER_MS_MODLR_DELTA, shifting=0, mls_order=0):
    case, ity = S.make_moving_square(dx=0.1, lx=2.0, ly=1.0, D=0.4, solver=solver, jitter=0.05, seed=7)
    water = np.r_[case.type, case.type] == S.TYPE_WATER
    case.vel = case.vel + np.where(water, S.fourier_perturbation(case.pos, n_modes=4, amp=0.2, seed=7), 0.0)
    cfg = case.cfg
    cfg.ghost_assign = 1
    cfg.shifting = shifting
    cfg.mls_order, cfg.mls_every = mls_order, 2
    lab = S.moving_square_labels(case, ity)
    dt = 0.25 * cfg.h / np.sqrt(cfg.c0sq)
    motion, _ = S.body_motion_schedule([0.5, 0.3, -0.1], NSTEPS, dt, period=NSTEPS * dt)
    return case, ity, lab, dt, motion


def _tangent(oracle, case, ity, lab, dt, motion, loss, cfg=None, **d):
    return oracle.tangent_ms(case.cfg if cfg is None else cfg, case.pos, case.vel, case.rho, case.mass, case.type,
                             ity, lab, 0.0, NSTEPS, dt, motion, loss, **d)


VARIANTS = [(0, 0), (1, 0), (0, 3), (1, 6), (1, 1)]      # (shifting, mls_order)


@pytest.mark.parametrize("shifting,mls_order", VARIANTS)
@pytest.mark.parametrize("solver", SOLVERS)
def test_tangent_ms_value_path_reproduces_the_oracle(oracle, solver, shifting, mls_order):
    case, ity, lab, dt, motion = _case(solver, shifting, mls_order)
    ke, _ = _tangent(oracle, case, ity, lab, dt, motion, S.LOSS_KINETIC_ENERGY)
    drag, _ = _tangent(oracle, case, ity, lab, dt, motion, S.LOSS_DRAG)
    sim = oracle.OracleSim(case.cfg, case.pos, case.vel, case.rho, case.mass, case.type)
    sim.set_initial_type(ity)
    total = 0.0
    for s in range(NSTEPS):
        oracle.set_ghost_state(lab, motion[s, :2], motion[s, 2:], s * dt)
        sim.run(1, dt)
        total += dt * sim.body_force()[4]
    _, vel, _, _ = sim.state()
    n = case.n
    water = case.type == S.TYPE_WATER
    ke_ref = 0.5 * float(np.sum(case.mass[water] * (vel[:n][water] ** 2 + vel[n:][water] ** 2)))
    assert ke == pytest.approx(ke_ref, rel=1e-12)
    assert drag == pytest.approx(total, rel=1e-10)
    assert drag != 0.0


@pytest.mark.parametrize("shifting,mls_order", VARIANTS)
@pytest.mark.parametrize("solver", SOLVERS)
@pytest.mark.parametrize("loss", [S.LOSS_DRAG, S.LOSS_KINETIC_ENERGY])
def test_tangent_ms_matches_its_central_differences(oracle, loss, solver, shifting, mls_order):
    case, ity, lab, dt, motion = _case(solver, shifting, mls_order)
    rng = np.random.default_rng(2)
    dmo = np.zeros_like(motion)
    dmo[:, 0] = rng.standard_normal(NSTEPS)
    dmo[:, 2] = rng.standard_normal(NSTEPS) * 10.0
    dv = rng.standard_normal(2 * case.n) * 0.1
    eps = 1e-7
    for what, kw, plus, minus in (
            ("motion", dict(dmotion=dmo), dict(motion=motion + eps * dmo), dict(motion=motion - eps * dmo)),
            ("velocity", dict(dvel=dv), dict(vel=dv * eps), dict(vel=-dv * eps))):
        _, dL = _tangent(oracle, case, ity, lab, dt, motion, loss, **kw)
        if what == "motion":
            Lp = _tangent(oracle, case, ity, lab, dt, plus["motion"], loss)[0]
            Lm = _tangent(oracle, case, ity, lab, dt, minus["motion"], loss)[0]
        else:
            c = case
            Lp = oracle.tangent_ms(c.cfg, c.pos, c.vel + plus["vel"], c.rho, c.mass, c.type, ity, lab, 0.0, NSTEPS,
                                   dt, motion, loss)[0]
            Lm = oracle.tangent_ms(c.cfg, c.pos, c.vel + minus["vel"], c.rho, c.mass, c.type, ity, lab, 0.0, NSTEPS,
                                   dt, motion, loss)[0]
        fd = (Lp - Lm) / (2 * eps)
        assert abs(dL - fd) <= 1e-5 * abs(dL), (what, dL, fd)
    _, dLn = _tangent(oracle, case, ity, lab, dt, motion, loss, dnu=1.0)
    c2 = case.cfg.copy()
    e = 1e-5 * c2.nu
    c2.nu = case.cfg.nu + e
    Lp = _tangent(oracle, case, ity, lab, dt, motion, loss, cfg=c2)[0]
    c2.nu = case.cfg.nu - e
    Lm = _tangent(oracle, case, ity, lab, dt, motion, loss, cfg=c2)[0]
    assert abs(dLn - (Lp - Lm) / (2 * e)) <= 1e-5 * abs(dLn)


def test_tangent_ms_rejects_configurations_outside_its_scope(oracle):
    case, ity, lab, dt, motion = _case()
    for field, value in (("laplacian", 0), ("free_surface", 1)):
        cfg = case.cfg.copy()
        setattr(cfg, field, value)
        with pytest.raises(RuntimeError):
            _tangent(oracle, case, ity, lab, dt, motion, S.LOSS_DRAG, cfg=cfg)
    cfg = case.cfg.copy()
    cfg.shifting, cfg.shift_n = 1, 2
    with pytest.raises(RuntimeError):
        _tangent(oracle, case, ity, lab, dt, motion, S.LOSS_DRAG, cfg=cfg)
