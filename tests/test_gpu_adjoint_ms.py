"""The discrete adjoint of the moving-square step (sph_adjoint_forward /
sph_adjoint_backward / sph_adjoint_motion_gradient) against central finite
differences of the FP64 forward run on the GPU.

The case: the moving-square modified linear Riemann solver, and the HLLC solver
(Solver_Normalized_HLLC_Riemann_Delta.f90, its state reversed on the sampled
region and wave speeds the forward took), with XSPH velocities in the
continuity flux, the Morris laplacian and the Euler predictor-corrector, the
library's ghost assignment at every RHS (Shepard interpolation onto the wall
and body ghosts, mirrored wall velocities, the shock-release branch) and the
body moved by a per-step schedule.  Losses: the drag impulse sum_s dt F_x and
the final kinetic energy.  Parameters: the motion amplitude (impulsive start),
four Fourier coefficients of the motion, the viscosity and the initial
velocity field.  The improved Gaussian kernel is cut off with a kink at 3h
(and the ghost kernel at 3 * 1.2h), so the difference steps are those of the
Gaussian Taylor-Green checks (1e-7 relative).

The water starts with a smooth velocity field rather than at rest: at rest
every pair sits exactly on the artificial-viscosity switch v.r = 0, where the
alpha term (alpha = 0.03 here, 0 in the Taylor-Green cases) has a kink, and a
central difference straddling it measures the mean of the one-sided slopes
while the adjoint takes the inactive branch."""
import numpy as np
import pytest

import sph_b200 as S

pytestmark = pytest.mark.gpu

NSTEPS = 16
REL_TOL = 1e-4


SOLVERS = [S.SOLVER_MS_MODLR_DELTA, S.SOLVER_MS_HLLC_DELTA]


def _case(jitter=0.05, seed=41, ghost_assign=1, solver=S.SOLVER_MS_MODLR_DELTA):
    case, ity = S.make_moving_square(solver=solver, jitter=jitter, seed=seed)
    water = np.r_[case.type, case.type] == S.TYPE_WATER
    case.vel = case.vel + np.where(water, S.fourier_perturbation(case.pos, n_modes=6, amp=0.2, seed=seed), 0.0)
    cfg = case.cfg
    cfg.ghost_assign = ghost_assign
    cfg.shifting = 0
    cfg.mls_order = 0
    lab = S.moving_square_labels(case, ity)
    dt = 0.25 * cfg.h / np.sqrt(cfg.c0sq)
    return case, ity, lab, dt


def _sim(case, ity, lab, cfg=None, vel=None):
    sim = S.Simulation(case.cfg if cfg is None else cfg, case.n)
    sim.set_state(case.pos, case.vel if vel is None else case.vel + vel, case.rho, case.mass, case.type)
    sim.set_initial_type(ity)
    sim.set_boundary_labels(lab)
    sim.set_time(0.0)
    return sim


def _loss(case, ity, lab, dt, motion, loss, cfg=None, vel=None):
    with _sim(case, ity, lab, cfg, vel) as sim:
        return sim.adjoint_forward(NSTEPS, dt, checkpoint_every=NSTEPS, loss=loss, body_motion=motion)


def _grad(case, ity, lab, dt, motion, loss, every=5):
    with _sim(case, ity, lab) as sim:
        L = sim.adjoint_forward(NSTEPS, dt, checkpoint_every=every, loss=loss, body_motion=motion)
        end = sim.get_state()
        g = sim.adjoint_backward(1.0)
        gm = sim.adjoint_motion_gradient()
        after = sim.get_state()
    return L, g, gm, end, after


def _check(ad, fd, what):
    assert abs(ad - fd) <= REL_TOL * abs(fd), (what, ad, fd, abs(ad - fd) / abs(fd))


def test_drag_loss_is_the_sum_of_the_step_forces(lib):
    """The forward drag loss equals sum_s dt * body_force[4] of time_iteration
    with the same per-step motion."""
    case, ity, lab, dt = _case()
    motion, _ = S.body_motion_schedule([0.6, 0.3, 0.0, 0.1, 0.0], NSTEPS, dt, period=NSTEPS * dt)
    L = _loss(case, ity, lab, dt, motion, S.LOSS_DRAG)
    with _sim(case, ity, lab) as sim:
        total = 0.0
        for s in range(NSTEPS):
            sim.set_body_motion(motion[s, :2], motion[s, 2:])
            d = sim.time_iteration(1, dt)
            total += dt * d.body_force[4]
    assert L == pytest.approx(total, rel=1e-12, abs=0)
    assert L != 0.0


@pytest.mark.parametrize("solver,loss", [(S.SOLVER_MS_MODLR_DELTA, S.LOSS_DRAG),
                                         (S.SOLVER_MS_MODLR_DELTA, S.LOSS_KINETIC_ENERGY),
                                         (S.SOLVER_MS_HLLC_DELTA, S.LOSS_DRAG)])
def test_motion_gradient_matches_central_differences(lib, solver, loss):
    """dL/d(amplitude) of the impulsive start and dL/d(Fourier coefficients)."""
    case, ity, lab, dt = _case(solver=solver)
    period = NSTEPS * dt
    coeffs = np.array([0.5, 0.4, -0.2, 0.15, 0.1])
    motion, jac = S.body_motion_schedule(coeffs, NSTEPS, dt, period=period)
    L, g, gm, end, after = _grad(case, ity, lab, dt, motion, loss)
    assert np.isfinite(L) and L != 0.0
    assert all(np.array_equal(a, b) for a, b in zip(end, after))
    assert np.all(np.isfinite(gm))
    gc = np.einsum("sq,sqk->k", gm, jac)
    for k in range(coeffs.size):
        eps = 1e-7
        cp, cm = coeffs.copy(), coeffs.copy()
        cp[k] += eps
        cm[k] -= eps
        fd = (_loss(case, ity, lab, dt, S.body_motion_schedule(cp, NSTEPS, dt, period=period)[0], loss)
              - _loss(case, ity, lab, dt, S.body_motion_schedule(cm, NSTEPS, dt, period=period)[0], loss)) / (2 * eps)
        _check(gc[k], fd, f"motion coefficient {k}")


@pytest.mark.parametrize("solver", SOLVERS)
def test_drag_gradient_velocity_and_viscosity(lib, solver):
    case, ity, lab, dt = _case(solver=solver)
    motion, _ = S.body_motion_schedule([1.0], NSTEPS, dt)
    L, g, gm, _, _ = _grad(case, ity, lab, dt, motion, S.LOSS_DRAG)
    n = case.n
    water = case.type == S.TYPE_WATER
    # ghost velocities are overwritten before use: no gradient
    assert np.all(g["vel0"][:n][~water] == 0) and np.all(g["vel0"][n:][~water] == 0)
    for k in range(2):
        rng = np.random.default_rng(300 + k)
        d = rng.standard_normal(2 * n) * 0.1
        eps = 1e-7
        fd = (_loss(case, ity, lab, dt, motion, S.LOSS_DRAG, vel=eps * d)
              - _loss(case, ity, lab, dt, motion, S.LOSS_DRAG, vel=-eps * d)) / (2 * eps)
        _check(float(g["vel0"] @ d), fd, f"velocity direction {k}")
    nu = case.cfg.nu
    e = 1e-5 * nu
    cp, cm = case.cfg.copy(), case.cfg.copy()
    cp.nu, cm.nu = nu + e, nu - e
    fd = (_loss(case, ity, lab, dt, motion, S.LOSS_DRAG, cfg=cp)
          - _loss(case, ity, lab, dt, motion, S.LOSS_DRAG, cfg=cm)) / (2 * e)
    _check(g["nu"], fd, "viscosity")


def test_adjoint_with_caller_given_ghosts(lib):
    """ghost_assign = 0: the ghost states are the caller's and stay constant, so
    their initial velocities are live inputs; the body does not move."""
    case, ity, lab, dt = _case(ghost_assign=0)
    motion, _ = S.body_motion_schedule([1.0], NSTEPS, dt)
    L, g, gm, _, _ = _grad(case, ity, lab, dt, motion, S.LOSS_DRAG)
    assert np.all(gm == 0)
    n = case.n
    rng = np.random.default_rng(310)
    d = rng.standard_normal(2 * n) * 0.1
    eps = 1e-7
    fd = (_loss(case, ity, lab, dt, motion, S.LOSS_DRAG, vel=eps * d)
          - _loss(case, ity, lab, dt, motion, S.LOSS_DRAG, vel=-eps * d)) / (2 * eps)
    _check(float(g["vel0"] @ d), fd, "velocity direction")
    ghost = np.r_[case.type, case.type] != S.TYPE_WATER
    assert np.any(g["vel0"][ghost] != 0)


def test_moving_square_adjoint_independent_of_checkpoint_interval(lib):
    case, ity, lab, dt = _case()
    motion, _ = S.body_motion_schedule([0.5, 0.4], NSTEPS, dt, period=NSTEPS * dt)
    ref = _grad(case, ity, lab, dt, motion, S.LOSS_DRAG, every=NSTEPS)
    for every in (1, 7):
        got = _grad(case, ity, lab, dt, motion, S.LOSS_DRAG, every=every)
        assert got[0] == ref[0]
        for key in ("vel0", "rho0", "pos0"):
            assert np.array_equal(got[1][key], ref[1][key]), (every, key)
        assert got[1]["nu"] == ref[1]["nu"]
        assert np.array_equal(got[2], ref[2])


@pytest.mark.parametrize("solver,shifting,mls_order", [(S.SOLVER_MS_MODLR_DELTA, 1, 0), (S.SOLVER_MS_HLLC_DELTA, 1, 0),
                                                      (S.SOLVER_MS_MODLR_DELTA, 0, 3),
                                                      (S.SOLVER_MS_HLLC_DELTA, 1, 6), (S.SOLVER_MS_MODLR_DELTA, 0, 1)])
def test_shifting_and_mls_adjoint_matches_central_differences(lib, solver, shifting, mls_order):
    """Particle shifting after every corrector (Shift_particle_position.f90:
    56-136 on the corrector RHS's pairs, ghosts included) and the density
    re-initialisation every fourth step (Moving_Square.../
    Reinitialize_particle_density.f90:92-200): drag gradient in two motion
    coefficients and one velocity direction, and the same gradient at every
    checkpoint interval (1: every corrector RHS kept from the segment re-run;
    16: all re-formed in the reverse step)."""
    case, ity, lab, dt = _case(solver=solver)
    case.cfg.shifting = shifting
    case.cfg.mls_order, case.cfg.mls_every = mls_order, 4
    period = NSTEPS * dt
    coeffs = np.array([0.5, 0.4, -0.2])
    motion, jac = S.body_motion_schedule(coeffs, NSTEPS, dt, period=period)
    L, g, gm, end, after = _grad(case, ity, lab, dt, motion, S.LOSS_DRAG)
    assert all(np.array_equal(a, b) for a, b in zip(end, after))
    with _sim(case, ity, lab) as sim:
        L0 = sim.adjoint_forward(NSTEPS, dt, checkpoint_every=NSTEPS, loss=S.LOSS_DRAG, body_motion=motion)
    assert L0 == L
    case.cfg.shifting, case.cfg.mls_order = 0, 0
    assert _loss(case, ity, lab, dt, motion, S.LOSS_DRAG) != L
    case.cfg.shifting, case.cfg.mls_order = shifting, mls_order
    gc = np.einsum("sq,sqk->k", gm, jac)
    for k in (0, 2):
        eps = 1e-7
        cp, cm = coeffs.copy(), coeffs.copy()
        cp[k] += eps
        cm[k] -= eps
        fd = (_loss(case, ity, lab, dt, S.body_motion_schedule(cp, NSTEPS, dt, period=period)[0], S.LOSS_DRAG)
              - _loss(case, ity, lab, dt, S.body_motion_schedule(cm, NSTEPS, dt, period=period)[0],
                      S.LOSS_DRAG)) / (2 * eps)
        _check(gc[k], fd, f"motion coefficient {k}")
    rng = np.random.default_rng(320)
    d = rng.standard_normal(2 * case.n) * 0.1
    eps = 1e-7
    fd = (_loss(case, ity, lab, dt, motion, S.LOSS_DRAG, vel=eps * d)
          - _loss(case, ity, lab, dt, motion, S.LOSS_DRAG, vel=-eps * d)) / (2 * eps)
    _check(float(g["vel0"] @ d), fd, "velocity direction")
    for every in (1, NSTEPS):
        got = _grad(case, ity, lab, dt, motion, S.LOSS_DRAG, every=every)
        assert got[0] == L
        for key in ("vel0", "rho0", "pos0"):
            assert np.array_equal(got[1][key], g[key]), (every, key)
        assert np.array_equal(got[2], gm)


def test_moving_square_adjoint_rejects_unsupported(lib):
    case, ity, lab, dt = _case()
    cfg = case.cfg.copy()
    cfg.laplacian = 0          # the Monaghan-form laplacian has no reverse
    with _sim(case, ity, lab, cfg) as sim:
        with pytest.raises(S.SphError) as e:
            sim.adjoint_forward(2, dt, loss=S.LOSS_DRAG)
        assert e.value.code == -7
    # the drag loss needs a body
    case2 = S.make_tgv(16, solver=S.SOLVER_MODLR_DELTA_SPS)
    case2.cfg.shifting = 0
    case2.cfg.mls_order = 0
    with S.Simulation(case2.cfg, case2.n) as sim:
        sim.set_state(case2.pos, case2.vel, case2.rho, case2.mass, case2.type)
        with pytest.raises(S.SphError) as e:
            sim.adjoint_forward(2, 1e-4, loss=S.LOSS_DRAG)
        assert e.value.code == -7


@pytest.mark.parametrize("shifting,mls_order", [(0, 0), (1, 0), (0, 3), (1, 6), (1, 1)])
@pytest.mark.parametrize("solver", SOLVERS)
@pytest.mark.parametrize("loss", [S.LOSS_DRAG, S.LOSS_KINETIC_ENERGY])
def test_moving_square_adjoint_matches_cpu_tangent_linear_reference(lib, oracle, loss, solver, shifting,
                                                                     mls_order):
    """g.delta from the GPU adjoint against the FP64 CPU tangent-linear model of
    the same steps (oracle/sph_tangent.cpp, oracle_tangent_ms) along directions
    in the initial velocity, position and density, the viscosity and the body
    motion: both are exact derivatives of the same discrete map (1e-8).  With
    shifting, each step ends with the capped shift of the corrector RHS; with
    mls_order, every fourth step re-initialises the density first (orders 3, 6:
    the moving-square variant, W V weights over every particle in the support,
    the ghosts with the density and mass the corrector RHS assigned them;
    order 1: the Shepard density over the corrector RHS's water pairs)."""
    case, ity = S.make_moving_square(dx=0.1, lx=2.0, ly=1.0, D=0.4, solver=solver, jitter=0.05, seed=8)
    water = np.r_[case.type, case.type] == S.TYPE_WATER
    case.vel = case.vel + np.where(water, S.fourier_perturbation(case.pos, n_modes=4, amp=0.2, seed=8), 0.0)
    cfg = case.cfg
    cfg.ghost_assign, cfg.shifting, cfg.mls_order, cfg.mls_every = 1, shifting, mls_order, 4
    lab = S.moving_square_labels(case, ity)
    dt = 0.25 * cfg.h / np.sqrt(cfg.c0sq)
    motion, _ = S.body_motion_schedule([0.5, 0.3, -0.1], NSTEPS, dt, period=NSTEPS * dt)
    L, g, gm, _, _ = _grad(case, ity, lab, dt, motion, loss)
    n = case.n
    rng = np.random.default_rng(500)
    dmo = np.zeros_like(motion)
    dmo[:, 0] = rng.standard_normal(NSTEPS)
    dmo[:, 1] = rng.standard_normal(NSTEPS)
    dmo[:, 2] = rng.standard_normal(NSTEPS) * 10.0
    dirs = [dict(dvel=rng.standard_normal(2 * n) * 0.1), dict(dpos=rng.standard_normal(2 * n) * 0.01 * cfg.dx),
            dict(drho=rng.standard_normal(n) * 1e-3), dict(dnu=1.0), dict(dmotion=dmo)]
    for d in dirs:
        Lt, dLt = oracle.tangent_ms(cfg, case.pos, case.vel, case.rho, case.mass, case.type, ity, lab, 0.0, NSTEPS,
                                    dt, motion, loss, **d)
        assert Lt == pytest.approx(L, rel=1e-10)
        key = list(d)[0]
        ad = {"dvel": lambda: float(g["vel0"] @ d["dvel"]), "dpos": lambda: float(g["pos0"] @ d["dpos"]),
              "drho": lambda: float(g["rho0"] @ d["drho"]), "dnu": lambda: g["nu"],
              "dmotion": lambda: float(np.sum(gm * d["dmotion"]))}[key]()
        assert abs(ad - dLt) <= 1e-8 * abs(dLt), (key, ad, dLt)


def test_motion_gradient_long_horizon_wendland(lib):
    """25 times the other checks' horizon with the Wendland C2 kernel (h = 1.3 dx,
    support 2h): its gradient is zero at the cut-off, so a pair crossing it puts
    no jump into the right-hand side and central differences keep converging over
    hundreds of steps (with the improved Gaussian they stop doing so after about
    200 steps at D/50).  Drag loss, motion amplitude and one Fourier coefficient."""
    case, ity, lab, _ = _case()
    cfg = case.cfg.copy()
    cfg.kernel_model, cfg.kernel_scale, cfg.h = S.KERNEL_WENDLAND2, 2.0, 1.3 * cfg.dx
    case.cfg = cfg
    dt = 0.25 * cfg.h / np.sqrt(cfg.c0sq)
    n = 25 * NSTEPS
    coeffs = np.array([0.5, 0.2, -0.1])
    motion, jac = S.body_motion_schedule(coeffs, n, dt, period=n * dt)

    def loss(c):
        mo = S.body_motion_schedule(c, n, dt, period=n * dt)[0]
        with _sim(case, ity, lab) as sim:
            return sim.adjoint_forward(n, dt, checkpoint_every=64, loss=S.LOSS_DRAG, body_motion=mo)

    with _sim(case, ity, lab) as sim:
        sim.adjoint_forward(n, dt, checkpoint_every=64, loss=S.LOSS_DRAG, body_motion=motion)
        sim.adjoint_backward(1.0)
        g = np.einsum("sq,sqk->k", sim.adjoint_motion_gradient(), jac)
    for k in (0, 1):
        eps = 1e-6
        cp, cm = coeffs.copy(), coeffs.copy()
        cp[k] += eps
        cm[k] -= eps
        _check(g[k], (loss(cp) - loss(cm)) / (2 * eps), ("coefficient", k))
