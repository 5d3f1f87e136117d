"""GPU parity of the moving-square ghost assignment (Assign_boundary_particles,
fixed wall ghosts and body ghosts, at every RHS) with the body moving at its
prescribed velocity, against the oracle: 10 Euler predictor-corrector steps of
both moving-square solvers, all particle states (ghosts included) and the body
force, FP64, 1e-10 norm-wise.

The moving body changes the cell sort order from step to step, so these cases
also check that the predictor takes each particle's own carried rates after
the re-sort."""
import numpy as np
import pytest

import sph_b200 as S

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("solver,wall_bc,t0", [(S.SOLVER_MS_HLLC_DELTA, 0, 0.0),
                                               (S.SOLVER_MS_MODLR_DELTA, 1, 0.0),
                                               (S.SOLVER_MS_HLLC_DELTA, 0, 20.0)])
def test_ghost_assignment_moving_body(lib, oracle, solver, wall_bc, t0):
    case, ity = S.make_moving_square(solver=solver, jitter=0.05, seed=31)
    case.cfg.ghost_assign = 1
    case.cfg.wall_bc = wall_bc
    lab = S.moving_square_labels(case, ity)
    U = (1.0, 0.0)
    dt = 0.25 * case.cfg.h / np.sqrt(case.cfg.c0sq)
    oracle.set_ghost_state(lab, U, (0.0, 0.0), t0)
    ref = oracle.OracleSim(case.cfg, case.pos, case.vel, case.rho, case.mass, case.type)
    ref.set_initial_type(ity)
    ref.run(10, dt)
    rpos, rvel, rrho, _ = ref.state()
    bref = ref.body_force()
    with S.Simulation(case.cfg, case.n) as sim:
        sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)
        sim.set_initial_type(ity)
        sim.set_boundary_labels(lab)
        sim.set_body_motion(U)
        sim.set_time(t0)
        d = sim.time_iteration(10, dt)
        pos, vel, rho, _ = sim.get_state()
    assert np.abs(pos - rpos).max() < 1e-12
    assert relerr(vel, rvel) < 1e-10
    assert relerr(rho - case.cfg.rho0, rrho - case.cfg.rho0) < 1e-10
    bf = np.array(d.body_force[:])
    assert np.abs(bf - bref).max() <= 1e-10 * np.abs(bref).max()
    # the body moved with its velocity, the wall ghosts took interpolated states
    body = ity == S.TYPE_BODY
    n = case.n
    assert np.allclose(pos[:n][body] - case.pos[:n][body], 10 * dt * U[0], rtol=0, atol=1e-12)
    assert np.abs(rho[lab != 0] - case.cfg.rho0).max() > 0


def test_cylinder_label_keeps_the_interpolated_velocity(lib, oracle):
    """Wall ghosts labelled -9 (along the cylinder, Assign_boundary_particles.f90:902-905)
    take the interpolated velocity without a mirror: the reference's radius_free_slip
    call there reads and writes the global particle arrays, not the ghost's own
    subdomain velocity.  Half of the horizontal-wall ghosts relabelled -9; GPU
    against the oracle over 10 steps, and against the unrelabelled run (the labels
    change the flow)."""
    case, ity = S.make_moving_square(solver=S.SOLVER_MS_HLLC_DELTA, jitter=0.05, seed=32)
    case.cfg.ghost_assign = 1
    lab = S.moving_square_labels(case, ity).copy()
    horiz = np.flatnonzero(lab == -6)
    assert horiz.size > 20
    lab9 = lab.copy()
    lab9[horiz[::2]] = -9
    U = (1.0, 0.0)
    dt = 0.25 * case.cfg.h / np.sqrt(case.cfg.c0sq)
    oracle.set_ghost_state(lab9, U, (0.0, 0.0), 0.0)
    ref = oracle.OracleSim(case.cfg, case.pos, case.vel, case.rho, case.mass, case.type)
    ref.set_initial_type(ity)
    ref.run(10, dt)
    rpos, rvel, rrho, _ = ref.state()
    out = {}
    for name, lb in (("-9", lab9), ("-6", lab)):
        with S.Simulation(case.cfg, case.n) as sim:
            sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)
            sim.set_initial_type(ity)
            sim.set_boundary_labels(lb)
            sim.set_body_motion(U)
            sim.time_iteration(10, dt)
            out[name] = sim.get_state()
    pos, vel, rho, _ = out["-9"]
    assert np.abs(pos - rpos).max() < 1e-12
    assert relerr(vel, rvel) < 1e-10
    assert relerr(rho - case.cfg.rho0, rrho - case.cfg.rho0) < 1e-10
    assert relerr(out["-6"][1], vel) > 1e-8
