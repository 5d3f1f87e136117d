"""Error paths of the time step, driven by failures injected on the host.

The reference prints and carries on where this library returns a status:
particles leaving the cell grid are tagged ill (type 120,
Taylor_Green_Vortex/Devide_block_and_send_tasks.f90:75-83), a background cell
or a particle's candidate list that overflows is reported and truncated
(Taylor_Green_Vortex/Assign_boundary_particles.f90:100-104,142-147), and so is
the pair array (Taylor_Green_Vortex/find_particle_pair.f90:89,116-118).  Here
each failure is made on the host -- a NaN in the state handed to
sph_set_state, a particle placed outside grid_lo..grid_hi, a velocity that
carries a particle past half the neighbour-list skin within one step, a stack
of particles that overflows the neighbour lists -- and the test checks the
code sph_step returns and that the same handle steps cleanly again once a
clean state is set.  No kernel is made to fault: every injected value stays in
the bounds the kernels check.
"""
import numpy as np
import pytest

import sph_b200 as S

pytestmark = pytest.mark.gpu

E_CAPACITY, E_NONFINITE, E_DOMAIN, E_SKIN = -2, -3, -8, -9


def _case(n_side=32):
    return S.make_tgv(n_side, solver=S.SOLVER_MUSCL_DELTA_SPS, jitter=0.1, seed=3)


def _step_code(sim, dt, nsteps=1):
    try:
        sim.time_iteration(nsteps, dt)
    except S.SphError as e:
        return e.code
    return 0


def _recovers(sim, case, dt):
    """The handle takes a clean state and steps without error afterwards."""
    sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)
    d = sim.time_iteration(2, dt)
    _, vel, rho, _ = sim.get_state()
    assert np.isfinite(vel).all() and np.isfinite(rho).all()
    assert d.kinetic_energy > 0.0


def test_nonfinite_velocity_is_reported(lib):
    case = _case()
    dt = S.baseline_dt(case.cfg)
    vel = case.vel.copy()
    vel[case.n // 2] = np.nan           # u of one water particle
    with S.Simulation(case.cfg, case.n) as sim:
        sim.set_state(case.pos, vel, case.rho, case.mass, case.type)
        assert _step_code(sim, dt) == E_NONFINITE
        _recovers(sim, case, dt)


def test_nonfinite_density_is_reported(lib):
    case = _case()
    dt = S.baseline_dt(case.cfg)
    rho = case.rho.copy()
    rho[7] = np.inf
    with S.Simulation(case.cfg, case.n) as sim:
        sim.set_state(case.pos, case.vel, rho, case.mass, case.type)
        assert _step_code(sim, dt) == E_NONFINITE
        _recovers(sim, case, dt)


def test_particle_outside_the_grid_is_reported(lib):
    case = _case()
    dt = S.baseline_dt(case.cfg)
    pos = case.pos.copy()
    # x = 3.0 in the unit periodic box: the periodic wrap moves it by one box
    # length (to 2.0), still beyond grid_hi, so it is not binned
    pos[5] = 3.0
    with S.Simulation(case.cfg, case.n) as sim:
        sim.set_state(pos, case.vel, case.rho, case.mass, case.type)
        assert _step_code(sim, dt) == E_DOMAIN
        _recovers(sim, case, dt)


def test_particle_outside_the_grid_non_periodic(lib):
    case, itype = S.make_moving_square(dx=0.1, lx=2.0, ly=1.0, D=0.4)
    cfg = case.cfg.copy()
    cfg.shifting = 0
    cfg.mls_order = 0
    dt = 0.25 * cfg.h / np.sqrt(cfg.c0sq)
    pos = case.pos.copy()
    pos[case.n + 3] = cfg.grid_hi[1] + 1.0          # y of a water particle above the grid
    with S.Simulation(cfg, case.n) as sim:
        sim.set_state(pos, case.vel, case.rho, case.mass, case.type)
        sim.set_initial_type(itype)
        assert _step_code(sim, dt) == E_DOMAIN
        sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)
        sim.set_initial_type(itype)
        sim.time_iteration(2, dt)


def test_displacement_beyond_the_skin_is_reported(lib):
    case = _case()
    dt = S.baseline_dt(case.cfg)
    # half the skin is 0.05 of the support 2h = 2.6 dx, i.e. 0.13 dx; one step
    # of dt = 0.0325 dx / U0 at speed 10 U0 moves a particle 0.325 dx
    skin_half = 0.5 * case.cfg.cell_skin * 2.0 * case.cfg.h
    speed = 10.0
    assert speed * dt > 2.0 * skin_half
    vel = case.vel.copy()
    k = case.n // 3
    vel[k] = speed
    vel[case.n + k] = 0.0
    with S.Simulation(case.cfg, case.n) as sim:
        sim.set_state(case.pos, vel, case.rho, case.mass, case.type)
        assert _step_code(sim, dt) == E_SKIN
        _recovers(sim, case, dt)


def test_neighbour_list_overflow_is_reported(lib):
    case = _case()
    dt = S.baseline_dt(case.cfg)
    n0 = case.n
    # the list holds about twice the lattice count inside the list radius (68
    # entries here); 90 extra particles 1e-6 apart around one point overflow it
    extra = 90
    x0, y0 = 0.5 + 0.3 * case.cfg.dx, 0.5 + 0.3 * case.cfg.dx
    ex = x0 + 1e-6 * np.arange(extra)
    ey = np.full(extra, y0)
    pos = np.concatenate([case.pos[:n0], ex, case.pos[n0:], ey])
    vel = np.concatenate([case.vel[:n0], np.zeros(extra), case.vel[n0:], np.zeros(extra)])
    rho = np.concatenate([case.rho, np.full(extra, case.rho.mean())])
    mass = np.concatenate([case.mass, np.full(extra, case.mass.mean())])
    typ = np.concatenate([case.type, np.full(extra, S.TYPE_WATER, np.int32)])
    n = n0 + extra
    with S.Simulation(case.cfg, n) as sim:
        sim.set_state(pos, vel, rho, mass, typ)
        assert _step_code(sim, dt) == E_CAPACITY
        _recovers(sim, case, dt)


def test_clean_state_reports_no_error(lib):
    """The injected cases above differ from this one only in the injected value."""
    case = _case()
    dt = S.baseline_dt(case.cfg)
    with S.Simulation(case.cfg, case.n) as sim:
        sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)
        assert _step_code(sim, dt, 3) == 0
