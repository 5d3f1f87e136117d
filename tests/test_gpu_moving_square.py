"""GPU parity of the moving-square solvers (HLLC and modified linear Riemann with
XSPH in the continuity flux), the Euler predictor-corrector, the body force, and
the free-surface detection, against the CPU oracle (FP64, 1e-10 norm-wise)."""
import numpy as np
import pytest

import sph_b200 as S

pytestmark = pytest.mark.gpu


def relerr(a, b):
    den = np.abs(b).max()
    return np.abs(a - b).max() / (den if den > 0 else 1.0)


MS_CASES = [
    ("hllc-lattice", dict(solver=S.SOLVER_MS_HLLC_DELTA)),
    ("hllc-jitter", dict(solver=S.SOLVER_MS_HLLC_DELTA, jitter=0.1, seed=3)),
    ("modlr-ms-jitter", dict(solver=S.SOLVER_MS_MODLR_DELTA, jitter=0.1, seed=4)),
]


@pytest.mark.parametrize("name,kw", MS_CASES)
def test_ms_rhs_parity(lib, oracle, name, kw):
    case, ity = S.make_moving_square(**kw)
    ref = oracle.rhs(case.cfg, case.pos, case.vel, case.rho, case.mass, case.type)
    bf_ref = oracle.rhs_body_force(case.cfg, case.pos, case.vel, case.rho, case.mass, case.type, ity)
    with S.Simulation(case.cfg, case.n) as sim:
        sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)
        sim.set_initial_type(ity)
        got = sim.single_step_compute()
        grads = sim.field(S.FIELD_GRADS)
        bf = np.array(sim.diagnostics().body_force[:])
    n = case.n
    assert relerr(got["drhodt"], ref["drhodt"]) < 1e-10
    assert relerr(got["acc"], ref["acc"]) < 1e-10
    assert relerr(got["avg_vel"], ref["avg_vel"]) < 1e-10
    assert relerr(grads[:2 * n], ref["grads"][:2 * n]) < 1e-10
    assert np.abs(bf - bf_ref).max() <= 1e-10 * np.abs(bf_ref).max()


def test_ms_monaghan_laplacian_rhs(lib, oracle):
    case, ity = S.make_moving_square(solver=S.SOLVER_MS_MODLR_DELTA, jitter=0.1, seed=5)
    case.cfg.laplacian = 0
    ref = oracle.rhs(case.cfg, case.pos, case.vel, case.rho, case.mass, case.type)
    with S.Simulation(case.cfg, case.n) as sim:
        sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)
        got = sim.single_step_compute()
    assert relerr(got["acc"], ref["acc"]) < 1e-10
    assert relerr(got["drhodt"], ref["drhodt"]) < 1e-10


@pytest.mark.parametrize("solver", [S.SOLVER_MS_HLLC_DELTA, S.SOLVER_MS_MODLR_DELTA])
def test_euler_pc_fp64_parity(lib, oracle, solver):
    """SPH_Time_Iteration Iteration_Method 2 with shifting, 10 steps; the body force
    of the last RHS (Calculate_Body_Force) alongside."""
    case, ity = S.make_moving_square(solver=solver, jitter=0.05, seed=6)
    dt = 0.25 * case.cfg.h / np.sqrt(case.cfg.c0sq)
    ref = oracle.OracleSim(case.cfg, case.pos, case.vel, case.rho, case.mass, case.type)
    ref.set_initial_type(ity)
    ref.run(10, dt)
    rpos, rvel, rrho, _ = ref.state()
    with S.Simulation(case.cfg, case.n) as sim:
        sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)
        sim.set_initial_type(ity)
        d = sim.time_iteration(10, dt)
        pos, vel, rho, _ = sim.get_state()
    assert relerr(vel, rvel) < 1e-10
    assert relerr(rho - case.cfg.rho0, rrho - case.cfg.rho0) < 1e-10
    assert np.abs(pos - rpos).max() < 1e-12
    bf = np.array(d.body_force[:])
    bref = ref.body_force()
    assert np.abs(bf - bref).max() <= 1e-10 * np.abs(bref).max()


def test_free_surface_detection(lib, oracle):
    """A water block with open edges (no periodic images): the volume-fraction
    candidates, the geometric normal test and the near-surface flags
    (Define_freesurface_and_Normailized_derivates.f90:119-440) match the oracle,
    and the near-surface particles take the averaged Riemann state."""
    case = S.make_tgv(40, solver=S.SOLVER_MODLR_DELTA_SPS, jitter=0.05, seed=8)
    case.cfg.periodic = 0
    ref = oracle.rhs(case.cfg, case.pos, case.vel, case.rho, case.mass, case.type)
    with S.Simulation(case.cfg, case.n) as sim:
        sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)
        got = sim.single_step_compute()
    assert ref["fs"].sum() > 100 and ref["near"].sum() > ref["fs"].sum()
    assert np.array_equal(got["fs"], ref["fs"])
    assert np.array_equal(got["near"], ref["near"])
    assert relerr(got["acc"], ref["acc"]) < 1e-10
    assert relerr(got["drhodt"], ref["drhodt"]) < 1e-10


@pytest.mark.parametrize("solver", [S.SOLVER_MS_HLLC_DELTA, S.SOLVER_MS_MODLR_DELTA])
def test_ms_mixed_rhs_close_to_fp64(lib, solver):
    """The mixed path (FP32 pair arithmetic from hi/lo records, the HLLC state
    formed in differences) against the FP64 path on one RHS of a jittered tank
    with a seeded velocity field: acceleration and density rate within a few
    FP32 roundings (L2 relative)."""
    out = {}
    for prec in (S.PREC_FP64, S.PREC_MIXED):
        case, ity = S.make_moving_square(solver=solver, precision=prec, jitter=0.1, seed=9)
        rng = np.random.default_rng(3)
        water = case.type == S.TYPE_WATER
        vel = case.vel.copy()
        vel[:case.n][water] += rng.uniform(-0.2, 0.2, water.sum())
        vel[case.n:][water] += rng.uniform(-0.2, 0.2, water.sum())
        with S.Simulation(case.cfg, case.n) as sim:
            sim.set_state(case.pos, vel, case.rho, case.mass, case.type)
            sim.set_initial_type(ity)
            out[prec] = sim.single_step_compute()
    a64, a32 = out[S.PREC_FP64], out[S.PREC_MIXED]
    for k, tol in (("acc", 1e-5), ("drhodt", 1e-5), ("avg_vel", 1e-5)):
        err = np.linalg.norm(a32[k] - a64[k]) / np.linalg.norm(a64[k])
        assert err < tol, (k, err)
