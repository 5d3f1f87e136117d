"""CPU tests of the oracle against the reference's own committed outputs
(tests/golden/tgv_reference.npz, extracted by tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

import sph_b200 as S

GOLD = os.path.join(os.path.dirname(__file__), "golden", "tgv_reference.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def test_tgv_initialiser_matches_reference_output(oracle, gold):
    """Distribute_Initial_Particle.f90:206-231 against Initial_particle_information.dat."""
    pos, vel, rho, mass, press = oracle.tgv_init(100, 100, rho0=1000.0, c0sq=100.0, sign=1, reference_literals=True)
    n = 10000
    idx = gold["init_index"]
    g = gold["init_rows"]
    # the file prints 10 decimals
    assert np.abs(pos[idx] - g[:, 0]).max() < 6e-11
    assert np.abs(pos[n + idx] - g[:, 1]).max() < 6e-11
    assert np.abs(vel[idx] - g[:, 2]).max() < 6e-11
    assert np.abs(vel[n + idx] - g[:, 3]).max() < 6e-11
    assert np.abs(rho[idx] - g[:, 4]).max() < 6e-11
    assert np.abs(press[idx] / 1000.0 - g[:, 5]).max() < 6e-11


def test_numpy_lattice_equals_oracle():
    import oracle_api as O
    a = O.tgv_init(32, 32, rho0=1.0, c0sq=100.0, sign=-1, reference_literals=False)
    b = S.tgv_lattice(32, rho0=1.0, c0sq=100.0, sign=-1)
    for x, y in zip(a, b):
        np.testing.assert_allclose(x, y, rtol=1e-14, atol=1e-15)


def test_kinetic_energy_decay_matches_reference_run(oracle, gold):
    """100 steps (t = 0.01) of the shipped TGV configuration: KE/KE0 against
    the reference's Kinetic_energy.dat row 1 (0.98334343).  The reference run
    used 5 MPI ranks and MLS re-initialisation every 20 steps, so the match is
    physical, not bitwise: 2e-5 relative."""
    case = S.make_tgv(100, reference=True)
    sim = oracle.OracleSim(case.cfg, case.pos, case.vel, case.rho, case.mass, case.type)
    ke0 = sim.kinetic_energy()
    sim.run(100, 1e-4)
    ratio = sim.kinetic_energy() / ke0
    ref = gold["kinetic_energy"][0]
    assert abs(ref[0] - 0.01) < 1e-12
    assert abs(ratio - ref[1]) / ref[1] < 2e-5, (ratio, ref[1])


def test_pair_set_properties(oracle):
    """find_particle_pair rules on a lattice: i < j, support and 1e-7 cut, neighbour count."""
    case = S.make_tgv(40, reference=False, solver=S.SOLVER_MUSCL_DELTA_SPS)
    pr = oracle.find_particle_pair(case.cfg, case.pos, case.type)
    assert np.all(pr["pair_i"] < pr["pair_j"])
    n = case.n
    i = pr["pair_i"] - 1
    j = pr["pair_j"] - 1
    d = np.hypot(case.pos[i] - case.pos[j], case.pos[n + i] - case.pos[n + j])
    assert d.max() <= case.cfg.kernel_scale * case.cfg.h
    # interior lattice particle: 20 neighbours inside 2.6 dx (a^2+b^2 <= 6.76)
    deg = np.bincount(np.concatenate([i, j]), minlength=n)
    assert deg.max() == 20
    # duplicates
    key = i.astype(np.int64) * n + j
    assert np.unique(key).size == key.size


def test_periodic_images_follow_reference_order(oracle):
    case = S.make_tgv(20, reference=True)
    pos, vel, rho, mass, typ, src = oracle.periodic_images(case.cfg, case.pos, case.vel, case.rho, case.mass,
                                                           case.type)
    n = case.n
    m = rho.size - n
    band = case.cfg.kernel_scale * case.cfg.h
    # every image sits outside the unit box, within band of it
    x, y = pos[:rho.size], pos[rho.size:]
    xi, yi = x[n:], y[n:]
    assert np.all(typ[n:] == S.TYPE_PERIODIC)
    outside = (xi < 0) | (xi > 1) | (yi < 0) | (yi > 1)
    assert np.all(outside)
    assert np.all((xi > -band - 1e-12) & (xi < 1 + band + 1e-12) & (yi > -band - 1e-12) & (yi < 1 + band + 1e-12))
    # 20x20 lattice, band 3.6 dx -> 4 rows per edge: 4*20*4 edges + 4*4*4 corners
    assert m == 4 * 20 * 4 + 4 * 16


def test_rhs_is_deterministic_across_threads(oracle):
    case = S.make_tgv(32, reference=False, jitter=0.1, seed=3)
    oracle.threads(1)
    a = oracle.rhs(case.cfg, case.pos, case.vel, case.rho, case.mass, case.type)
    oracle.threads(4)
    b = oracle.rhs(case.cfg, case.pos, case.vel, case.rho, case.mass, case.type)
    oracle.threads(0)
    for k in ("drhodt", "acc", "tau", "grads", "binv"):
        assert np.array_equal(a[k], b[k]), k


def test_muscl_limiter_ties_on_exact_lattice(oracle):
    """The reference MUSCL limiter (function_module.f90:34-80) is discontinuous at
    di == dj and at lim == 0.5 dphi.  On an exact lattice the Taylor-Green field
    puts many pairs exactly on those ties, so the reference's own result is decided
    by round-off: a 1e-15 relative change of the positions changes drhodt by O(1).
    On a jittered lattice the same perturbation stays at round-off level.  Parity
    of the MUSCL solver is therefore tested on jittered lattices."""
    out = {}
    for jit in (0.0, 0.1):
        case = S.make_tgv(48, solver=S.SOLVER_MUSCL_DELTA_SPS, jitter=jit, seed=1)
        ext = oracle.periodic_images(case.cfg, case.pos, case.vel, case.rho, case.mass, case.type)[:5]
        a = oracle.rhs(case.cfg, *ext)
        b = oracle.rhs(case.cfg, ext[0] * (1 + 1e-15), *ext[1:])
        n = case.n
        out[jit] = np.abs(a["drhodt"][:n] - b["drhodt"][:n]).max() / np.abs(a["drhodt"][:n]).max()
    assert out[0.0] > 1e-3
    assert out[0.1] < 1e-11


def test_plain_delta_sph_method_decays_like_taylor_green(oracle):
    """The plain method of the 100x100 Taylor-Green case (Solver_Normalized_Delta_SPH_SPS,
    Wendland C2, h = 1.3 dx, rho0 = 1, c0 = 10, Re = 100, dt = 0.25 h / c0): the reference
    committed no run of this solver, so the oracle's restatement is checked against the
    analytic decay KE/KE0 = exp(-16 pi^2 nu t).  Measured: 0.35 % below it after 80 steps
    (t = 0.026; numerical dissipation, the modified linear Riemann solver is 0.49 % below);
    bound 0.5 %, from below.  One right-hand side of the plain method must also differ
    from the modified linear Riemann solver's (the solver switch is live)."""
    case = S.make_tgv(100, solver=S.SOLVER_DELTA_SPS)
    dt = S.baseline_dt(case.cfg)
    sim = oracle.OracleSim(case.cfg, case.pos, case.vel, case.rho, case.mass, case.type)
    ke0 = sim.kinetic_energy()
    sim.run(80, dt)
    ratio = sim.kinetic_energy() / ke0
    analytic = np.exp(-16 * np.pi ** 2 * case.cfg.nu * 80 * dt)
    assert -5e-3 < (ratio - analytic) / analytic < 0.0, (ratio, analytic)
    small = S.make_tgv(32, solver=S.SOLVER_DELTA_SPS, jitter=0.1, seed=3)
    other = small.cfg.copy()
    other.solver = S.SOLVER_MODLR_DELTA_SPS
    ext = oracle.periodic_images(small.cfg, small.pos, small.vel, small.rho, small.mass, small.type)[:5]
    a = oracle.rhs(small.cfg, *ext)
    b = oracle.rhs(other, *ext)
    assert np.abs(a["drhodt"] - b["drhodt"]).max() > 1e-3 * np.abs(b["drhodt"]).max()
