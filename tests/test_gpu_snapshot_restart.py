"""Snapshot streaming (sph_snapshot_begin / query / wait) and the exact restart
image (sph_restart_save / sph_restart_load).

A snapshot holds the state of the moment it was queued, bit for bit, even when
more steps run while its transfer is in flight; a handle restored from a
restart image continues bit-identically to the one that saved it, across the
first-step rate evaluation, the carried rates, MLS density re-initialisation,
shifting, periodic images, and the moving-square ghost assignment with a moving
body and the physical time."""
import numpy as np
import pytest

import sph_b200 as S

pytestmark = pytest.mark.gpu


def _pinned(n):
    import torch
    return torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()


def test_snapshot_holds_the_state_of_its_moment(lib):
    case = S.make_tgv(128, solver=S.SOLVER_MUSCL_DELTA_SPS, jitter=0.05, seed=3)
    dt = S.baseline_dt(case.cfg)
    n = case.n
    with S.Simulation(case.cfg, n) as sim:
        sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)
        sim.time_iteration(3, dt)
        ref = sim.get_state()
        bufs = [_pinned(2 * n), _pinned(2 * n), _pinned(n), _pinned(n)]
        sim.snapshot_begin(*bufs)
        sim.time_iteration(5, dt)                 # runs while the transfer may be in flight
        sim.snapshot_wait()
        assert sim.snapshot_query()
        later = sim.get_state()
    for a, b in zip(bufs[:3], ref[:3]):
        assert np.array_equal(a, b)
    assert np.allclose(bufs[3], ref[3], rtol=1e-15, atol=1e-12)
    assert not np.array_equal(later[1], ref[1])
    # pageable buffers work too (the transfer completes within the call)
    with S.Simulation(case.cfg, n) as sim:
        sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)
        v = np.empty(2 * n)
        sim.snapshot_begin(None, v, None, None)
        sim.snapshot_wait()
        assert np.array_equal(v, case.vel)


def _continue_check(cfg, n, setup, k, dt):
    with S.Simulation(cfg, n) as sim:
        setup(sim)
        sim.time_iteration(2 * k, dt)
        want = sim.get_state()
    with S.Simulation(cfg, n) as sim:
        setup(sim)
        sim.time_iteration(k, dt)
        image = sim.restart_save()
    assert len(image) == 64 + 108 * n
    with S.Simulation(cfg, n) as sim:
        sim.restart_load(image)
        sim.time_iteration(k, dt)
        got = sim.get_state()
    for a, b in zip(got, want):
        assert np.array_equal(a, b)


def test_restart_continues_bit_identically_taylor_green(lib):
    case = S.make_tgv(64, reference=True, jitter=0.05, seed=5)   # shifting, MLS every 20 steps
    dt = S.baseline_dt(case.cfg)

    def setup(sim):
        sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)

    _continue_check(case.cfg, case.n, setup, 12, dt)


def test_restart_continues_bit_identically_moving_square(lib):
    case, ity = S.make_moving_square(solver=S.SOLVER_MS_HLLC_DELTA, jitter=0.05, seed=9)
    case.cfg.ghost_assign = 1
    lab = S.moving_square_labels(case, ity)
    dt = 0.25 * case.cfg.h / np.sqrt(case.cfg.c0sq)

    def setup(sim):
        sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)
        sim.set_initial_type(ity)
        sim.set_boundary_labels(lab)
        sim.set_body_motion((1.0, 0.0), (0.5, 0.0))
        sim.set_time(0.25)

    _continue_check(case.cfg, case.n, setup, 6, dt)


def test_restart_load_rejects_bad_images(lib):
    case = S.make_tgv(16)
    with S.Simulation(case.cfg, case.n) as sim:
        sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)
        image = bytearray(sim.restart_save())
        with pytest.raises(S.SphError):
            sim.restart_load(bytes(image[:100]))
        image[0:8] = b"XXXXXXXX"
        with pytest.raises(S.SphError):
            sim.restart_load(bytes(image))
    with S.Simulation(case.cfg, case.n // 2) as small:
        with pytest.raises(S.SphError) as e:
            small.restart_load(sim_image := bytes(bytearray(b"SPHB200R") + bytes(image[8:])))
        assert e.value.code == -2
