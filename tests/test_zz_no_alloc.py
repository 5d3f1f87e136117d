"""The pair search for callers that cannot allocate GPU memory.

Hosts whose GPU memory belongs to another framework (or that run where
allocation is not allowed) hand sph_find_particle_pair_noalloc their own device
buffers; the library does the search in a fixed static device array instead of
cudaMalloc.  Here the test plays that host: it owns the buffers (allocated with
torch) and checks the result against sph_find_particle_pair, twice in a row, so
that the second call proves the shared array is cleared between calls.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

import sph_b200 as S

pytestmark = pytest.mark.gpu


def _reference_pairs(cfg, case):
    with S.Simulation(cfg, case.n) as sim:
        sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)
        return sim.find_particle_pair(case.n * 20 + 1024)


def _noalloc(lib, cfg, pos_d, type_d, n, cap, out):
    cnt = ctypes.c_longlong(0)
    rc = lib.sph_find_particle_pair_noalloc(ctypes.byref(cfg), n, pos_d.data_ptr(), type_d.data_ptr(), cap,
                                            out["pi"].data_ptr(), out["pj"].data_ptr(), out["w"].data_ptr(),
                                            out["dw"].data_ptr(), ctypes.byref(cnt), None)
    return rc, cnt.value


@pytest.mark.parametrize("kw", [dict(n_side=96, jitter=0.1, seed=1), dict(n_side=64, reference=True, jitter=0.1, seed=2)])
def test_noalloc_pairs_match_allocating_entry_point(lib, kw):
    import torch
    case = S.make_tgv(**kw)
    cfg = case.cfg.copy()
    cfg.periodic = 0          # the no-alloc search works on exactly the given particles
    ref = _reference_pairs(cfg, case)
    n = case.n
    cap = ref["pair_number"] + 512
    dev = torch.device("cuda:0")
    pos_d = torch.from_numpy(case.pos.copy()).to(dev)
    type_d = torch.from_numpy(case.type.copy()).to(dev)
    for call in range(2):
        out = {"pi": torch.full((cap,), -1, dtype=torch.int32, device=dev),
               "pj": torch.full((cap,), -1, dtype=torch.int32, device=dev),
               "w": torch.zeros(cap, dtype=torch.float64, device=dev),
               "dw": torch.zeros(2 * cap, dtype=torch.float64, device=dev)}
        rc, m = _noalloc(lib, cfg, pos_d, type_d, n, cap, out)
        assert rc == 0, (call, rc)
        assert m == ref["pair_number"], (call, m)
        assert np.array_equal(out["pi"][:m].cpu().numpy(), ref["pair_i"])
        assert np.array_equal(out["pj"][:m].cpu().numpy(), ref["pair_j"])
        # same kernel code on the same FP64 inputs: w and dwdx agree to round-off
        np.testing.assert_allclose(out["w"][:m].cpu().numpy(), ref["w"], rtol=1e-12, atol=0)
        dw = out["dw"].cpu().numpy()
        got = np.stack([dw[:m], dw[cap:cap + m]])
        assert np.abs(got - ref["dwdx"]).max() <= 1e-12 * np.abs(ref["dwdx"]).max()


def test_noalloc_rejects_sizes_beyond_the_static_limit(lib):
    import torch
    case = S.make_tgv(260)        # 67,600 particles > 65,536
    dev = torch.device("cuda:0")
    pos_d = torch.from_numpy(case.pos.copy()).to(dev)
    type_d = torch.from_numpy(case.type.copy()).to(dev)
    out = {k: torch.zeros(16, dtype=torch.int32 if k in ("pi", "pj") else torch.float64, device=dev)
           for k in ("pi", "pj", "w", "dw")}
    rc, _ = _noalloc(lib, case.cfg, pos_d, type_d, case.n, 8, out)
    assert rc == -2   # SPH_E_CAPACITY


def _device_case(kw):
    import torch
    case = S.make_tgv(**kw)
    cfg = case.cfg.copy()
    cfg.periodic = 0
    dev = torch.device("cuda:0")
    pos_d = torch.from_numpy(case.pos.copy()).to(dev)
    type_d = torch.from_numpy(case.type.copy()).to(dev)
    return case, cfg, pos_d, type_d


def _outputs(cap):
    import torch
    dev = torch.device("cuda:0")
    return {"pi": torch.full((max(cap, 1),), -1, dtype=torch.int32, device=dev),
            "pj": torch.full((max(cap, 1),), -1, dtype=torch.int32, device=dev),
            "w": torch.zeros(max(cap, 1), dtype=torch.float64, device=dev),
            "dw": torch.zeros(2 * max(cap, 1), dtype=torch.float64, device=dev)}


def test_noalloc_count_only_then_emit(lib):
    """pair_cap = 0 counts (SPH_OK, as sph_find_particle_pair); a second call
    with exactly that capacity emits the same pairs."""
    case, cfg, pos_d, type_d = _device_case(dict(n_side=48, jitter=0.1, seed=4))
    ref = _reference_pairs(cfg, case)
    rc, m = _noalloc(lib, cfg, pos_d, type_d, case.n, 0, _outputs(0))
    assert rc == 0 and m == ref["pair_number"]
    out = _outputs(m)
    rc, m2 = _noalloc(lib, cfg, pos_d, type_d, case.n, m, out)
    assert rc == 0 and m2 == m
    assert np.array_equal(out["pi"][:m].cpu().numpy(), ref["pair_i"])
    assert np.array_equal(out["pj"][:m].cpu().numpy(), ref["pair_j"])


def test_noalloc_short_capacity_fills_the_prefix(lib):
    """A pair_cap below the count returns SPH_E_CAPACITY with the full count and
    the first pair_cap pairs in the reference's order."""
    case, cfg, pos_d, type_d = _device_case(dict(n_side=40, jitter=0.1, seed=6))
    ref = _reference_pairs(cfg, case)
    cap = ref["pair_number"] // 3
    out = _outputs(cap)
    rc, m = _noalloc(lib, cfg, pos_d, type_d, case.n, cap, out)
    assert rc == -2 and m == ref["pair_number"]
    assert np.array_equal(out["pi"].cpu().numpy(), ref["pair_i"][:cap])
    assert np.array_equal(out["pj"].cpu().numpy(), ref["pair_j"][:cap])


def test_noalloc_particle_outside_the_grid(lib):
    import torch
    case, cfg, pos_d, type_d = _device_case(dict(n_side=32))
    pos = case.pos.copy()
    pos[9] = cfg.grid_hi[0] + 1.0
    pos_d = torch.from_numpy(pos).to(pos_d.device)
    rc, _ = _noalloc(lib, cfg, pos_d, type_d, case.n, 16, _outputs(16))
    assert rc == -8   # SPH_E_DOMAIN


def test_noalloc_per_particle_limit(lib):
    """More than 256 pairs (i, j > i) for one particle: SPH_E_CAPACITY with a
    count of -1, which tells the caller that a larger pair_cap will not help."""
    import torch
    case = S.make_tgv(16)
    cfg = case.cfg.copy()
    cfg.periodic = 0
    n = 300
    ang = 2.0 * np.pi * np.arange(n) / n
    r = 0.1 * cfg.h
    pos = np.concatenate([0.5 + r * np.cos(ang), 0.5 + r * np.sin(ang)])
    dev = torch.device("cuda:0")
    pos_d = torch.from_numpy(pos).to(dev)
    type_d = torch.full((n,), S.TYPE_WATER, dtype=torch.int32, device=dev)
    cap = n * n
    rc, m = _noalloc(lib, cfg, pos_d, type_d, n, cap, _outputs(cap))
    assert rc == -2 and m == -1
    # a valid input afterwards works (the array is cleared per call)
    case2, cfg2, pos2, type2 = _device_case(dict(n_side=24, jitter=0.1, seed=8))
    ref = _reference_pairs(cfg2, case2)
    out = _outputs(ref["pair_number"])
    rc, m = _noalloc(lib, cfg2, pos2, type2, case2.n, ref["pair_number"], out)
    assert rc == 0 and m == ref["pair_number"]
    assert np.array_equal(out["pj"].cpu().numpy(), ref["pair_j"])
