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
