"""The oracle's MLS density re-initialisation reproduces the fields its basis
spans: quadratic densities exactly with the quadratic basis (order 6),
linear ones with the linear basis (order 3, moving-square variant), for every
particle whose support lies inside the particle block."""
import numpy as np
import pytest

import sph_b200 as S


@pytest.mark.parametrize("order", [6, 3])
def test_mls_reproduces_its_basis(oracle, order):
    case = S.make_tgv(32, reference=True, jitter=0.1, seed=3)
    cfg = case.cfg.copy()
    cfg.periodic = 0
    cfg.mls_order = order
    if order == 3:
        cfg.solver = S.SOLVER_MS_MODLR_DELTA      # the moving-square variant (self included, W V)
    n = case.n
    x, y = case.pos[:n], case.pos[n:]
    f = 1000.0 + 3 * x - 2 * y
    if order == 6:
        f = f + 5 * x * x - 4 * x * y + 7 * y * y
    out = oracle.mls_reinit(cfg, case.pos, f, case.mass, case.type)
    r = cfg.kernel_scale * cfg.h * 1.01
    inner = (x > r) & (x < 1 - r) & (y > r) & (y < 1 - r)
    assert inner.sum() > 400
    assert np.abs(out - f)[inner].max() <= 1e-11 * 1000.0
    # near the block edge the fit is one-sided but still close
    assert np.abs(out - f).max() <= 1e-8 * 1000.0
