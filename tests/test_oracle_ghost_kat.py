"""Known answers for the oracle's ghost fill: linear data is reproduced exactly.

Copy (same-size neighbours), average (fine -> coarse: the mean of four fine cells
of a linear field is its value at the coarse centre) and interpolation (coarse ->
fine with the limited slopes of fclaw2d_clawpatch_utils.f: for linear data the
left, right and centred differences agree, so the slope is exact) all reproduce
q = a + b x + c y at every ghost cell centre inside the domain, faces and corners,
across levels of an adaptive forest.  Ghost cells outside the domain hold
physical-BC values and are skipped, as are cells within two coarse cells of the
boundary, whose interpolation slopes see those values.  The device ghost fill is bitwise equal to
the oracle's (test_gpu_parity), so this checks it too.
"""
import numpy as np
import pytest

from tests.cases import DAM, TSUNAMI, make


def _centres(cfg, info, mx, my, mbc):
    lev, gx, gy = info[:, 0], info[:, 2], info[:, 3]
    w = (cfg.bx - cfg.ax) / (cfg.mi * 2.0 ** lev)
    h = (cfg.by - cfg.ay) / (cfg.mj * 2.0 ** lev)
    i = np.arange(mx + 2 * mbc) - mbc + 0.5
    j = np.arange(my + 2 * mbc) - mbc + 0.5
    X = cfg.ax + gx[:, None, None] * w[:, None, None] + i[None, None, :] * (w / mx)[:, None, None]
    Y = cfg.ay + gy[:, None, None] * h[:, None, None] + j[None, :, None] * (h / my)[:, None, None]
    return np.broadcast_to(X, (len(lev), my + 2 * mbc, mx + 2 * mbc)), \
        np.broadcast_to(Y, (len(lev), my + 2 * mbc, mx + 2 * mbc))


@pytest.mark.parametrize("problem,kw", [
    (DAM, dict(mx=8, my=8, minlevel=2, maxlevel=4, subcycle=1, time_sync=1)),
    (DAM, dict(mx=16, my=16, minlevel=2, maxlevel=5, subcycle=1, time_sync=1)),
    (TSUNAMI, dict(mx=8, my=8, minlevel=2, maxlevel=4, subcycle=1, time_sync=1)),
])
def test_ghost_fill_reproduces_linear_data(problem, kw):
    from oracle import pyoracle as po
    oc, _ = make(problem, **kw)
    o = po.OracleSim(oc)
    o.initialize()
    info = o.patch_info()
    assert len(set(info[:, 0].tolist())) >= 2, "the forest must be adaptive"
    mx, my, mbc = oc.mx, oc.my, oc.mbc
    X, Y = _centres(oc, info, mx, my, mbc)
    q = o.get_q()
    coef = [(1.0, 0.3, -0.2), (-0.5, 0.7, 0.4), (0.25, -0.6, 0.9)]
    lin = np.stack([a + b * X + c * Y for a, b, c in coef[:q.shape[1]]], axis=1)
    start = lin.copy()
    start[:, :, :mbc, :] = 1e30
    start[:, :, -mbc:, :] = 1e30
    start[:, :, :, :mbc] = 1e30
    start[:, :, :, -mbc:] = 1e30
    o.set_q(start)
    o.ghost_update(0.0)
    out = o.get_q()
    # cells whose interpolation stencil stays inside the domain: two coarse cells
    # (four of the patch's own) from the boundary, where physical-BC ghost cells of
    # the coarser level, which are not linear, enter the slopes
    lev = info[:, 0]
    dx = ((oc.bx - oc.ax) / (oc.mi * 2.0 ** lev) / mx)[:, None, None]
    dy = ((oc.by - oc.ay) / (oc.mj * 2.0 ** lev) / my)[:, None, None]
    inside = (X > oc.ax + 4 * dx) & (X < oc.bx - 4 * dx) & (Y > oc.ay + 4 * dy) & (Y < oc.by - 4 * dy)
    ghost = np.ones((my + 2 * mbc, mx + 2 * mbc), bool)
    ghost[mbc:-mbc, mbc:-mbc] = False
    check = inside & ghost[None]
    assert check.sum() > 0
    for m in range(q.shape[1]):
        err = np.abs(out[:, m][check] - lin[:, m][check])
        assert err.max() < 1e-12, (m, err.max())
    # every ghost cell is filled (domain-boundary ones by the physical BC)
    assert np.all(np.abs(out) < 1e29)
    # interiors untouched
    assert np.array_equal(out[:, :, mbc:-mbc, mbc:-mbc], lin[:, :, mbc:-mbc, mbc:-mbc])
