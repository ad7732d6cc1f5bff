"""Known-answer tests of the CPU oracle (no GPU).

The reference pins no field values (its regression files only count AMR events),
so the oracle is pinned by the mathematics of the method: limiter formulas,
exact preservation of a state at rest, exact translation at CFL 1, conservation
to round-off with the time-sync correction, symmetry, and committed fixtures that
freeze the oracle's own output (tests/golden, regenerated by make_golden.py).
"""
import os

import numpy as np
import pytest

from tests.cases import DAM, SWIRL, TSUNAMI, make, swirl_dt

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_limiter_formulas(oracle_lib):
    po = oracle_lib
    for r in (-2.0, -0.5, 0.0, 0.3, 0.5, 1.0, 1.7, 3.0, 10.0):
        assert po.limiter_phi(1, r) == max(0.0, min(1.0, r))
        assert po.limiter_phi(2, r) == max(0.0, min(1.0, 2 * r), min(2.0, r))
        assert po.limiter_phi(3, r) == (r + abs(r)) / (1.0 + abs(r))
        assert po.limiter_phi(4, r) == max(0.0, min((1.0 + r) / 2.0, 2.0, 2.0 * r))
        assert po.limiter_phi(5, r) == r
        th = float(np.float32(1.3))
        assert po.limiter_phi(6, r) == max(0.0, min(th * r, (1 + r) / 2.0, th))


def _patch(meqn, mx=16, mbc=2):
    n = mx + 2 * mbc
    return np.zeros((meqn, n, n), np.float64)


def test_translation_at_cfl_one(oracle_lib):
    """First-order upwind with u = 1, v = 0 and dt = dx shifts q by one cell exactly."""
    po = oracle_lib
    cfg = po.make_config(mx=16, my=16, mbc=2, meqn=1, maux=2, mwaves=1, mthlim=(0,), order=(1, 0), rp=0)
    rng = np.random.default_rng(0)
    q = rng.random((1, 20, 20))
    aux = np.zeros((2, 20, 20))
    aux[0] = 1.0
    q0 = q.copy()
    dx = 1.0 / 16
    cfl, *_ = po.patch_step2(cfg, q, aux, dx, dx, dx)
    assert cfl == 1.0
    # interior cells i=1..mx (padded 2..17): q_new(i) = q_old(i-1)
    assert np.array_equal(q[0, 2:18, 2:18], q0[0, 2:18, 1:17])


def test_state_at_rest_preserved_amr(oracle_lib):
    po = oracle_lib
    oc, _ = make(DAM, mx=16, my=16, minlevel=2, maxlevel=4, subcycle=1, time_sync=1, hin=1.0, hout=1.0,
                 refine_threshold=-1.0)
    s = po.OracleSim(oc)
    s.initialize()
    t, dt = 0.0, 0.01
    for _ in range(3):
        s.advance(t, dt)
        t += dt
    q = s.get_q()
    interior = q[:, :, 2:-2, 2:-2]
    assert np.all(interior[:, 0] == 1.0)
    assert np.all(interior[:, 1:] == 0.0)


def test_swirl_mass_conserved(oracle_lib):
    po = oracle_lib
    oc, _ = make(SWIRL, mx=32, my=32, minlevel=2, maxlevel=2)
    s = po.OracleSim(oc)
    s.initialize()
    m0 = s.mass()
    dt = swirl_dt(32, 2)
    t = 0.0
    for _ in range(20):
        s.advance(t, dt)
        t += dt
    m1 = s.mass()
    assert abs(m1[0] - m0[0]) <= 1e-14 * abs(m0[0])


@pytest.mark.parametrize("time_sync", [1, 0])
def test_dam_amr_conservation(oracle_lib, time_sync):
    """With time sync the subcycled AMR run conserves h to 1e-12; without it, it does not."""
    po = oracle_lib
    oc, _ = make(DAM, mx=16, my=16, minlevel=2, maxlevel=4, subcycle=1, time_sync=time_sync)
    s = po.OracleSim(oc)
    s.initialize()
    m0 = s.mass()
    t, dt = 0.0, 0.01
    for n in range(8):
        c = s.advance(t, dt)
        t += dt
        dt *= 0.9 / c
        if n % 2 == 1:
            s.regrid()
    rel = abs(s.mass()[0] - m0[0]) / abs(m0[0])
    if time_sync:
        assert rel <= 1e-12
    else:
        assert rel > 1e-12


def test_dam_transpose_symmetry(oracle_lib):
    """The radial dam is symmetric under x <-> y (with hu <-> hv) to round-off."""
    po = oracle_lib
    oc, _ = make(DAM, mx=16, my=16, minlevel=3, maxlevel=3)
    s = po.OracleSim(oc)
    s.initialize()
    t, dt = 0.0, 0.005
    for _ in range(10):
        s.advance(t, dt)
        t += dt
    q = s.get_q()
    info = s.patch_info()
    n = 8
    h = np.zeros((n * 16, n * 16))
    hu = np.zeros_like(h)
    hv = np.zeros_like(h)
    for k, (lev, blk, gx, gy) in enumerate(info):
        h[gy * 16:(gy + 1) * 16, gx * 16:(gx + 1) * 16] = q[k, 0, 2:-2, 2:-2]
        hu[gy * 16:(gy + 1) * 16, gx * 16:(gx + 1) * 16] = q[k, 1, 2:-2, 2:-2]
        hv[gy * 16:(gy + 1) * 16, gx * 16:(gx + 1) * 16] = q[k, 2, 2:-2, 2:-2]
    assert np.max(np.abs(h - h.T)) < 1e-12
    assert np.max(np.abs(hu - hv.T)) < 1e-12
    # 180 degree rotation: h(-x,-y) = h(x,y)
    assert np.max(np.abs(h - h[::-1, ::-1])) < 1e-12


def _load(name):
    return np.load(os.path.join(GOLDEN, name))


@pytest.mark.parametrize("case", ["swirl_l2_32", "dam_amr_l2_4", "tsunami_amr_8"])
def test_oracle_matches_committed_fixture(oracle_lib, case):
    """Freezes the oracle: its output must not change unless the fixtures are regenerated."""
    from tests.golden.make_golden import run_case
    ref = _load(case + ".npz")
    out = run_case(case)
    assert np.array_equal(out["info"], ref["info"])
    assert np.array_equal(out["cfl"], ref["cfl"])
    assert np.array_equal(out["q"], ref["q"])
