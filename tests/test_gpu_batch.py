"""Batches of independent forests: one solver holding several tsunami instances
(own levels, bathymetry, humps and time step each) must reproduce, instance by
instance, the oracle running each instance alone -- bit for bit in FP64 (every
cell, ghost cells included, and every CFL number), across regrids.  The
FP32-wave batch must conserve each instance's mass on its own to 1e-12.
"""
import numpy as np
import pytest

from tests.cases import TSUNAMI, make

pytestmark = pytest.mark.gpu

# (minlevel, maxlevel, pdata): bathymetry centre, number of humps, [A, w, x, y] per hump
INSTANCES = [
    (2, 4, (0.1, -0.2, 2, 0.2, 0.1, 0.3, 0.2, 0.1, 0.15, -0.4, -0.3)),
    (3, 5, (-0.3, 0.25, 1, 0.25, 0.12, -0.2, 0.1)),
    (2, 3, (0.0, 0.0, 3, 0.1, 0.08, 0.5, 0.5, 0.15, 0.1, -0.5, 0.2, 0.05, 0.2, 0.0, -0.6)),
    (3, 3, (0.2, 0.2, 1, 0.3, 0.15, 0.0, 0.0)),
]
COMMON = dict(mx=8, my=8, subcycle=1, time_sync=1)


def _batch(precision=None, **kw):
    import forestclaw_b200 as fb
    opts = dict(COMMON, **kw)
    if precision is not None:
        opts["precision"] = precision
    _, gc = make(TSUNAMI, minlevel=0, maxlevel=0, **opts)
    g = fb.Solver(gc)
    g.set_instances([dict(minlevel=lo, maxlevel=hi, pdata=pd, ax=-1.0, bx=1.0, ay=-1.0, by=1.0, mi=1, mj=1)
                     for lo, hi, pd in INSTANCES])
    g.initialize()
    return g


def _oracles(**kw):
    from oracle import pyoracle as po
    sims = []
    for lo, hi, pd in INSTANCES:
        oc, _ = make(TSUNAMI, minlevel=lo, maxlevel=hi, pdata=pd, **dict(COMMON, **kw))
        o = po.OracleSim(oc)
        o.initialize()
        sims.append(o)
    return sims


def _split(g):
    """Patch slots of each instance, in batch order (level-major within an instance)."""
    inst = g.patch_instance()
    return [np.nonzero(inst == i)[0] for i in range(len(INSTANCES))]


def _check_same(sims, g, what):
    q = g.get_q()
    info = g.patch_info()
    for i, (o, slots) in enumerate(zip(sims, _split(g))):
        oi = o.patch_info()
        assert len(slots) == len(oi), f"{what}: instance {i} has {len(slots)} patches, oracle {len(oi)}"
        assert np.array_equal(oi[:, [0, 2, 3]], info[slots][:, [0, 2, 3]]), f"{what}: instance {i} forest differs"
        qo = o.get_q()
        if not np.array_equal(qo, q[slots]):
            d = np.abs(qo - q[slots])
            raise AssertionError(f"{what}: instance {i} q differs, max {d.max():.3e}, "
                                 f"{np.count_nonzero(d)} values")


def test_batch_matches_standalone_runs_bitwise():
    g = _batch()
    sims = _oracles()
    _check_same(sims, g, "initial")
    dt = np.array([0.01, 0.008, 0.012, 0.006])
    t = np.zeros(len(INSTANCES))
    for n in range(6):
        cfl = g.advance_instances(dt)
        for i, o in enumerate(sims):
            co = o.advance(t[i], dt[i])
            assert co == cfl[i], f"step {n} instance {i}: CFL {co!r} vs {cfl[i]!r}"
        _check_same(sims, g, f"step {n}")
        t += dt
        dt = dt * 0.9 / cfl
        if n == 2:
            g.regrid()
            for o in sims:
                o.regrid()
            _check_same(sims, g, f"regrid after step {n}")
    m = g.mass_instances()
    for i, o in enumerate(sims):
        np.testing.assert_allclose(m[i], o.mass(), rtol=1e-12, atol=1e-14)


def test_batch_fp32wave_conserves_each_instance():
    import forestclaw_b200 as fb
    g = _batch(precision=fb.PREC_FP32WAVE, mthbc=(3, 3, 3, 3))
    dt = np.array([0.01, 0.008, 0.012, 0.006])
    m0 = None
    for n in range(6):
        cfl = g.advance_instances(dt)
        assert np.all(np.isfinite(cfl)) and np.all(cfl < 1.0)
        if m0 is None:
            # the first step runs on qinit's ghost cells (no ghost fill at initialization,
            # as in the reference), which are no mirror images at the walls
            m0 = g.mass_instances()
        dt = dt * 0.9 / cfl
        if n == 3:
            g.regrid()
    m = g.mass_instances()
    np.testing.assert_allclose(m[:, 0], m0[:, 0], rtol=1e-12)
