"""The cubed sphere on the B200 against the CPU oracle.

The device metric (areas from finest-level sub-quads, capacity, edge velocities
from stream-function differences) uses the same fixed-order arithmetic as the
oracle, so aux is bit for bit equal; the FP64 update with fix_corners at the
cube corners, the ghost fill across rotated block faces (copy, area-weighted
average, interpolation) and the manifold regrid (fixcapaq2, area-weighted
average2coarse) are bitwise equal too, ghost cells included.
"""
import numpy as np
import pytest

from tests.cases import SPHERE, make

pytestmark = pytest.mark.gpu


def _pair(**kw):
    from oracle import pyoracle as po
    import forestclaw_b200 as fb
    oc, gc = make(SPHERE, **kw)
    o = po.OracleSim(oc)
    g = fb.Solver(gc)
    o.initialize()
    g.initialize()
    return o, g


def _same(o, g, what):
    a, b = o.patch_info(), g.patch_info()
    assert a.shape == b.shape and np.array_equal(a[:, [0, 2, 3]], b[:, [0, 2, 3]]), f"{what}: forest differs"
    qo, qg = o.get_q(), g.get_q()
    if not np.array_equal(qo, qg):
        d = np.abs(qo - qg)
        raise AssertionError(f"{what}: q differs, max {d.max():.3e} at {np.unravel_index(d.argmax(), d.shape)}, "
                             f"{np.count_nonzero(d)} values")


def test_sphere_metric_bitwise():
    o, g = _pair(mx=8, my=8, minlevel=1, maxlevel=3)
    assert np.array_equal(o.get_aux(), g.get_aux())
    _same(o, g, "initial")


@pytest.mark.parametrize("kw", [dict(minlevel=2, maxlevel=2), dict(minlevel=1, maxlevel=3, subcycle=1)])
def test_sphere_fp64_bitwise(kw):
    o, g = _pair(mx=8, my=8, **kw)
    t, dt = 0.0, 0.004
    for n in range(8):
        co, cg = o.advance(t, dt), g.advance(t, dt)
        assert co == cg, (n, co, cg)
        _same(o, g, f"step {n}")
        t += dt
        dt *= 0.9 / co
        if kw["maxlevel"] > kw["minlevel"] and (n + 1) % 2 == 0:
            assert o.regrid() == g.regrid()
            _same(o, g, f"regrid after step {n}")
            assert np.array_equal(o.get_aux(), g.get_aux()), "aux after regrid"
    np.testing.assert_allclose(g.mass(), o.mass(), rtol=1e-12)


def test_sphere_fp32wave_error():
    import forestclaw_b200 as fb
    from oracle import pyoracle as po
    oc, gc = make(SPHERE, mx=8, my=8, minlevel=1, maxlevel=3, subcycle=1)
    gc.precision = fb.PREC_FP32WAVE
    o, g = po.OracleSim(oc), fb.Solver(gc)
    o.initialize(); g.initialize()
    t, dt = 0.0, 0.004
    for n in range(8):
        co, cg = o.advance(t, dt), g.advance(t, dt)
        assert abs(cg - co) <= 1e-5 * co
        t += dt
        dt *= 0.9 / co
    qo, qg = o.get_q()[:, 0, 2:-2, 2:-2], g.get_q()[:, 0, 2:-2, 2:-2]
    assert np.abs(qo - qg).sum() / np.abs(qo).sum() < 2e-6
    np.testing.assert_allclose(g.mass(), o.mass(), rtol=1e-9)
