"""The oracle's cubed sphere on the CPU: connectivity, metric and properties of
the manifold advection that hold whatever the mapping's rounding.

The connectivity of the six blocks is derived from the mapping (the reference's
p4est cubed connectivity is not in its tree); the metric sums bilinear-quad
areas over finest-level sub-quads (fclaw2d_metric_default_fort.f90:110-176)."""
import math

import numpy as np

from tests.cases import SPHERE, make


def _sim(**kw):
    from oracle import pyoracle as po
    oc, _ = make(SPHERE, **kw)
    o = po.OracleSim(oc)
    o.initialize()
    return o


def test_uniform_sphere_patches_and_area():
    o = _sim(mx=8, my=8, minlevel=2, maxlevel=2)
    assert o.num_patches == 6 * 16
    aux = o.get_aux()
    info = o.patch_info()
    # kappa * dx * dy = cell area; blocks are [0,1]^2 with 2^l patches a side
    dx = 1.0 / (8 * 4)
    total = (aux[:, 0, 2:-2, 2:-2] * dx * dx).sum()
    assert abs(total - 4 * math.pi) < 2e-3 * 4 * math.pi
    # every block holds 16 patches
    assert sorted(np.bincount(info[:, 1]).tolist()) == [16] * 6


def test_sphere_area_is_consistent_across_levels():
    # a finer uniform forest with the same maxlevel sums the same sub-quads
    a = _sim(mx=8, my=8, minlevel=1, maxlevel=3)
    b = _sim(mx=8, my=8, minlevel=3, maxlevel=3)
    def total(o, lev_of):
        aux, info = o.get_aux(), o.patch_info()
        s = 0.0
        for p in range(o.num_patches):
            dx = 1.0 / (8 * 2 ** info[p, 0])
            s += (aux[p, 0, 2:-2, 2:-2] * dx * dx).sum()
        return s
    assert abs(total(a, None) - total(b, None)) < 1e-10


def test_sphere_constant_state_is_kept():
    o = _sim(mx=8, my=8, minlevel=1, maxlevel=2, subcycle=1)
    q = o.get_q()
    q[:] = 0.7
    o.set_q(q)
    t, dt = 0.0, 0.004
    for _ in range(4):
        o.advance(t, dt)
        t += dt
    q = o.get_q()
    assert np.abs(q[:, 0, 2:-2, 2:-2] - 0.7).max() == 0.0


def test_sphere_rotation_moves_the_gaussians():
    # one tenth of a revolution moves each Gaussian by 36 degrees along the equator
    o = _sim(mx=8, my=8, minlevel=2, maxlevel=2)
    q0 = o.get_q()
    t, dt = 0.0, 0.002
    while t < 0.1 - 1e-12:
        step = min(dt, 0.1 - t)
        c = o.advance(t, step)
        t += step
        dt = step * 0.9 / c
    q1 = o.get_q()
    assert q1[:, 0, 2:-2, 2:-2].max() > 0.3           # still a bump
    assert np.abs(q1 - q0)[:, 0, 2:-2, 2:-2].max() > 0.2
    assert q1[:, 0, 2:-2, 2:-2].min() > 0.09           # background stays (upwind, positive)
