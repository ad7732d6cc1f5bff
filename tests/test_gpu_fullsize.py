"""Parity at the benchmark configurations' full sizes.

C1 exactly as stated (swirl, uniform level 4 of 32x32 patches, 200 steps), C2 at
its levels 3-7 with subcycling, time sync and a regrid every 4 coarse steps for 20
coarse steps, and C4 at its levels 4-8, each FP64 and bit for bit against the
oracle.  The FP32-wave form of C2 is held to per-field error bounds against the
oracle: relative L1 (sum |dq| area / sum |q| area) <= 2e-5, relative Linf
(max |dq| / max |q|) <= 1e-4, and mass (the sum of h times the cell areas) equal
to 1e-12 relative."""
import numpy as np
import pytest

from tests.cases import DAM, SHOCKBUBBLE, SWIRL, make, swirl_dt

pytestmark = pytest.mark.gpu


def _pair(problem, **kw):
    from oracle import pyoracle as po
    import forestclaw_b200 as fb
    oc, gc = make(problem, **kw)
    o = po.OracleSim(oc)
    g = fb.Solver(gc)
    o.initialize()
    g.initialize()
    assert np.array_equal(o.patch_info()[:, [0, 2, 3]], g.patch_info()[:, [0, 2, 3]])
    return o, g


def _bitwise(a, b, what):
    if not np.array_equal(a, b):
        d = np.abs(a - b)
        raise AssertionError(f"{what}: max |diff| {d.max():.3e}, {np.count_nonzero(a != b)} of {a.size} differ")


def test_c1_swirl_level4_32x32_200_steps_bitwise():
    o, g = _pair(SWIRL, mx=32, my=32, minlevel=4, maxlevel=4)
    assert g.num_patches == 256
    dt, t = swirl_dt(32, 4), 0.0
    for n in range(200):
        co, cg = o.advance(t, dt), g.advance(t, dt)
        assert co == cg, (n, co, cg)
        t += dt
        if (n + 1) % 50 == 0:
            _bitwise(o.get_q(), g.get_q(), f"q after step {n + 1}")
    g.close()


def _dam_run(o, g, nsteps, regrid_every):
    t, dt = 0.0, 0.002
    for n in range(nsteps):
        co, cg = o.advance(t, dt), g.advance(t, dt)
        assert co == cg, (n, co, cg)
        t += dt
        dt = dt * 0.9 / co
        if regrid_every and (n + 1) % regrid_every == 0:
            assert o.regrid() == g.regrid()
            assert np.array_equal(o.patch_info()[:, [0, 2, 3]], g.patch_info()[:, [0, 2, 3]])
            _bitwise(o.get_q(), g.get_q(), f"q after regrid at step {n + 1}")
    return t


def test_c2_radialdam_levels_3_7_20_steps_regrid_bitwise():
    o, g = _pair(DAM, mx=16, my=16, minlevel=3, maxlevel=7, subcycle=1, time_sync=1)
    _dam_run(o, g, 20, 4)
    _bitwise(o.get_q(), g.get_q(), "q after 20 coarse steps")
    _bitwise(o.get_registers(), g.get_registers(), "conservation registers")
    mo, mg = o.mass(), g.mass()
    # per field to 1e-12 of the depth's mass (the momenta sum to round-off around zero)
    assert np.all(np.abs(mo - mg) <= 1e-12 * abs(mo[0])), (mo, mg)
    g.close()


def test_c4_shockbubble_levels_4_8_bitwise():
    o, g = _pair(SHOCKBUBBLE, mx=16, my=16, minlevel=4, maxlevel=8, subcycle=1)
    t, dt = 0.0, 2e-4
    for n in range(3):
        co, cg = o.advance(t, dt), g.advance(t, dt)
        assert co == cg, (n, co, cg)
        t += dt
        dt = dt * 0.9 / co
    _bitwise(o.get_q(), g.get_q(), "q after 3 coarse steps")
    g.close()


def error_vs_oracle(qg, qo, area):
    """Per-field relative L1 and Linf of qg against qo, and (for the caller) the masses."""
    d = np.abs(qg - qo)
    w = area[:, None, None, None]
    l1 = (d * w).sum(axis=(0, 2, 3)) / np.maximum((np.abs(qo) * w).sum(axis=(0, 2, 3)), 1e-300)
    linf = d.max(axis=(0, 2, 3)) / np.maximum(np.abs(qo).max(axis=(0, 2, 3)), 1e-300)
    return l1, linf


def test_c2_fp32wave_error_bounds_against_oracle():
    import forestclaw_b200 as fb
    o, g = _pair(DAM, mx=16, my=16, minlevel=3, maxlevel=7, subcycle=1, time_sync=1,
                 precision=fb.PREC_FP32WAVE)
    t, dt = 0.0, 0.002
    for n in range(8):                              # one forest: no regrid, the same dt
        co = o.advance(t, dt)
        g.advance(t, dt)
        t += dt
    info = o.patch_info()
    mbc = 2
    inner = (slice(None), slice(None), slice(mbc, -mbc), slice(mbc, -mbc))
    dx = 2.0 / (16 * 2.0 ** info[:, 0])
    l1, linf = error_vs_oracle(g.get_q()[inner], o.get_q()[inner], dx * dx)
    assert np.all(l1 <= 2e-5), l1
    assert np.all(linf <= 1e-4), linf
    mo, mg = o.mass(), g.mass()
    assert abs(mg[0] - mo[0]) <= 1e-12 * abs(mo[0]), (mo, mg)          # mass (h)
    g.close()
