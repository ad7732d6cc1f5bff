"""Patch-to-CTA variants of the fused update and the autotuner.

Every variant maps the same per-interface arithmetic onto a CTA differently
(threads per CTA, occupancy target, one thread per interface or a strided
loop), so the FP64 variants must give the oracle's bits, and the FP32-wave
variants must agree with each other to FP32 accuracy.  The autotuner times the
variants with dt = 0 and must leave q untouched.
"""
import numpy as np
import pytest

from tests.cases import DAM, SHOCKBUBBLE, TSUNAMI, make

pytestmark = pytest.mark.gpu


def _solver(problem, precision=None, **kw):
    import forestclaw_b200 as fb
    _, gc = make(problem, **kw)
    if precision is not None:
        gc.precision = precision
    g = fb.Solver(gc)
    g.initialize()
    return g


def _run(g, dt, nsteps, regrid_every=0):
    t = 0.0
    for n in range(nsteps):
        c = g.advance(t, dt)
        t += dt
        dt *= 0.9 / c
        if regrid_every and (n + 1) % regrid_every == 0:
            g.regrid()
    return g.get_q()


@pytest.mark.parametrize("problem,kw", [
    (DAM, dict(mx=16, my=16, minlevel=2, maxlevel=4, subcycle=1, time_sync=1)),
    (DAM, dict(mx=8, my=8, minlevel=2, maxlevel=4, subcycle=1, time_sync=1)),
    (TSUNAMI, dict(mx=8, my=8, minlevel=2, maxlevel=4, subcycle=1, time_sync=1)),
])
def test_fp64_variants_match_oracle_bitwise(problem, kw):
    from oracle import pyoracle as po
    oc, _ = make(problem, **kw)
    o = po.OracleSim(oc)
    o.initialize()
    ref = _run(o, 0.01, 4, regrid_every=2)
    nv = len(_solver(problem, **kw).variants())
    assert nv >= 3
    for v in range(nv):
        g = _solver(problem, **kw)
        g.set_variant(v)
        q = _run(g, 0.01, 4, regrid_every=2)
        assert np.array_equal(q, ref), f"variant {v} {g.variants()[v]} differs from the oracle"


def test_fp32wave_variants_agree():
    import forestclaw_b200 as fb
    kw = dict(mx=16, my=16, minlevel=2, maxlevel=4, subcycle=1, time_sync=1)
    g0 = _solver(DAM, fb.PREC_FP32WAVE, **kw)
    ref = _run(g0, 0.01, 4)
    m0 = g0.mass()
    for v in range(1, len(g0.variants())):
        g = _solver(DAM, fb.PREC_FP32WAVE, **kw)
        g.set_variant(v)
        q = _run(g, 0.01, 4)
        h = slice(2, -2)
        err = np.abs(q[:, 0, h, h] - ref[:, 0, h, h]).sum() / np.abs(ref[:, 0, h, h]).sum()
        assert err < 1e-6, (v, err)
        assert abs(g.mass()[0] - m0[0]) <= 1e-12 * abs(m0[0])


@pytest.mark.parametrize("problem,kw", [
    (DAM, dict(mx=16, my=16, minlevel=2, maxlevel=4, subcycle=1, time_sync=1)),
    (SHOCKBUBBLE, dict(mx=8, my=8, minlevel=2, maxlevel=3, subcycle=1)),
])
def test_autotune_leaves_state_and_picks_a_variant(problem, kw):
    g = _solver(problem, **kw)
    _run(g, 0.002, 2)
    q0, r0 = g.get_q(), g.get_registers()
    best, ms = g.autotune(reps=2)
    assert 0 <= best < len(ms) and g.variant == best
    assert np.all(ms > 0) and ms[best] == ms.min()
    # per-level choices: a compiled variant for every level present
    lv = g.level_variants()
    for l in set(int(x) for x in g.patch_info()[:, 0]):
        assert 0 <= lv[l] < len(ms)
    assert np.array_equal(g.get_q(), q0) and np.array_equal(g.get_registers(), r0)
    # the tuned solver continues exactly like an untuned one
    h = _solver(problem, **kw)
    _run(h, 0.002, 2)
    assert np.array_equal(_run(g, 0.002, 2), _run(h, 0.002, 2))


def test_level_variants_carry_over_to_a_new_solver():
    """A tuned solver's per-level choice applied to a fresh solver of the same shape
    (fc2d_b200_set_level_variants): the same variants, the same trajectory, and an
    index outside the compiled variants is refused."""
    import forestclaw_b200 as fb
    kw = dict(mx=16, my=16, minlevel=2, maxlevel=4, subcycle=1, time_sync=1)
    g = _solver(DAM, fb.PREC_FP32WAVE, **kw)
    _run(g, 0.002, 2)
    g.autotune(reps=1)
    lv = g.level_variants()
    h = _solver(DAM, fb.PREC_FP32WAVE, **kw)
    _run(h, 0.002, 2)
    h.set_level_variants(lv)
    assert np.array_equal(h.level_variants(), lv)
    assert np.array_equal(_run(g, 0.002, 2), _run(h, 0.002, 2))
    bad = lv.copy()
    bad[3] = len(g.variants())
    with pytest.raises(fb.B200Error):
        h.set_level_variants(bad)
    assert np.array_equal(h.level_variants(), lv)
