"""Parity of the sm_100a FP64 path with the CPU oracle, through the C ABI.

The FP64 kernels are compiled without FMA contraction and follow the oracle's
evaluation order, so the bar is bit-for-bit equality of every cell (ghost cells
included), of the conservation registers and of the CFL numbers; mass sums
(different summation trees) must agree to 1e-12 relative.
"""
import numpy as np
import pytest

from tests.cases import DAM, SWIRL, TSUNAMI, make, swirl_dt

pytestmark = pytest.mark.gpu


def _pair(problem, **kw):
    from oracle import pyoracle as po
    import forestclaw_b200 as fb
    oc, gc = make(problem, **kw)
    o = po.OracleSim(oc)
    g = fb.Solver(gc)
    o.initialize()
    g.initialize()
    return o, g


def _same_forest(o, g):
    a, b = o.patch_info(), g.patch_info()
    assert a.shape == b.shape
    # level, gx, gy must agree slot by slot (level-major, p4est order)
    assert np.array_equal(a[:, [0, 2, 3]], b[:, [0, 2, 3]])


def _assert_bitwise(a, b, what):
    if not np.array_equal(a, b):
        diff = np.abs(a - b)
        idx = np.unravel_index(np.argmax(diff), diff.shape)
        raise AssertionError(f"{what} differs: max |diff| = {diff.max():.3e} at {idx}, "
                             f"{np.count_nonzero(a != b)} of {a.size} values differ")


def _run(o, g, dt, nsteps, regrid_every=0, cfl_target=None):
    t = 0.0
    for n in range(nsteps):
        co = o.advance(t, dt)
        cg = g.advance(t, dt)
        assert co == cg, f"step {n}: CFL {co!r} vs {cg!r}"
        _assert_bitwise(o.get_q(), g.get_q(), f"q after step {n}")
        t += dt
        if cfl_target:
            dt = dt * cfl_target / co
        if regrid_every and (n + 1) % regrid_every == 0:
            ro, rg = o.regrid(), g.regrid()
            assert ro == rg
            _same_forest(o, g)
            _assert_bitwise(o.get_q(), g.get_q(), f"q after regrid {n}")
    return t


def test_swirl_uniform_bitwise():
    o, g = _pair(SWIRL, mx=32, my=32, minlevel=2, maxlevel=2)
    _same_forest(o, g)
    _assert_bitwise(o.get_q(), g.get_q(), "initial q")
    _run(o, g, swirl_dt(32, 2), 12)


def test_swirl_16x16_bitwise():
    o, g = _pair(SWIRL, mx=16, my=16, minlevel=3, maxlevel=3)
    _run(o, g, swirl_dt(16, 3), 8)


def test_shallow_uniform_bitwise():
    o, g = _pair(DAM, mx=16, my=16, minlevel=3, maxlevel=3)
    _run(o, g, 0.004, 10)


def test_shallow_8x8_bitwise():
    o, g = _pair(DAM, mx=8, my=8, minlevel=3, maxlevel=3, mthbc=(3, 1, 3, 1))
    _run(o, g, 0.004, 6)


def test_shallow_amr_subcycle_timesync_bitwise():
    o, g = _pair(DAM, mx=16, my=16, minlevel=2, maxlevel=4, subcycle=1, time_sync=1)
    _same_forest(o, g)
    _assert_bitwise(o.get_q(), g.get_q(), "initial q")
    _run(o, g, 0.01, 8, regrid_every=2, cfl_target=0.9)
    _assert_bitwise(o.get_registers(), g.get_registers(), "conservation registers")
    mo, mg = o.mass(), g.mass()
    assert abs(mo[0] - mg[0]) <= 1e-12 * abs(mo[0])


def test_shallow_amr_no_subcycle_bitwise():
    o, g = _pair(DAM, mx=16, my=16, minlevel=2, maxlevel=4, subcycle=0, time_sync=1)
    _run(o, g, 0.004, 4, regrid_every=2)


def test_fwave_bathymetry_bitwise():
    o, g = _pair(TSUNAMI, mx=8, my=8, minlevel=2, maxlevel=4, subcycle=1, time_sync=1)
    _run(o, g, 0.01, 6, regrid_every=2, cfl_target=0.9)


def test_deterministic_repeat():
    import forestclaw_b200 as fb
    _, gc = make(DAM, mx=16, my=16, minlevel=2, maxlevel=4, subcycle=1, time_sync=1)
    outs = []
    for _ in range(2):
        g = fb.Solver(gc)
        g.initialize()
        t, dt = 0.0, 0.01
        for n in range(4):
            c = g.advance(t, dt)
            t += dt
            dt *= 0.9 / c
            if n == 1:
                g.regrid()
        outs.append(g.get_q())
        g.close()
    assert np.array_equal(outs[0], outs[1])


def test_single_step_protocol_matches_level_update():
    import forestclaw_b200 as fb
    _, gc = make(DAM, mx=16, my=16, minlevel=3, maxlevel=3)
    a, b = fb.Solver(gc), fb.Solver(gc)
    a.initialize(); b.initialize()
    np_ = a.num_patches
    ca = a.level_update(3, 0.0, 0.004)
    cb = 0.0
    for it in range(np_):
        cb = b.single_step_update(3, it, np_, 0.0, 0.004)
    assert ca == cb
    assert np.array_equal(a.get_q(), b.get_q())


# ---------------------------------------------------------------------------
# FP32-wave path: tolerance against the FP64 oracle, FP64 conservation
# ---------------------------------------------------------------------------
FP32_L1_TOL = 2e-5      # relative L1 error of every field vs the FP64 oracle


def _l1_rel(a, b, field):
    num = np.abs(a[:, field, 2:-2, 2:-2] - b[:, field, 2:-2, 2:-2]).sum()
    den = np.abs(b[:, field, 2:-2, 2:-2]).sum()
    return num / max(den, 1e-300)


def _run_fp32(problem, nsteps, dt, cfl_target=None, **kw):
    from oracle import pyoracle as po
    import forestclaw_b200 as fb
    oc, gc = make(problem, **kw)
    gc.precision = fb.PREC_FP32WAVE
    o, g = po.OracleSim(oc), fb.Solver(gc)
    o.initialize(); g.initialize()
    _same_forest(o, g)
    m0 = g.mass()
    t = 0.0
    for _ in range(nsteps):
        co = o.advance(t, dt)
        cg = g.advance(t, dt)
        assert abs(cg - co) <= 1e-4 * co
        t += dt
        if cfl_target:
            dt *= cfl_target / co
    return o, g, m0


def test_fp32wave_dam_uniform_error_and_mass():
    o, g, m0 = _run_fp32(DAM, 20, 0.004, mx=16, my=16, minlevel=4, maxlevel=4)
    qo, qg = o.get_q(), g.get_q()
    h_err = _l1_rel(qg, qo, 0)
    assert h_err < FP32_L1_TOL, h_err
    for f in (1, 2):
        assert np.abs(qg[:, f, 2:-2, 2:-2] - qo[:, f, 2:-2, 2:-2]).sum() <= FP32_L1_TOL * np.abs(qo[:, 0, 2:-2, 2:-2]).sum()
    m1 = g.mass()
    assert abs(m1[0] - m0[0]) <= 1e-12 * abs(m0[0])


def test_fp32wave_dam_amr_timesync_mass():
    o, g, m0 = _run_fp32(DAM, 8, 0.01, cfl_target=0.9, mx=16, my=16, minlevel=2, maxlevel=4, subcycle=1,
                         time_sync=1)
    qo, qg = o.get_q(), g.get_q()
    assert _l1_rel(qg, qo, 0) < FP32_L1_TOL
    m1 = g.mass()
    assert abs(m1[0] - m0[0]) <= 1e-12 * abs(m0[0])


def test_fp32wave_swirl_error():
    o, g, m0 = _run_fp32(SWIRL, 12, swirl_dt(32, 2), mx=32, my=32, minlevel=2, maxlevel=2)
    assert _l1_rel(g.get_q(), o.get_q(), 0) < FP32_L1_TOL


def test_fp32wave_fwave_error():
    o, g, m0 = _run_fp32(TSUNAMI, 6, 0.01, cfl_target=0.9, mx=8, my=8, minlevel=2, maxlevel=4, subcycle=1,
                         time_sync=1)
    qo, qg = o.get_q(), g.get_q()
    assert _l1_rel(qg, qo, 0) < FP32_L1_TOL


def test_graph_replay_matches_eager():
    """advance() replayed from the captured graph equals the eager launches, across a regrid."""
    import forestclaw_b200 as fb
    _, gc = make(DAM, mx=16, my=16, minlevel=2, maxlevel=4, subcycle=1, time_sync=1)
    outs = []
    for graphs in (True, False):
        g = fb.Solver(gc)
        g.set_graphs(graphs)
        g.initialize()
        t, dt = 0.0, 0.01
        for n in range(6):
            c = g.advance(t, dt)
            t += dt
            dt *= 0.9 / c
            if n == 2:
                g.regrid()
        outs.append((g.get_q(), g.get_registers()))
        g.close()
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])


@pytest.mark.parametrize("precision", ["fp64", "fp32wave"])
def test_programmatic_launch_matches_plain_launches(precision):
    """Programmatic dependent launch only hides launch gaps: graph replay with it
    on equals plain launches bit for bit, across a regrid, for both precisions."""
    import forestclaw_b200 as fb
    _, gc = make(DAM, mx=16, my=16, minlevel=2, maxlevel=5, subcycle=1, time_sync=1)
    if precision == "fp32wave":
        gc.precision = fb.PREC_FP32WAVE
    outs = []
    for on in (True, False):
        g = fb.Solver(gc)
        g.set_programmatic_launch(on)
        g.initialize()
        t, dt = 0.0, 0.01
        for n in range(6):
            c = g.advance(t, dt)
            t += dt
            dt *= 0.9 / c
            if n == 2:
                g.regrid()
        outs.append((g.get_q(), g.get_registers()))
        g.close()
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])


def test_fp32wave_reflecting_walls_conserve_mass():
    """Roe and f-wave solvers in the FP32-wave path with flow reaching reflecting walls.
    Once the ghost cells mirror the interior (after the first step: initialization
    fills no ghost cells, as in the reference) the mass through each wall is exactly
    zero, so the total is kept to round-off; the first step matches the FP64 path."""
    from oracle import pyoracle as po
    import forestclaw_b200 as fb
    for problem, kw in ((DAM, dict(x0=0.75, y0=-0.7)),
                        (TSUNAMI, dict(pdata=(0.0, 0.0, 1, 0.3, 0.15, 0.0, -0.8)))):
        oc, gc = make(problem, mthbc=(3, 3, 3, 3), mx=8, my=8, minlevel=2, maxlevel=4, subcycle=1, time_sync=1, **kw)
        gc.precision = fb.PREC_FP32WAVE
        o, g = po.OracleSim(oc), fb.Solver(gc)
        o.initialize(); g.initialize()
        t, dt, m1 = 0.0, 0.01, None
        for n in range(10):
            co = o.advance(t, dt)
            cg = g.advance(t, dt)
            assert abs(cg - co) <= 1e-4 * co, (problem["rp"], n, cg, co)
            if m1 is None:
                m1 = g.mass()
            t += dt
            dt *= 0.9 / co
        m = g.mass()
        assert abs(m[0] - m1[0]) <= 1e-12 * abs(m1[0]), (problem["rp"], m[0] - m1[0])
        assert _l1_rel(g.get_q(), o.get_q(), 0) < FP32_L1_TOL


def test_consecutive_level_updates_share_one_launch():
    """A subcycled coarse step over levels 2-4 updates level 4 four times, level 3
    twice and level 2 once; the updates issued back to back (4-3-2, 4, 4-3, 4) go out
    as four launches, each patch with its own level's parameters, and the result
    stays bitwise equal to the oracle (the oracle tests above run the same forests)."""
    import forestclaw_b200 as fb
    from oracle import pyoracle as po
    oc, gc = make(DAM, mx=8, my=8, minlevel=2, maxlevel=4, subcycle=1, time_sync=1)
    g = fb.Solver(gc)
    g.initialize()
    o = po.OracleSim(oc)
    o.initialize()
    levels = set(int(l) for l in g.patch_info()[:, 0])
    assert levels == {2, 3, 4}
    cg = g.advance(0.0, 0.01)
    co = o.advance(0.0, 0.01)
    st = g.last_update_stats()
    assert st["update_launches"] == 4
    assert cg == co and np.array_equal(g.get_q(), o.get_q())
    assert np.array_equal(g.get_registers(), o.get_registers())
    g.close()
