"""Kernel-side failures come back as FC2D_B200_EDEVICE with the device status word's
reason, and the solver stays usable.  The failures are made on the host: bad values
are written into q through the ABI before a step (no kernel is made to fault)."""
import numpy as np
import pytest

from tests.cases import DAM, SHOCKBUBBLE, make

pytestmark = pytest.mark.gpu
EDEVICE = -4


def _solver(problem, **kw):
    import forestclaw_b200 as fb
    _, gc = make(problem, **kw)
    g = fb.Solver(gc)
    g.initialize()
    return g


def _expect_device_error(g, match, dt):
    import forestclaw_b200 as fb
    with pytest.raises(fb.B200Error, match=match) as e:
        g.advance(0.0, dt)
    assert e.value.code == EDEVICE


@pytest.mark.parametrize("precision", [0, 1])
def test_negative_depth_is_reported(precision):
    g = _solver(DAM, mx=16, my=16, minlevel=2, maxlevel=3, subcycle=1, precision=precision)
    q0 = g.get_q()
    q = q0.copy()
    q[3, 0, 8, 8] = -0.5                        # one interior cell of patch 3
    g.set_q(q)
    _expect_device_error(g, "negative water depth", 0.001)
    g.set_q(q0)                                 # the context is intact: a clean step runs
    assert g.advance(0.0, 0.001) > 0


def test_nan_in_q_is_reported():
    g = _solver(DAM, mx=16, my=16, minlevel=2, maxlevel=2)
    q = g.get_q()
    q[0, 1, 5, 5] = np.nan
    g.set_q(q)
    _expect_device_error(g, "non-finite value in q", 0.001)


@pytest.mark.parametrize("precision", [0, 1])
def test_negative_pressure_fails_newton(precision):
    """A cell whose energy is below its kinetic energy has negative pressure: the exact
    solver's Newton iteration cannot converge there, from the seed or from PVRS."""
    g = _solver(SHOCKBUBBLE, mx=16, my=16, minlevel=2, maxlevel=2, precision=precision)
    q0 = g.get_q()
    q = q0.copy()
    q[5, 3, 9, 9] = -1.0                        # E < 0
    g.set_q(q)
    _expect_device_error(g, "Newton iteration", 1e-4)
    g.set_q(q0)
    assert g.advance(0.0, 1e-4) > 0


def test_run_stops_on_device_failure():
    import forestclaw_b200 as fb
    g = _solver(DAM, mx=16, my=16, minlevel=2, maxlevel=3, subcycle=1, tfinal=0.01, initial_dt=0.002)
    q = g.get_q()
    q[0, 0, 6, 6] = -1.0
    g.set_q(q)
    with pytest.raises(fb.B200Error, match="negative water depth"):
        g.run()
