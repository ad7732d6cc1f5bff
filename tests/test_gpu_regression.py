"""The B200 path against the reference's regression values and the oracle.

fc2d_b200_run (fclaw2d_run outstyle 1) on the reference's regression runs must
reproduce the reference's counters (tests/golden/reference_regression.json, from
its regression_values_N.csv) and end bit for bit on the oracle's forest and
fields; the CFL retake path must agree with the oracle's as well."""
import numpy as np
import pytest

from oracle import pyoracle as po
from tests import regression_cases as rc
from tests.cases import make

pytestmark = pytest.mark.gpu
CASES = rc.load()
KEYS = ("count_amr_advance", "global_num_patches", "count_amr_new_domain")


def _both(prob, **kw):
    import forestclaw_b200 as fb
    oc, gc = make(prob, **kw)
    o = po.OracleSim(oc)
    g = fb.Solver(gc)
    o.initialize()
    g.initialize()
    return o, g


@pytest.mark.parametrize("name", sorted(CASES))
def test_run_reproduces_reference_counters_bitwise_with_oracle(name):
    case = CASES[name]
    o, g = _both(rc.problem(case))
    ro, rg = o.run(), g.run()
    assert {k: rg[k] for k in KEYS} == case["expected"], (name, rg)
    assert rg == ro
    assert np.array_equal(g.patch_info(), o.patch_info())
    assert np.array_equal(g.get_q(), o.get_q())
    # the same fields; the per-field sums (Kahan over patches on both sides, in a
    # different grouping) agree to round-off of the largest field's mass
    mg, mo = g.mass(), o.mass()
    assert np.all(np.abs(mg - mo) <= 1e-12 * np.abs(mo[0]))
    g.close()


def test_run_retakes_rejected_steps_like_the_oracle():
    """A first step of CFL 1.22 (above max_cfl 1) is rejected and retaken with
    dt * desired_cfl / cfl, as fclaw2d_run does (src/fclaw2d_run.c:220-236)."""
    case = CASES["radialdam_claw46"]
    o, g = _both(rc.problem(case), initial_dt=0.11, tfinal=0.2)
    ro, rg = o.run(), g.run()
    assert rg["rejected"] >= 1 and rg == ro
    assert np.array_equal(g.get_q(), o.get_q())
    g.close()


def test_run_stops_on_a_step_that_breaks_the_fields():
    """A first step of CFL ~10 drives depths negative and q non-finite.  The
    reference would take the maximum of its finite CFL numbers and retake the step;
    the B200 run stops with the device status instead of retaking from fields whose
    CFL number is not defined."""
    import forestclaw_b200 as fb
    case = CASES["radialdam_claw46"]
    _, g = _both(rc.problem(case), initial_dt=0.5, tfinal=0.2)
    with pytest.raises(fb.B200Error, match="device status"):
        g.run()
    g.close()


def test_save_restore_step_on_device():
    import forestclaw_b200 as fb
    o, g = _both(rc.problem(CASES["swirl_claw46"]))
    q0 = g.get_q()
    g.save_step()
    g.advance(0.0, 0.005)
    assert not np.array_equal(g.get_q(), q0)
    g.restore_step()
    assert np.array_equal(g.get_q(), q0)
    g.regrid()          # a new forest: the saved copy no longer applies
    if g.num_patches != q0.shape[0]:
        with pytest.raises(fb.B200Error, match="no saved step"):
            g.restore_step()
    g.close()


@pytest.mark.parametrize("crit", ["value", "difference", "gradient"])
def test_tagging_criteria_match_oracle(crit):
    """Every refinement criterion of the reference, through initialization and
    regrids with smoothing, gives the oracle's forest and fields."""
    base = rc.problem(CASES["radialdam_claw46"])
    thr = {"value": (1.5, 1.2), "difference": (0.05, 0.02), "gradient": (0.5, 0.25)}[crit]
    o, g = _both(base, refinement_criteria=rc._CRIT[crit], refine_threshold=thr[0], coarsen_threshold=thr[1],
                 tfinal=0.2)
    ro, rg = o.run(), g.run()
    assert rg == ro
    assert np.array_equal(g.patch_info(), o.patch_info())
    assert np.array_equal(g.get_q(), o.get_q())
    g.close()
