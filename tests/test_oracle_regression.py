"""The oracle against the reference's own regression values.

The reference's app regression tests (applications/.../regressions.sh) check three
counters at the end of a run (src/fclaw2d_finalize.c:119-165): coarse advances
taken (retaken steps included), patches at the end, and regrids that changed the
forest.  They depend on the initial refinement, the tagging criterion, the
refinement smoothing, p4est's adapt and 2:1 balance, the CFL-driven time step
of fclaw2d_run and, through the field values that tagging reads, on the update,
ghost fill and subcycling.  The options and values come from the reference's
own files (tests/golden/reference_regression.json)."""
import pytest

from oracle import pyoracle as po
from tests import regression_cases as rc
from tests.cases import make

CASES = rc.load()


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_reproduces_reference_counters(name):
    case = CASES[name]
    oc, _ = make(rc.problem(case))
    o = po.OracleSim(oc)
    o.initialize()
    r = o.run()
    got = {k: r[k] for k in ("count_amr_advance", "global_num_patches", "count_amr_new_domain")}
    assert got == case["expected"], (name, r)
    assert r["rejected"] == 0 and abs(r["t_final"] - float(case["options"]["options:tfinal"])) < 1e-12


def test_counters_depend_on_refinement_smoothing():
    """Without the smoothing the same runs give other counters, so matching them
    pins the smoothing rule (and is not a property of any forest code)."""
    for name, case in CASES.items():
        oc, _ = make(rc.problem(case), smooth_refine=0)
        o = po.OracleSim(oc)
        o.initialize()
        r = o.run()
        assert r["global_num_patches"] != case["expected"]["global_num_patches"], name


def test_cfl_rejection_retakes_the_step():
    """fclaw2d_run.c:210-226: a step above max_cfl is undone (restore_time_step) and
    retaken with dt scaled by desired_cfl / cfl; the retaken steps still count as
    advances."""
    case = CASES["radialdam_claw46"]
    oc, _ = make(rc.problem(case), initial_dt=0.5, tfinal=0.2)
    o = po.OracleSim(oc)
    o.initialize()
    r = o.run()
    assert r["rejected"] >= 1
    assert r["count_amr_advance"] == r["steps"] + r["rejected"]
    assert abs(r["t_final"] - 0.2) < 1e-12


def test_save_restore_step_roundtrip():
    import numpy as np
    oc, _ = make(rc.problem(CASES["swirl_claw46"]))
    o = po.OracleSim(oc)
    o.initialize()
    q0 = o.get_q()
    o.save_step()
    o.advance(0.0, 0.005)
    assert not np.array_equal(o.get_q(), q0)
    o.restore_step()
    assert np.array_equal(o.get_q(), q0)
