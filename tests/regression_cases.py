"""The reference's regression runs (tests/golden/reference_regression.json, made by
tests/golden/make_regression_values.py from the reference's regression.ini,
fclaw_options.ini and regression_values_N.csv) as problem dictionaries of this
package's tests."""
from __future__ import annotations

import json
import os

from oracle import pyoracle as po
import forestclaw_b200 as fb

_FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_regression.json")

_CRIT = {"value": fb.TAG_VALUE, "difference": fb.TAG_DIFFERENCE, "minmax": fb.TAG_MINMAX,
         "gradient": fb.TAG_GRADIENT}


def load() -> dict:
    with open(_FIX) as f:
        return json.load(f)


def _b(v: str) -> int:
    return 1 if v.strip().upper().startswith("T") else 0


def _ints(v: str):
    return tuple(int(x) for x in v.split())


def problem(case: dict) -> dict:
    """Options of one regression case in the keys of tests.cases.make."""
    o = case["options"]
    g = lambda k, d=None: o.get(k, d)  # noqa: E731
    d = dict(mx=int(g("clawpatch:mx")), my=int(g("clawpatch:my")), mbc=int(g("clawpatch:mbc")),
             meqn=int(g("clawpatch:meqn")), mwaves=int(g("clawpack46:mwaves")),
             order=_ints(g("clawpack46:order")), mthlim=_ints(g("clawpack46:mthlim")),
             mthbc=_ints(g("clawpack46:mthbc")), mcapa=int(g("clawpack46:mcapa")),
             minlevel=int(g("options:minlevel")), maxlevel=int(g("options:maxlevel")),
             regrid_interval=int(g("options:regrid_interval")),
             refine_threshold=float(g("options:refine_threshold")),
             coarsen_threshold=float(g("options:coarsen_threshold")),
             smooth_refine=_b(g("options:smooth-refine", "F")), smooth_level=int(g("options:smooth-level", "0")),
             refinement_criteria=_CRIT[g("clawpatch:refinement-criteria", "minmax")],
             threshold_variable=int(g("clawpatch:threshold-variable", "1")),
             tfinal=float(g("options:tfinal")), initial_dt=float(g("options:initial_dt")),
             use_fixed_dt=_b(g("options:use_fixed_dt", "F")), max_cfl=float(g("options:max_cfl")),
             desired_cfl=float(g("options:desired_cfl")), nout=int(g("options:nout")),
             subcycle=_b(g("options:subcycle", "F")), time_sync=_b(g("options:time-sync", "F")),
             ax=float(g("options:ax")), bx=float(g("options:bx")), ay=float(g("options:ay")), by=float(g("options:by")))
    if g("user:period") is not None:
        # swirl: scalar advection, stream-function velocities with period T; the
        # reference allocates maux = 3 but its b4step2 fills two fields
        d.update(problem=po.PROB_SWIRL, app=fb.APP_SWIRL, rp=fb.RP_ADVECTION, maux=2, tperiod=float(g("user:period")))
    else:
        # radial dam (example 0): Roe shallow water, the disc as cell averages (cellave2)
        d.update(problem=po.PROB_RADIALDAM, app=fb.APP_RADIALDAM, rp=fb.RP_SW_ROE, maux=int(g("clawpatch:maux")),
                 grav=float(g("user:g")), x0=float(g("user:x0")), y0=float(g("user:y0")), r0=float(g("user:r0")),
                 hin=float(g("user:hin")), hout=float(g("user:hout")), qinit_cellave=1)
    return d
