"""Shared problem definitions for the tests: one description, two configurations
(CPU oracle and B200 solver) with identical option values."""
from __future__ import annotations

from oracle import pyoracle as po
import forestclaw_b200 as fb
from forestclaw_b200.problems import DAM as _DAM, SWIRL as _SWIRL, TSUNAMI as _TSUNAMI, swirl_dt  # noqa: F401
from forestclaw_b200.problems import SHOCKBUBBLE as _SHOCKBUBBLE, SPHERE as _SPHERE

SWIRL = dict(_SWIRL, problem=po.PROB_SWIRL)
DAM = dict(_DAM, problem=po.PROB_RADIALDAM)
TSUNAMI = dict(_TSUNAMI, problem=po.PROB_TSUNAMI)
SHOCKBUBBLE = dict(_SHOCKBUBBLE, problem=po.PROB_SHOCKBUBBLE)
SPHERE = dict(_SPHERE, problem=po.PROB_SPHERE)

_ORC_KEYS = {"mx", "my", "mbc", "meqn", "maux", "mwaves", "order", "mthlim", "mthbc", "mcapa", "use_fwaves",
             "rp", "minlevel", "maxlevel", "subcycle", "time_sync", "flux_correction", "fluctuation_correction",
             "refine_threshold", "coarsen_threshold", "ax", "bx", "ay", "by", "mi", "mj", "problem", "grav",
             "tperiod", "r0", "hin", "hout", "x0", "y0", "pdata", "nthreads", "gamma", "mach", "rhob",
             "newton_tol", "smooth_refine", "smooth_level", "threshold_variable", "regrid_interval", "tfinal",
             "initial_dt", "max_cfl", "desired_cfl", "nout", "use_fixed_dt"}
# option names that differ between the two configurations
_ORC_RENAME = {"refinement_criteria": "tag_criteria"}


def _orc_kwargs(d: dict) -> dict:
    out = {k: v for k, v in d.items() if k in _ORC_KEYS}
    for a, b in _ORC_RENAME.items():
        if a in d:
            out[b] = d[a]
    if "qinit_cellave" in d:
        out["qinit_sharp"] = 0 if d["qinit_cellave"] else 1
    return out


def make(problem: dict, **kw):
    """Return (oracle config, B200 Options) for one problem with overrides."""
    d = dict(problem)
    d.update(kw)
    orc = po.make_config(**_orc_kwargs(d))
    gpu = fb.Options(**{k: v for k, v in d.items() if k in set(fb.Options.__dataclass_fields__)})
    return orc, gpu
