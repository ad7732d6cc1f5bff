"""Shared problem definitions: one description, two configurations (CPU oracle and
B200 solver) with identical option values."""
from __future__ import annotations

import math

from oracle import pyoracle as po
import forestclaw_b200 as fb

SWIRL = dict(meqn=1, maux=2, mwaves=1, mthlim=(4,), rp=0, problem=po.PROB_SWIRL, app=fb.APP_SWIRL,
             tperiod=8.0, mthbc=(1, 1, 1, 1), ax=0.0, bx=1.0, ay=0.0, by=1.0)
DAM = dict(meqn=3, maux=0, mwaves=3, mthlim=(4, 4, 4), rp=1, problem=po.PROB_RADIALDAM,
           app=fb.APP_RADIALDAM, grav=1.0, r0=0.3, hin=2.0, hout=1.0, x0=0.0, y0=0.0,
           ax=-1.0, bx=1.0, ay=-1.0, by=1.0, mthbc=(1, 1, 1, 1),
           refine_threshold=0.01, coarsen_threshold=0.002)
TSUNAMI = dict(meqn=3, maux=1, mwaves=3, mthlim=(4, 4, 4), rp=2, use_fwaves=1, problem=po.PROB_TSUNAMI,
               app=fb.APP_TSUNAMI, grav=1.0, ax=-1.0, bx=1.0, ay=-1.0, by=1.0, mthbc=(1, 1, 1, 1),
               refine_threshold=0.01, coarsen_threshold=0.002,
               pdata=(0.1, -0.2, 2, 0.2, 0.1, 0.3, 0.2, 0.1, 0.15, -0.4, -0.3))

_ORC_KEYS = {"mx", "my", "mbc", "meqn", "maux", "mwaves", "order", "mthlim", "mthbc", "mcapa", "use_fwaves",
             "rp", "minlevel", "maxlevel", "subcycle", "time_sync", "flux_correction", "fluctuation_correction",
             "refine_threshold", "coarsen_threshold", "ax", "bx", "ay", "by", "mi", "mj", "problem", "grav",
             "tperiod", "r0", "hin", "hout", "x0", "y0", "pdata", "nthreads"}
_GPU_KEYS = {"mx", "my", "mbc", "meqn", "maux", "mwaves", "order", "mthlim", "mthbc", "mcapa", "use_fwaves",
             "rp", "minlevel", "maxlevel", "subcycle", "time_sync", "flux_correction", "fluctuation_correction",
             "refine_threshold", "coarsen_threshold", "ax", "bx", "ay", "by", "mi", "mj", "app", "grav",
             "tperiod", "r0", "hin", "hout", "x0", "y0", "pdata", "precision"}


def make(problem: dict, **kw):
    """Return (oracle config, B200 Options) for one problem with overrides."""
    d = dict(problem)
    d.update(kw)
    orc = po.make_config(**{k: v for k, v in d.items() if k in _ORC_KEYS})
    gpu = fb.Options(**{k: v for k, v in d.items() if k in _GPU_KEYS})
    return orc, gpu


def swirl_dt(mx: int, level: int) -> float:
    """Fixed dt = 0.9 dx / max|s| with max|s| from the t=0 edge velocities (swirl)."""
    import numpy as np
    n = mx * (1 << level)
    dx = 1.0 / n
    pi = 4.0 * math.atan(1.0)
    x = np.arange(n + 1) * dx

    def psi(a, b):
        return (np.sin(pi * a) ** 2 * np.sin(pi * b) ** 2) / pi

    X, Y = np.meshgrid(x[:-1], x[:-1], indexing="ij")
    p0 = psi(X, Y)
    u = np.abs((psi(X, Y + dx) - p0) / dx)
    v = np.abs((psi(X + dx, Y) - p0) / dx)
    return 0.9 * dx / float(max(u.max(), v.max()))
