"""Option presets of the built-in problems (the apps' .ini values, as the
benchmark configurations state them)."""
from __future__ import annotations

import math

from . import (APP_RADIALDAM, APP_SHOCKBUBBLE, APP_SWIRL, APP_TSUNAMI, RP_ADVECTION, RP_EULER_EXACT, RP_SW_FWAVE,
               RP_SW_ROE)

# applications/clawpack/advection/2d/swirl: MC limiter, T = 8 (velocity factor cos(pi t / 4))
SWIRL = dict(meqn=1, maux=2, mwaves=1, mthlim=(4,), rp=RP_ADVECTION, app=APP_SWIRL, tperiod=8.0,
             mthbc=(1, 1, 1, 1), ax=0.0, bx=1.0, ay=0.0, by=1.0)
# applications/clawpack/shallow/2d/radialdam on [-1,1]^2, r0 = 0.3, g = 1, extrapolation BCs
DAM = dict(meqn=3, maux=0, mwaves=3, mthlim=(4, 4, 4), rp=RP_SW_ROE, app=APP_RADIALDAM, grav=1.0, r0=0.3,
           hin=2.0, hout=1.0, x0=0.0, y0=0.0, ax=-1.0, bx=1.0, ay=-1.0, by=1.0, mthbc=(1, 1, 1, 1),
           refine_threshold=0.01, coarsen_threshold=0.002)
# shallow water with bathymetry (rpn2_tsunami f-waves); pdata = (cx, cy, nbumps, [A, w, x, y] * nbumps)
TSUNAMI = dict(meqn=3, maux=1, mwaves=3, mthlim=(4, 4, 4), rp=RP_SW_FWAVE, use_fwaves=1, app=APP_TSUNAMI,
               grav=1.0, ax=-1.0, bx=1.0, ay=-1.0, by=1.0, mthbc=(1, 1, 1, 1), refine_threshold=0.01,
               coarsen_threshold=0.002, pdata=(0.1, -0.2, 2, 0.2, 0.1, 0.3, 0.2, 0.1, 0.15, -0.4, -0.3))


# applications/clawpack/euler/2d/shockbubble on [0,2]x[0,1] (2x1 brick): Mach 1.22 shock at
# x = 0.2 into (rho, p) = (1, 1) at rest, bubble rho = 0.138 of radius 0.2 at (0.5, 0.5);
# inflow on the left (mthbc 0), extrapolation on the right, reflecting walls top and bottom;
# exact Riemann solver, Newton tolerance 1e-10; refine on |grad rho| dx
SHOCKBUBBLE = dict(meqn=4, maux=0, mwaves=3, mthlim=(4, 4, 4), rp=RP_EULER_EXACT, app=APP_SHOCKBUBBLE,
                   mthbc=(0, 1, 3, 3), ax=0.0, bx=2.0, ay=0.0, by=1.0, mi=2, mj=1, x0=0.5, y0=0.5, r0=0.2,
                   gamma=1.4, mach=1.22, rhob=0.138, newton_tol=1e-10, refine_threshold=0.05,
                   coarsen_threshold=0.01)


def options(problem: dict, **kw):
    """forestclaw_b200.Options for a preset with overrides."""
    from . import Options
    d = dict(problem)
    d.update(kw)
    keys = set(Options.__dataclass_fields__)
    return Options(**{k: v for k, v in d.items() if k in keys})


def swirl_dt(mx: int, level: int) -> float:
    """Fixed dt = 0.9 dx / max|s| with max|s| from the t = 0 edge velocities (swirl)."""
    import numpy as np
    n = mx * (1 << level)
    dx = 1.0 / n
    pi = 4.0 * math.atan(1.0)
    x = np.arange(n) * dx

    def psi(a, b):
        return (np.sin(pi * a) ** 2 * np.sin(pi * b) ** 2) / pi

    X, Y = np.meshgrid(x, x, indexing="ij")
    p0 = psi(X, Y)
    u = np.abs((psi(X, Y + dx) - p0) / dx)
    v = np.abs((psi(X + dx, Y) - p0) / dx)
    return 0.9 * dx / float(max(u.max(), v.max()))
