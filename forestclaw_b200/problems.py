"""Option presets of the built-in problems (the apps' .ini values, as the
benchmark configurations state them)."""
from __future__ import annotations

import math

from . import (APP_RADIALDAM, APP_SHOCKBUBBLE, APP_SPHERE, APP_SWIRL, APP_TSUNAMI, RP_ADVECTION,
               RP_ADVECTION_MANIFOLD, RP_EULER_EXACT, RP_SW_FWAVE, RP_SW_ROE)

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


# applications/clawpack/advection/2d/sphere on the cubed sphere (6 blocks, manifold metric):
# solid-body rotation about the axis (0, cos 45, sin 45) (the y axis tilted 45 degrees
# toward z), one revolution per unit time (omega = 2 pi); q = 0.1 + two Gaussians of width
# 0.1 rad centred on the rotation's equator at (1, 0, 0) and (0, cos 45, -sin 45);
# minmax tagging with the reference app's thresholds 0.25 / 0.05, MC limiter, capacity.
_C45 = math.sqrt(0.5)
SPHERE = dict(meqn=1, maux=3, mwaves=1, mthlim=(4,), rp=RP_ADVECTION_MANIFOLD, app=APP_SPHERE, mcapa=1,
              mthbc=(1, 1, 1, 1), refine_threshold=0.25, coarsen_threshold=0.05,
              pdata=(0.0, _C45, _C45, 2.0 * math.pi, 1.0, 0.0, 0.0, 0.0, _C45, -_C45, 0.1, 0.1))


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


class _Xoshiro256ss:
    """xoshiro256** (Blackman and Vigna, 2018) seeded by SplitMix64: a small portable
    generator so that batch workloads are the same on every machine."""

    M = (1 << 64) - 1

    def __init__(self, seed: int):
        x = seed & self.M
        self.s = []
        for _ in range(4):
            x = (x + 0x9E3779B97F4A7C15) & self.M
            z = x
            z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & self.M
            z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & self.M
            self.s.append(z ^ (z >> 31))

    @staticmethod
    def _rotl(v: int, k: int) -> int:
        return ((v << k) | (v >> (64 - k))) & _Xoshiro256ss.M

    def next(self) -> int:
        s = self.s
        r = (self._rotl((s[1] * 5) & self.M, 7) * 9) & self.M
        t = (s[1] << 17) & self.M
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = self._rotl(s[3], 45)
        return r

    def uniform(self, a: float, b: float) -> float:
        return a + (b - a) * ((self.next() >> 11) * (1.0 / (1 << 53)))

    def choice(self, seq):
        return seq[self.next() % len(seq)]


def tsunami_instances(n: int = 64, base_seed: int = 0, mx: int | None = None):
    """n independent tsunami forests for a batch: instance k draws from its own
    generator (seed base_seed + k) minlevel in {2, 3, 4}, maxlevel in minlevel+1..8
    (at most 5..8), the bathymetry centre in [-0.5, 0.5]^2 and 1 to 3 Gaussian
    humps of amplitude U[0.05, 0.3], width U[0.05, 0.2] and centre in [-1, 1]^2.
    Returns (instances, patch sizes): the patch size (8 or 16) is the instance's last
    draw unless mx is given."""
    out, sizes = [], []
    for k in range(n):
        g = _Xoshiro256ss(base_seed + k)
        lo = g.choice((2, 3, 4))
        hi = g.choice(tuple(range(max(lo + 1, 5), 9)))
        cx, cy = g.uniform(-0.5, 0.5), g.uniform(-0.5, 0.5)
        nb = g.choice((1, 2, 3))
        pd = [cx, cy, float(nb)]
        for _ in range(nb):
            pd += [g.uniform(0.05, 0.3), g.uniform(0.05, 0.2), g.uniform(-1.0, 1.0), g.uniform(-1.0, 1.0)]
        out.append(dict(minlevel=lo, maxlevel=hi, ax=-1.0, bx=1.0, ay=-1.0, by=1.0, mi=1, mj=1, pdata=tuple(pd)))
        size = g.choice((8, 16))
        sizes.append(mx if mx is not None else size)
    return out, sizes
