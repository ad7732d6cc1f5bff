"""Golden vectors from the reference's own CUDA patch update (run from the repo root,
on a machine with a GPU, after ``make -C oracle ref``):

    python -m tests.golden.make_cudaclaw_pin [output.npz]

The reference's ``cudaclaw_flux2_and_update_batch`` (src/solvers/fc2d_cudaclaw/
cuda_source/cudaclaw_flux2.cu) with the reference's cudaclaw app Riemann
solvers, all compiled from the reference tree into oracle/_ref/libpin_cudaclaw.so,
advances seeded patches once per (order, limiters) case of three families:

  swirl        scalar advection, cell velocities (rpn2adv.cu / rpt2adv.cu)
  swirl_fwave  the same solver's output taken as f-waves (use_fwaves = 1): the
               f-wave form of the update (clawpack46_flux2fw.f) -- limiting of
               f-waves, corrections scaled by sign(s), transverse f-waves
  radialdam    shallow water, Roe solver (radialdam_cuda/user_cuda/rpn2shallow.cu)

and its limiter function is sampled.  The shock-bubble app's transverse solver
(applications/cudaclaw/euler/2d/shockbubble/user_cuda/rp2euler.cu,
shockbubble_rpt2euler4) is evaluated on seeded interface states in both
directions.  The fixture pins the CPU oracle's update, its clawpack 4.6 Riemann
solvers, the Euler transverse split and its limiters
(tests/test_oracle_pin_cudaclaw.py).

Where the reference's GPU path and its clawpack 4.6 path differ by design, the
inputs stay where they agree:
  * the reference adds the second-order correction to the transverse solves
    whenever transverse propagation is on (cudaclaw_flux2.cu:528-532), clawpack
    4.6 only with method(3) = 2: second-order cases use order (2, 2) or (2, 0);
  * the reference scales the y-correction by dt/dx (cudaclaw_flux2.cu:593):
    square cells;
  * the reference's GPU Roe solver has no entropy fix, clawpack46_rpn2.f applies
    Harten-Hyman's at transonic rarefactions: subsonic states (|u| <= 0.3 c),
    where the fix is inactive;
  * the shallow-water f-wave solver is not pinned: the reference's GPU port
    (tsunami_cuda/user_cuda/rpn2_tsunami.cu:74) takes the Roe celerity as
    sqrt(g (hl + hr)) / 2, its Fortran solver (rp/rpn2_tsunami.f90:118), which
    the oracle restates, as sqrt(g (hl + hr) / 2), so their speeds differ on
    every interface with a jump.
"""
from __future__ import annotations

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "cudaclaw_pin.npz")

# family -> solver id, meqn, maux, use_fwaves, grav, [(order, limiters per wave)]
FAMILIES = {
    "swirl": (0, 1, 2, 0, 1.0,
              [((1, 0), (0,)), ((1, 1), (0,)), ((1, 2), (0,)), ((2, 0), (0,)), ((2, 0), (4,)), ((2, 2), (0,)),
               ((2, 2), (1,)), ((2, 2), (2,)), ((2, 2), (3,)), ((2, 2), (4,)), ((2, 2), (5,))]),
    "swirl_fwave": (0, 1, 2, 1, 1.0,
                    [((1, 0), (0,)), ((1, 2), (0,)), ((2, 0), (4,)), ((2, 2), (0,)), ((2, 2), (1,)),
                     ((2, 2), (2,)), ((2, 2), (3,)), ((2, 2), (4,))]),
    "radialdam": (1, 3, 0, 0, 1.0,
                  [((1, 0), (0, 0, 0)), ((1, 2), (0, 0, 0)), ((2, 2), (0, 0, 0)), ((2, 2), (4, 4, 4)),
                   ((2, 2), (1, 2, 3)), ((2, 0), (3, 3, 3))]),
}


def inputs(family: str, seed: int = 20261203, npatch: int = 4, mx: int = 16, mbc: int = 2):
    """Seeded patches with ghost cells: smooth data plus jumps and noise (shallow water:
    depth >= 0.8, speeds <= 0.3 of the celerity); dx = dy = 1/mx,
    dt at CFL 0.45 per direction.  Returns q (npatch, meqn, n, n), aux (npatch, maux, n, n)
    or None, dx, dt."""
    solver, meqn, maux, _, grav, _ = FAMILIES[family]
    rng = np.random.default_rng(seed + 1000 * solver)
    n = mx + 2 * mbc
    x = (np.arange(n) - mbc + 0.5) / mx
    X, Y = np.meshgrid(x, x)
    q = np.empty((npatch, meqn, n, n))
    aux = np.empty((npatch, maux, n, n)) if maux else None
    smax = 0.0
    for p in range(npatch):
        a, b, c = rng.uniform(0.5, 3.0, 3)
        x0, y0 = rng.uniform(0.2, 0.8, 2)
        blob = (X - x0) ** 2 + (Y - y0) ** 2 < 0.1
        if family.startswith("swirl"):
            q[p, 0] = np.sin(2 * np.pi * (a * X + b * Y)) + c * blob + 0.5 * (X > x0) \
                + 0.05 * rng.standard_normal((n, n))
            w = rng.uniform(-1.0, 1.0)
            aux[p, 0] = np.clip(-w * (Y - 0.5) + 0.3 * rng.uniform(-1, 1, (n, n)), -1.0, 1.0)
            aux[p, 1] = np.clip(w * (X - 0.5) + 0.3 * rng.uniform(-1, 1, (n, n)), -1.0, 1.0)
            smax = max(smax, np.abs(aux[p]).max())
        else:
            h = 1.0 + 0.2 * c * blob + 0.15 * np.sin(2 * np.pi * (a * X + b * Y)) + 0.1 * (X > x0) \
                + 0.01 * rng.standard_normal((n, n))
            cel = np.sqrt(grav * h)
            u = 0.3 * cel * np.clip(np.sin(2 * np.pi * b * Y) + 0.3 * rng.uniform(-1, 1, (n, n)), -1, 1)
            v = 0.3 * cel * np.clip(np.cos(2 * np.pi * a * X) + 0.3 * rng.uniform(-1, 1, (n, n)), -1, 1)
            q[p, 0], q[p, 1], q[p, 2] = h, h * u, h * v
            if maux:
                aux[p, 0] = 0.05 * np.sin(2 * np.pi * (b * X - a * Y)) + 0.01 * rng.standard_normal((n, n))
            smax = max(smax, (np.maximum(np.abs(u), np.abs(v)) + cel).max() * 1.3)
    dx = 1.0 / mx
    dt = 0.45 * dx / smax
    return q, aux, dx, dt


def euler_inputs(seed: int = 20261204, n: int = 512):
    """Seeded pairs of Euler states (rho, rho u, rho v, E) for gamma 1.4 -- density
    0.3-3, velocities in [-1.5, 1.5], pressure 0.3-3 -- and fluctuations asdq of
    both signs."""
    rng = np.random.default_rng(seed)
    def states():
        rho = rng.uniform(0.3, 3.0, n)
        u, v = rng.uniform(-1.5, 1.5, n), rng.uniform(-1.5, 1.5, n)
        p = rng.uniform(0.3, 3.0, n)
        return np.stack([rho, rho * u, rho * v, p / 0.4 + 0.5 * rho * (u * u + v * v)], axis=1)
    return states(), states(), rng.standard_normal((n, 4))


def limiter_samples():
    return np.concatenate([np.linspace(-3.0, 3.0, 121), [0.0, 0.5, 1.0, 2.0, -0.0, 1e-300, 1e300, -1e300]])


def main(out_path: str = OUT) -> None:
    from oracle import pin_reference as pr
    if not pr.available():
        raise SystemExit("oracle/_ref/libpin_cudaclaw.so missing: make -C oracle ref")
    out = {}
    total = 0
    for fam, (solver, meqn, maux, fw, grav, cases) in FAMILIES.items():
        q, aux, dx, dt = inputs(fam)
        out[f"{fam}_q_in"] = q
        if aux is not None:
            out[f"{fam}_aux"] = aux
        out[f"{fam}_dx"] = np.float64(dx)
        out[f"{fam}_dt"] = np.float64(dt)
        for k, (order, lim) in enumerate(cases):
            qo, _ = pr.step(solver, q, aux, dx, dt, order, lim, use_fwaves=fw, grav=grav)
            out[f"{fam}_q_out_{k}"] = qo
            total += 1
    ql, qr, asdq = euler_inputs()
    out["euler_ql"], out["euler_qr"], out["euler_asdq"] = ql, qr, asdq
    for idir in (0, 1):
        out[f"euler_bm_{idir}"], out[f"euler_bp_{idir}"] = pr.euler_rpt2(idir, ql, qr, asdq, 1.4)
    r = limiter_samples()
    out["limiter_r"] = r
    for lim in range(0, 6):
        out[f"limiter_phi_{lim}"] = pr.limiter(lim, r)
    np.savez_compressed(out_path, **out)
    print(f"wrote {out_path}: {total} update cases in {len(FAMILIES)} families, 6 limiters x {r.size} samples")


if __name__ == "__main__":
    import sys
    main(sys.argv[1] if len(sys.argv) > 1 else OUT)
