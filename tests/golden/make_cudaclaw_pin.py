"""Golden vectors from the reference's own CUDA patch update (run from the repo root,
on a machine with a GPU, after ``make -C oracle ref``):

    python -m tests.golden.make_cudaclaw_pin [output.npz]

The reference's ``cudaclaw_flux2_and_update_batch`` (src/solvers/fc2d_cudaclaw/
cuda_source/cudaclaw_flux2.cu, compiled from the reference tree into
oracle/_ref/libpin_cudaclaw.so) advances seeded scalar-advection patches -- random
cell velocities, smooth data with jumps, ghost cells filled with data of the same
kind -- once for each (order, limiter) the reference's GPU solver runs like
clawpack 4.6, and its limiter function is sampled.  The fixture pins the CPU
oracle's update and limiters (tests/test_oracle_pin_cudaclaw.py).

Cases: the reference adds the second-order correction to the transverse solves
whenever transverse propagation is on (cudaclaw_flux2.cu:528-532), as clawpack
4.6 does only with method(3) = 2, so second-order cases use order (2, 2) or
(2, 0); square cells, since the reference scales the y-correction by dt/dx
(cudaclaw_flux2.cu:593).
"""
from __future__ import annotations

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "cudaclaw_advection_pin.npz")

# (order, limiter)
CASES = [((1, 0), 0), ((1, 1), 0), ((1, 2), 0), ((2, 0), 0), ((2, 0), 4), ((2, 2), 0), ((2, 2), 1),
         ((2, 2), 2), ((2, 2), 3), ((2, 2), 4), ((2, 2), 5)]


def inputs(seed: int = 20261203, npatch: int = 4, mx: int = 16, mbc: int = 2):
    """Seeded patches: q = smooth field + jumps, cell velocities in [-1, 1]^2 (a smooth
    rotation plus noise), dx = dy = 1/mx, dt at CFL 0.45 per direction."""
    rng = np.random.default_rng(seed)
    n = mx + 2 * mbc
    x = (np.arange(n) - mbc + 0.5) / mx
    X, Y = np.meshgrid(x, x)
    q = np.empty((npatch, n, n))
    aux = np.empty((npatch, 2, n, n))
    for p in range(npatch):
        a, b, c = rng.uniform(0.5, 3.0, 3)
        x0, y0 = rng.uniform(0.2, 0.8, 2)
        q[p] = np.sin(2 * np.pi * (a * X + b * Y)) + c * ((X - x0) ** 2 + (Y - y0) ** 2 < 0.1) \
            + 0.5 * (X > x0) + 0.05 * rng.standard_normal((n, n))
        w = rng.uniform(-1.0, 1.0)
        aux[p, 0] = np.clip(-w * (Y - 0.5) + 0.3 * rng.uniform(-1, 1, (n, n)), -1.0, 1.0)
        aux[p, 1] = np.clip(w * (X - 0.5) + 0.3 * rng.uniform(-1, 1, (n, n)), -1.0, 1.0)
    dx = 1.0 / mx
    dt = 0.45 * dx / max(np.abs(aux).max(), 1e-12)
    return q, aux, dx, dt


def limiter_samples():
    r = np.concatenate([np.linspace(-3.0, 3.0, 121), [0.0, 0.5, 1.0, 2.0, -0.0, 1e-300, 1e300, -1e300]])
    return r


def main(out_path: str = OUT) -> None:
    from oracle import pin_reference as pr
    if not pr.available():
        raise SystemExit("oracle/_ref/libpin_cudaclaw.so missing: make -C oracle ref")
    q, aux, dx, dt = inputs()
    out = {"q_in": q, "aux": aux, "dx": np.float64(dx), "dt": np.float64(dt),
           "orders": np.array([c[0] for c in CASES], np.int32), "limiters": np.array([c[1] for c in CASES], np.int32)}
    for k, (order, lim) in enumerate(CASES):
        qo, cfl = pr.advection_step(q, aux, dx, dx, dt, order, lim)
        out[f"q_out_{k}"] = qo
        out[f"cfl_{k}"] = cfl
    r = limiter_samples()
    out["limiter_r"] = r
    for lim in range(0, 6):
        out[f"limiter_phi_{lim}"] = pr.limiter(lim, r)
    np.savez_compressed(out_path, **out)
    print(f"wrote {out_path}: {len(CASES)} update cases of {q.shape[0]} patches, 6 limiters x {r.size} samples")


if __name__ == "__main__":
    import sys
    main(sys.argv[1] if len(sys.argv) > 1 else OUT)
