"""Generate the committed oracle fixtures under tests/golden (run from the repo root):

    python -m tests.golden.make_golden

Each fixture stores the patch layout, the CFL sequence and the final q of a short
run of the CPU oracle.  They freeze the oracle so any change to it is visible.
"""
from __future__ import annotations

import os

import numpy as np

from oracle import pyoracle as po
from tests.cases import DAM, SWIRL, TSUNAMI, make, swirl_dt

HERE = os.path.dirname(os.path.abspath(__file__))

CASES = {
    "swirl_l2_32": (SWIRL, dict(mx=32, my=32, minlevel=2, maxlevel=2), 6, 0, None),
    "dam_amr_l2_4": (DAM, dict(mx=16, my=16, minlevel=2, maxlevel=4, subcycle=1, time_sync=1), 6, 2, 0.9),
    "tsunami_amr_8": (TSUNAMI, dict(mx=8, my=8, minlevel=2, maxlevel=4, subcycle=1, time_sync=1), 4, 2, 0.9),
}


def run_case(name: str) -> dict:
    prob, kw, nsteps, regrid_every, cfl_target = CASES[name]
    oc, _ = make(prob, nthreads=1, **kw)
    s = po.OracleSim(oc)
    s.initialize()
    dt = swirl_dt(kw["mx"], kw["minlevel"]) if prob is SWIRL else 0.01
    t = 0.0
    cfls = []
    for n in range(nsteps):
        c = s.advance(t, dt)
        cfls.append(c)
        t += dt
        if cfl_target:
            dt *= cfl_target / c
        if regrid_every and (n + 1) % regrid_every == 0:
            s.regrid()
    return {"info": s.patch_info(), "cfl": np.array(cfls), "q": s.get_q()}


if __name__ == "__main__":
    for name in CASES:
        out = run_case(name)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, out["q"].shape, out["cfl"][-1])
