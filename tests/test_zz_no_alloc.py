"""fc2d_b200_mass_noalloc: the mass diagnostic for callers that may not
allocate device memory between steps (an application that hands out all device
memory from its own pool, or one whose other streams must not be stalled by the
synchronisation of cudaFree).  Its scratch is a static device array instead of
allocated memory.  It must give the same bits as fc2d_b200_mass, on two calls
in a row and on a second solver of the same process, and refuse forests that do
not fit the scratch.  This file is collected last on purpose."""
import numpy as np
import pytest

from tests.cases import DAM, make

pytestmark = pytest.mark.gpu


def _scratch_doubles() -> int:
    """FC2D_B200_MASS_SCRATCH_DOUBLES as the public header declares it."""
    import os
    import re
    hdr = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "fc2d_b200.h")
    with open(hdr) as f:
        return int(re.search(r"#define FC2D_B200_MASS_SCRATCH_DOUBLES (\d+)", f.read()).group(1))


SCRATCH_DOUBLES = _scratch_doubles()


def _solver(**kw):
    import forestclaw_b200 as fb
    _, gc = make(DAM, **kw)
    g = fb.Solver(gc)
    g.initialize()
    return g


def test_mass_noalloc_matches_mass_two_calls_in_a_row():
    g = _solver(mx=16, my=16, minlevel=2, maxlevel=4, subcycle=1, time_sync=1)
    t, dt = 0.0, 0.01
    for step in range(3):
        ref = g.mass()
        a = g.mass_noalloc()
        b = g.mass_noalloc()
        assert np.array_equal(a, ref), (step, a, ref)
        assert np.array_equal(b, ref), (step, b, ref)
        c = g.advance(t, dt)
        t += dt
        dt *= 0.9 / c
    g.close()


def test_mass_noalloc_first_and_repeated_calls_leave_device_memory_alone():
    """On a fresh solver the allocation-free call comes first (before any
    fc2d_b200_mass, whose buffer would hide an allocation), and free device
    memory does not change across repeated calls."""
    import torch
    g = _solver(mx=16, my=16, minlevel=2, maxlevel=3)
    dev = g.opts.device
    first = g.mass_noalloc()
    free0, _ = torch.cuda.mem_get_info(dev)
    for _ in range(3):
        assert np.array_equal(g.mass_noalloc(), first)
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0
    assert np.array_equal(first, g.mass())
    g.close()


def test_mass_noalloc_second_solver():
    g1 = _solver(mx=8, my=8, minlevel=3, maxlevel=3)
    g2 = _solver(mx=16, my=16, minlevel=4, maxlevel=4)
    for g in (g1, g2, g1):
        assert np.array_equal(g.mass_noalloc(), g.mass())
    g1.close()
    g2.close()


def test_mass_noalloc_rejects_oversize():
    import forestclaw_b200 as fb
    g = _solver(mx=8, my=8, minlevel=8, maxlevel=8)     # 65536 patches * 3 fields > scratch
    assert g.num_patches * 3 + 3 > SCRATCH_DOUBLES
    with pytest.raises(fb.B200Error, match="exceeds the static scratch"):
        g.mass_noalloc()
    ref = g.mass()
    assert ref[0] > 0
    g.close()
