"""Application-supplied __device__ solvers (include/fc2d_b200_user.cuh).

The solver pairs, b4step2 and src2 live outside the package, in
tests/user_solvers/*.cu, written with cudaclaw's device signatures
(fc2d_cudaclaw_cuda.h:52-73): the reference GPU app's radial acoustics pair with a
damping source, and its swirl advection pair with a b4step2 that sets the edge
velocities each step.  Registered inline (template) and through device function
pointers (the cudaclaw protocol), they must advance an adaptive, subcycled forest
bit for bit like the oracle running its C restatement of the same functions."""
import ctypes

import numpy as np
import pytest

from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def _module(name: str):
    import forestclaw_b200 as fb
    from forestclaw_b200 import build
    fb.load_library()
    for p in build.build_user_examples():
        if p.endswith("lib" + name + ".so"):
            return ctypes.CDLL(p)
    raise FileNotFoundError(name)


COMMON = dict(mx=16, my=16, mbc=2, minlevel=2, maxlevel=3, subcycle=1, mthbc=(1, 1, 1, 1),
              refine_threshold=0.02, coarsen_threshold=0.005)


def _pair(orc_kw: dict, gpu_kw: dict, register):
    import forestclaw_b200 as fb
    o = po.OracleSim(po.make_config(**COMMON, **orc_kw))
    o.initialize()
    info = o.patch_info()
    assert len(np.unique(info[:, 0])) == 2          # an adaptive forest: two levels
    keys = set(fb.Options.__dataclass_fields__)
    g = fb.Solver(fb.Options(**{k: v for k, v in {**COMMON, **gpu_kw}.items() if k in keys}))
    register(g)
    g.set_forest(info[:, 0], info[:, 2], info[:, 3])
    g.set_q(o.get_q())
    if orc_kw.get("maux", 0) > 0:
        g.set_aux(o.get_aux())
    return o, g


def _advance_both(o, g, dt, nsteps):
    t = 0.0
    for _ in range(nsteps):
        co = o.advance(t, dt)
        cg = g.advance(t, dt)
        assert cg == co
        t += dt
    assert np.array_equal(g.get_q(), o.get_q())


def _acoustics(register_name: str):
    import forestclaw_b200 as fb
    lib = _module("acoustics_user")
    rho, bulk, rate = 1.0, 4.0, 0.5
    assert lib.acoustics_set_params(ctypes.c_double(rho), ctypes.c_double(bulk), ctypes.c_double(rate)) == 0
    pdata = [0.0] * 32
    pdata[24], pdata[25] = rho, bulk
    orc = dict(meqn=3, maux=0, mwaves=2, mthlim=(4, 4), rp=po.RP_ACOUSTICS, problem=po.PROB_ACOUSTICS,
               x0=0.45, y0=0.55, r0=0.2, hin=2.0, hout=1.0, pdata=pdata, src_kind=1, src_rate=rate)
    gpu = dict(meqn=3, maux=0, mwaves=2, mthlim=(4, 4), rp=fb.RP_USER, app=fb.APP_NONE)
    fn = getattr(lib, register_name)
    fn.argtypes = [ctypes.c_void_p]

    def register(g):
        rc = fn(g.h)
        assert rc == 0, g.lib.fc2d_b200_last_error()
    return _pair(orc, gpu, register)


@pytest.mark.parametrize("how", ["acoustics_register_inline", "acoustics_register_by_pointer"])
def test_user_acoustics_with_src2_bitwise_with_oracle(how):
    o, g = _acoustics(how)
    _advance_both(o, g, 0.005, 6)
    g.close()


def test_user_advection_with_b4step2_bitwise_with_oracle():
    import forestclaw_b200 as fb
    lib = _module("rotation_user")
    omega = 6.0
    assert lib.rotation_set_params(ctypes.c_double(omega)) == 0
    pdata = [0.0] * 32
    pdata[26] = omega
    orc = dict(meqn=1, maux=2, mwaves=1, mthlim=(4,), rp=po.RP_ADVECTION, problem=po.PROB_ROTATION,
               x0=0.7, y0=0.5, r0=0.15, pdata=pdata)
    gpu = dict(meqn=1, maux=2, mwaves=1, mthlim=(4,), rp=fb.RP_USER, app=fb.APP_NONE)
    fn = lib.rotation_register_inline
    fn.argtypes = [ctypes.c_void_p]
    o, g = _pair(orc, gpu, lambda g: fn(g.h) == 0 or pytest.fail(g.lib.fc2d_b200_last_error()))
    _advance_both(o, g, 0.0015, 6)
    assert np.array_equal(g.get_aux(), o.get_aux())     # b4step2 wrote the same aux
    g.close()


def test_user_registration_checks():
    import forestclaw_b200 as fb
    lib = _module("acoustics_user")
    fn = lib.acoustics_register_inline
    fn.argtypes = [ctypes.c_void_p]
    # a solver built for a package solver id refuses application kernels
    g = fb.Solver(fb.Options(**{**COMMON, "meqn": 3, "mwaves": 2, "rp": fb.RP_SW_ROE}))
    assert fn(g.h) == -1
    g.close()
    # meqn of the application solver and of the options must agree
    g = fb.Solver(fb.Options(**{**COMMON, "meqn": 1, "mwaves": 2, "rp": fb.RP_USER}))
    assert fn(g.h) == -1
    g.close()
    # no registered kernel: an advance is refused, not launched
    g = fb.Solver(fb.Options(**{**COMMON, "meqn": 3, "mwaves": 2, "rp": fb.RP_USER}))
    gx, gy = np.meshgrid(np.arange(4), np.arange(4), indexing="ij")
    g.set_forest(np.full(16, 2), gx.ravel(), gy.ravel())
    with pytest.raises(fb.B200Error, match="register the application solver"):
        g.advance(0.0, 0.001)
    g.close()
