"""The CPU oracle pinned against the reference's own CUDA patch update.

The reference's ``cudaclaw_flux2_and_update_batch`` and ``cudaclaw_limiter``
(src/solvers/fc2d_cudaclaw/cuda_source/cudaclaw_flux2.cu, cudaclaw_limiters.cu)
with the reference's cudaclaw app Riemann solvers -- swirl advection (also in
the f-wave form of the update) and radialdam Roe shallow water -- compiled from
the reference tree into oracle/_ref/libpin_cudaclaw.so, advanced seeded patches
on a B200; ``tests/golden/make_cudaclaw_pin.py`` stored the results in
``tests/golden/cudaclaw_pin.npz``.  The oracle's clawpack 4.6 update (normal
solves, wave limiting with every limiter the reference's GPU solver has,
second-order corrections, transverse propagation, the conservative update) with
its clawpack 4.6 Riemann solvers must give the same interior cells to rounding,
and the same limiter values bit for bit.  The FP64 CUDA kernels are bitwise
equal to the oracle (test_gpu_parity), so this pins them too.

Tolerance: the reference adds the transverse terms with atomicAdd in whatever
order the threads arrive and lets nvcc contract multiply-adds; the oracle keeps
the Fortran order without contraction (and the Fortran Roe solver forms apdq as
the total fluctuation minus amdq).  Per cell the results differ by a few units
in the last place: |q_oracle - q_reference| <= 2e-15 max |q| per field.  The
reference's per-patch CFL is not compared: every thread stores the result of a
block reduction that only thread 0 holds (cudaclaw_flux2.cu:462).
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from tests.golden import make_cudaclaw_pin as mk

REL_TOL = 2e-15
MBC = 2


def _oracle_step(family, q, aux, dx, dt, order, lim):
    from oracle import pyoracle as po
    solver, meqn, maux, fw, grav, _ = mk.FAMILIES[family]
    rp = {0: po.RP_ADVECTION, 1: po.RP_SW_ROE}[solver]
    npatch, _, n, _ = q.shape
    mx = n - 2 * MBC
    cfg = po.make_config(mx=mx, my=mx, mbc=MBC, meqn=meqn, maux=maux, mwaves=len(lim), rp=rp, use_fwaves=fw,
                         grav=grav, order=tuple(order), mthlim=tuple(int(v) for v in lim) + (0,) * (8 - len(lim)))
    out = np.empty_like(q)
    for p in range(npatch):
        qq = np.ascontiguousarray(q[p]).ravel().copy()
        a = np.ascontiguousarray(aux[p]).ravel().copy() if aux is not None else None
        po.patch_step2(cfg, qq, a, dx, dx, dt)
        out[p] = qq.reshape(q.shape[1:])
    return out


def _assert_close(out, ref, what):
    s = slice(MBC, -MBC)
    for p in range(ref.shape[0]):
        for m in range(ref.shape[1]):
            scale = np.abs(ref[p, m][s, s]).max()
            err = np.abs(out[p, m][s, s] - ref[p, m][s, s]).max()
            assert err <= REL_TOL * scale, f"{what} patch {p} field {m}: max |dq| {err:.3e} > {REL_TOL:g} x {scale:.3e}"


def _fixture():
    if not os.path.exists(mk.OUT):
        pytest.fail(f"fixture {mk.OUT} missing")
    return np.load(mk.OUT)


@pytest.mark.parametrize("family", sorted(mk.FAMILIES))
def test_fixture_inputs_are_reproducible(family):
    """The stored inputs are those of the seeded generator."""
    d = _fixture()
    q, aux, dx, dt = mk.inputs(family)
    assert np.array_equal(q, d[f"{family}_q_in"])
    assert (aux is None) == (f"{family}_aux" not in d.files)
    if aux is not None:
        assert np.array_equal(aux, d[f"{family}_aux"])
    assert float(d[f"{family}_dx"]) == dx and float(d[f"{family}_dt"]) == dt


@pytest.mark.parametrize("family", sorted(mk.FAMILIES))
def test_oracle_update_matches_reference_cudaclaw(family):
    d = _fixture()
    q = d[f"{family}_q_in"]
    aux = d[f"{family}_aux"] if f"{family}_aux" in d.files else None
    dx, dt = float(d[f"{family}_dx"]), float(d[f"{family}_dt"])
    for k, (order, lim) in enumerate(mk.FAMILIES[family][5]):
        ref = d[f"{family}_q_out_{k}"]
        # the reference updates the interior only; its ghost cells are the inputs
        assert np.array_equal(ref[..., :MBC, :], q[..., :MBC, :]) and np.array_equal(ref[..., -MBC:], q[..., -MBC:])
        assert not np.array_equal(ref, q)
        _assert_close(_oracle_step(family, q, aux, dx, dt, order, lim), ref, f"{family} order {order} limiters {lim}")


EULER_TOL = 1e-13


def _euler_check(ql, qr, asdq, bm_ref, bp_ref, idir):
    from oracle import pyoracle as po
    for k in range(ql.shape[0]):
        bm, bp = po.euler_rpt2(1.4, idir + 1, ql[k], qr[k], asdq[k])
        scale = max(np.abs(bm_ref[k]).max(), np.abs(bp_ref[k]).max(), np.abs(asdq[k]).max())
        err = max(np.abs(bm - bm_ref[k]).max(), np.abs(bp - bp_ref[k]).max())
        assert err <= EULER_TOL * scale, f"interface {k} idir {idir}: {err:.3e} > {EULER_TOL:g} x {scale:.3e}"


def test_oracle_euler_transverse_matches_reference_cudaclaw():
    """clawpack46_rpt2_euler4 as the oracle restates it (Roe averages of the two
    cells, three waves, split by the sign of their speeds) against the reference's
    GPU port shockbubble_rpt2euler4.  The port takes 1/(2a) as 0.5 rsqrt(a^2), one
    unit in the last place from the division, so the outputs agree to 1e-13 of the
    interface's largest value."""
    d = _fixture()
    ql, qr, asdq = mk.euler_inputs()
    assert np.array_equal(ql, d["euler_ql"]) and np.array_equal(asdq, d["euler_asdq"])
    for idir in (0, 1):
        _euler_check(ql, qr, asdq, d[f"euler_bm_{idir}"], d[f"euler_bp_{idir}"], idir)


def test_oracle_limiters_match_reference_cudaclaw_bitwise():
    from oracle import pyoracle as po
    d = _fixture()
    r = d["limiter_r"]
    for lim in range(6):
        mine = np.array([po.limiter_phi(lim, float(x)) for x in r])
        assert np.array_equal(mine, d[f"limiter_phi_{lim}"]), f"limiter {lim}"


@pytest.mark.gpu
@pytest.mark.parametrize("family", sorted(mk.FAMILIES))
@pytest.mark.parametrize("seed", [1, 2])
def test_oracle_update_matches_reference_cudaclaw_live(family, seed):
    """The same comparison on fresh seeds, running the reference's kernel now."""
    from oracle import pin_reference as pr
    if not pr.available():
        pytest.skip("oracle/_ref/libpin_cudaclaw.so not built (reference tree absent at build time)")
    solver, _, _, fw, grav, cases = mk.FAMILIES[family]
    q, aux, dx, dt = mk.inputs(family, seed=seed, npatch=8)
    for order, lim in cases:
        ref, _ = pr.step(solver, q, aux, dx, dt, order, lim, use_fwaves=fw, grav=grav)
        _assert_close(_oracle_step(family, q, aux, dx, dt, order, lim), ref,
                      f"{family} seed {seed} order {order} limiters {lim}")


@pytest.mark.gpu
def test_oracle_euler_transverse_matches_reference_cudaclaw_live():
    from oracle import pin_reference as pr
    if not pr.available():
        pytest.skip("oracle/_ref/libpin_cudaclaw.so not built (reference tree absent at build time)")
    ql, qr, asdq = mk.euler_inputs(seed=7, n=2048)
    for idir in (0, 1):
        bm, bp = pr.euler_rpt2(idir, ql, qr, asdq, 1.4)
        _euler_check(ql, qr, asdq, bm, bp, idir)
