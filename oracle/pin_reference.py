"""The reference's own CUDA patch update, run to pin the CPU oracle.

Test infrastructure (the checker's checker): ``oracle/_ref/libpin_cudaclaw.so``
is built by ``make -C oracle ref`` from the reference tree's
``src/solvers/fc2d_cudaclaw/cuda_source/cudaclaw_flux2.cu`` and
``cudaclaw_limiters.cu``, the cudaclaw app Riemann solvers (swirl advection,
radialdam Roe, shock-bubble Euler transverse) and ``oracle/ref_cudaclaw/{pin_harness,
ref_app_solvers}.cu``.  Calling it needs a GPU; only the golden-vector script and
the tests load it.
"""
from __future__ import annotations

import ctypes
import os
import shutil
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_ref", "libpin_cudaclaw.so")
_lib = None


def build() -> bool:
    """Compile the library when the reference tree (FCB_REFERENCE_TREE) and nvcc are
    present; True if the library exists.  Without the variable nothing is compiled."""
    ref = os.environ.get("FCB_REFERENCE_TREE", "")
    if ref and os.path.isdir(os.path.join(ref, "src", "solvers", "fc2d_cudaclaw")) and shutil.which("make"):
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF={ref}"], check=True)
    return os.path.exists(LIB)


def available() -> bool:
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        I = ctypes.c_int
        L.pin_cudaclaw_step.argtypes = [I, I, I, I, I, I, I, I, I, ip, ip, ctypes.c_double, dp, dp, dp, dp, dp, dp]
        L.pin_cudaclaw_step.restype = ctypes.c_int
        L.pin_ref_euler_rpt2.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, dp, dp, dp, dp, dp]
        L.pin_ref_euler_rpt2.restype = ctypes.c_int
        L.pin_cudaclaw_limiter.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int]
        L.pin_cudaclaw_limiter.restype = ctypes.c_int
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


SWIRL, RADIALDAM = 0, 1          # reference solver pairs


def step(solver, q, aux, dx, dt, order, mthlim, use_fwaves=0, grav=1.0, dry_tolerance=1e-3, sea_level=0.0,
         mbc=2):
    """One cudaclaw update of square-cell patches.  q: (npatch, meqn, ny, nx) with mbc
    ghost cells, aux: (npatch, maux, ny, nx) or None; returns (q after, cfl per patch)."""
    q = np.ascontiguousarray(q, np.float64).copy()
    npatch, meqn, ny, nx = q.shape
    if aux is None:
        aux = np.zeros((npatch, 0, ny, nx))
    aux = np.ascontiguousarray(aux, np.float64)
    maux = aux.shape[1]
    mwaves = len(mthlim)
    mx, my = nx - 2 * mbc, ny - 2 * mbc
    d = np.full(npatch, float(dx))
    cfl = np.zeros(npatch)
    prm = np.array([grav, dry_tolerance, sea_level], np.float64)
    o = (ctypes.c_int * 2)(*order)
    lim = (ctypes.c_int * mwaves)(*mthlim)
    auxp = aux if maux > 0 else np.zeros(1)
    rc = lib().pin_cudaclaw_step(solver, mx, my, mbc, meqn, maux, mwaves, int(use_fwaves), npatch, o, lim,
                                 float(dt), _dp(d), _dp(d), _dp(prm), _dp(q), _dp(auxp), _dp(cfl))
    if rc != 0:
        raise RuntimeError(f"cudaclaw update failed: code {rc}")
    return q, cfl


def euler_rpt2(idir, ql, qr, asdq, gamma=1.4):
    """The reference's Euler transverse solver (shockbubble_rpt2euler4) on n interfaces:
    ql, qr the cells below / above, asdq the fluctuation, all (n, 4); returns bm, bp."""
    a, b, c = (np.ascontiguousarray(x, np.float64) for x in (ql, qr, asdq))
    bm, bp = np.zeros_like(a), np.zeros_like(a)
    rc = lib().pin_ref_euler_rpt2(int(idir), a.shape[0], float(gamma), _dp(a), _dp(b), _dp(c), _dp(bm), _dp(bp))
    if rc != 0:
        raise RuntimeError(f"reference Euler transverse solver failed: code {rc}")
    return bm, bp


def limiter(lim, r):
    r = np.ascontiguousarray(r, np.float64)
    phi = np.zeros_like(r)
    rc = lib().pin_cudaclaw_limiter(int(lim), _dp(r), _dp(phi), r.size)
    if rc != 0:
        raise RuntimeError(f"cudaclaw limiter failed: CUDA error {rc}")
    return phi
