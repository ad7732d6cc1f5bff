"""The reference's own CUDA patch update, run to pin the CPU oracle.

Test infrastructure (the checker's checker): ``oracle/_ref/libpin_cudaclaw.so``
is built by ``make -C oracle ref`` from the reference tree's
``src/solvers/fc2d_cudaclaw/cuda_source/cudaclaw_flux2.cu`` and
``cudaclaw_limiters.cu`` plus ``oracle/ref_cudaclaw/pin_harness.cu``.  Calling it
needs a GPU; only the golden-vector script and the tests load it.
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
    """Compile the library when the reference tree and nvcc are present; True if it exists."""
    ref = os.environ.get("FCB_REFERENCE_TREE", "/root/reference")
    if os.path.isdir(os.path.join(ref, "src", "solvers", "fc2d_cudaclaw")) and shutil.which("make"):
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
        L.pin_cudaclaw_advection_step.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ip,
                                                  ctypes.c_int, ctypes.c_double, dp, dp, dp, dp, dp]
        L.pin_cudaclaw_advection_step.restype = ctypes.c_int
        L.pin_cudaclaw_limiter.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int]
        L.pin_cudaclaw_limiter.restype = ctypes.c_int
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def advection_step(q, aux, dx, dy, dt, order, mthlim, mbc=2):
    """One cudaclaw update of scalar-advection patches.  q: (npatch, ny, nx) with
    mbc ghost cells, aux: (npatch, 2, ny, nx) velocities; returns (q after, cfl per patch)."""
    q = np.ascontiguousarray(q, np.float64).copy()
    aux = np.ascontiguousarray(aux, np.float64)
    npatch, ny, nx = q.shape
    mx, my = nx - 2 * mbc, ny - 2 * mbc
    dx = np.ascontiguousarray(np.broadcast_to(np.asarray(dx, np.float64), (npatch,)))
    dy = np.ascontiguousarray(np.broadcast_to(np.asarray(dy, np.float64), (npatch,)))
    cfl = np.zeros(npatch)
    o = (ctypes.c_int * 2)(*order)
    rc = lib().pin_cudaclaw_advection_step(mx, my, mbc, npatch, o, int(mthlim), float(dt), _dp(dx), _dp(dy),
                                           _dp(q), _dp(aux), _dp(cfl))
    if rc != 0:
        raise RuntimeError(f"cudaclaw update failed: CUDA error {rc}")
    return q, cfl


def limiter(lim, r):
    r = np.ascontiguousarray(r, np.float64)
    phi = np.zeros_like(r)
    rc = lib().pin_cudaclaw_limiter(int(lim), _dp(r), _dp(phi), r.size)
    if rc != 0:
        raise RuntimeError(f"cudaclaw limiter failed: CUDA error {rc}")
    return phi
