"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle is the checker the CUDA product is compared against and the timed
CPU baseline.  Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg
of ``bench.py`` import this module; the product package never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liborc.so")

RP_ADVECTION, RP_SW_ROE, RP_SW_FWAVE, RP_EULER_EXACT, RP_ADVECTION_MANIFOLD, RP_ACOUSTICS = 0, 1, 2, 3, 4, 5
PROB_SWIRL, PROB_RADIALDAM, PROB_UNIFORM_SW, PROB_TSUNAMI, PROB_SHOCKBUBBLE, PROB_SPHERE = 0, 1, 2, 3, 4, 5
PROB_ROTATION, PROB_ACOUSTICS = 6, 7


class OrcConfig(ctypes.Structure):
    _fields_ = [
        ("mx", ctypes.c_int), ("my", ctypes.c_int), ("mbc", ctypes.c_int),
        ("meqn", ctypes.c_int), ("maux", ctypes.c_int),
        ("mwaves", ctypes.c_int), ("order", ctypes.c_int * 2), ("mthlim", ctypes.c_int * 8),
        ("mthbc", ctypes.c_int * 4), ("mcapa", ctypes.c_int), ("use_fwaves", ctypes.c_int),
        ("rp", ctypes.c_int),
        ("minlevel", ctypes.c_int), ("maxlevel", ctypes.c_int), ("subcycle", ctypes.c_int),
        ("time_sync", ctypes.c_int), ("flux_correction", ctypes.c_int),
        ("fluctuation_correction", ctypes.c_int), ("regrid_interval", ctypes.c_int),
        ("refine_threshold", ctypes.c_double), ("coarsen_threshold", ctypes.c_double),
        ("ax", ctypes.c_double), ("bx", ctypes.c_double), ("ay", ctypes.c_double), ("by", ctypes.c_double),
        ("mi", ctypes.c_int), ("mj", ctypes.c_int),
        ("problem", ctypes.c_int), ("grav", ctypes.c_double), ("tperiod", ctypes.c_double),
        ("r0", ctypes.c_double), ("hin", ctypes.c_double), ("hout", ctypes.c_double),
        ("x0", ctypes.c_double), ("y0", ctypes.c_double), ("qinit_sharp", ctypes.c_int),
        ("pdata", ctypes.c_double * 32),
        ("gamma", ctypes.c_double), ("mach", ctypes.c_double), ("rhob", ctypes.c_double),
        ("newton_tol", ctypes.c_double),
        ("nthreads", ctypes.c_int),
        ("smooth_refine", ctypes.c_int), ("smooth_level", ctypes.c_int),
        ("tag_criteria", ctypes.c_int), ("threshold_variable", ctypes.c_int),
        ("tfinal", ctypes.c_double), ("initial_dt", ctypes.c_double),
        ("max_cfl", ctypes.c_double), ("desired_cfl", ctypes.c_double),
        ("nout", ctypes.c_int), ("use_fixed_dt", ctypes.c_int),
        ("src_kind", ctypes.c_int), ("src_rate", ctypes.c_double),
    ]


TAG_APP, TAG_VALUE, TAG_DIFFERENCE, TAG_MINMAX, TAG_GRADIENT, TAG_GRADIENT_DX = 0, 1, 2, 3, 4, 5


class OrcRunStats(ctypes.Structure):
    _fields_ = [("count_amr_advance", ctypes.c_int), ("count_amr_regrid", ctypes.c_int),
                ("count_amr_new_domain", ctypes.c_int), ("global_num_patches", ctypes.c_int),
                ("rejected", ctypes.c_int), ("steps", ctypes.c_int), ("t_final", ctypes.c_double)]


def build(force: bool = False) -> str:
    """Compile liborc.so from the sources beside this file (make; a no-op when up to date)."""
    cmd = ["make", "-s", "-C", _HERE] + (["-B"] if force else [])
    try:
        subprocess.run(cmd, check=True)
    except (OSError, subprocess.CalledProcessError):
        if force or not os.path.exists(_LIB):
            raise
    return _LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB)
        P = ctypes.c_void_p
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.orc_create.restype = P
        L.orc_create.argtypes = [ctypes.POINTER(OrcConfig)]
        L.orc_destroy.argtypes = [P]
        L.orc_initialize.argtypes = [P]
        L.orc_advance.restype = ctypes.c_double
        L.orc_advance.argtypes = [P, ctypes.c_double, ctypes.c_double]
        L.orc_regrid.argtypes = [P]
        L.orc_ghost_update_all.argtypes = [P, ctypes.c_double]
        L.orc_run.argtypes = [P, ctypes.POINTER(OrcRunStats)]
        L.orc_save_step.argtypes = [P]
        L.orc_restore_step.argtypes = [P]
        L.orc_num_patches.argtypes = [P]
        L.orc_patch_info.argtypes = [P, ip, ip, ip, ip]
        L.orc_get_q.argtypes = [P, dp]
        L.orc_set_q.argtypes = [P, dp]
        L.orc_get_aux.argtypes = [P, dp]
        L.orc_mass.argtypes = [P, dp]
        L.orc_cell_updates.restype = ctypes.c_double
        L.orc_cell_updates.argtypes = [P]
        L.orc_registers_size.argtypes = [P]
        L.orc_get_registers.argtypes = [P, dp]
        L.orc_patch_step2.restype = ctypes.c_double
        L.orc_patch_step2.argtypes = [ctypes.POINTER(OrcConfig), dp, dp, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, dp, dp, dp, dp]
        L.orc_limiter_phi.restype = ctypes.c_double
        L.orc_limiter_phi.argtypes = [ctypes.c_int, ctypes.c_double]
        for fn in ("orc_log", "orc_exp"):
            getattr(L, fn).restype = ctypes.c_double
            getattr(L, fn).argtypes = [ctypes.c_double]
        L.orc_pow.restype = ctypes.c_double
        L.orc_pow.argtypes = [ctypes.c_double, ctypes.c_double]
        L.orc_euler_star.restype = ctypes.c_int
        L.orc_euler_star.argtypes = [ctypes.c_double, dp, dp, ctypes.c_double, ctypes.c_double, dp]
        L.orc_euler_interface.restype = ctypes.c_int
        L.orc_euler_interface.argtypes = [ctypes.c_double, ctypes.c_double, dp, dp, ctypes.c_double, dp, dp, dp, dp]
        L.orc_euler_postshock.argtypes = [ctypes.c_double, ctypes.c_double, dp]
        L.orc_euler_rpt2_point.argtypes = [ctypes.c_double, ctypes.c_int, dp, dp, dp, dp, dp]
        L.orc_euler_rpt2_point.restype = None
        L.orc_newton_hist.argtypes = [ctypes.POINTER(ctypes.c_long), ctypes.c_int]
        _lib = L
    return _lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def make_config(**kw) -> OrcConfig:
    c = OrcConfig()
    defaults = dict(mx=16, my=16, mbc=2, meqn=1, maux=0, mwaves=1, mcapa=0, use_fwaves=0, rp=0,
                    minlevel=0, maxlevel=0, subcycle=0, time_sync=0, flux_correction=1,
                    fluctuation_correction=1, regrid_interval=1, refine_threshold=0.5,
                    coarsen_threshold=0.1, ax=0.0, bx=1.0, ay=0.0, by=1.0, mi=1, mj=1,
                    problem=0, grav=1.0, tperiod=0.0, r0=0.3, hin=2.0, hout=1.0, x0=0.0, y0=0.0,
                    qinit_sharp=1, gamma=1.4, mach=1.22, rhob=0.138, newton_tol=1e-10, nthreads=0,
                    smooth_refine=0, smooth_level=0, tag_criteria=0, threshold_variable=1,
                    tfinal=0.0, initial_dt=0.0, max_cfl=1.0, desired_cfl=0.9, nout=1, use_fixed_dt=0,
                    src_kind=0, src_rate=0.0)
    defaults.update(kw)
    order = defaults.pop("order", (2, 2))
    mthlim = defaults.pop("mthlim", (4,) * 8)
    mthbc = defaults.pop("mthbc", (1, 1, 1, 1))
    pdata = defaults.pop("pdata", ())
    for k, v in defaults.items():
        setattr(c, k, v)
    for i, v in enumerate(order):
        c.order[i] = v
    for i, v in enumerate(mthlim):
        c.mthlim[i] = v
    for i, v in enumerate(mthbc):
        c.mthbc[i] = v
    for i, v in enumerate(pdata):
        c.pdata[i] = v
    return c


class OracleSim:
    """One oracle simulation: a forest of patches advanced on the host cores."""

    def __init__(self, cfg: OrcConfig):
        self.cfg = cfg
        self._cfg_ref = ctypes.byref(cfg)
        self.h = lib().orc_create(self._cfg_ref)
        self.nx = cfg.mx + 2 * cfg.mbc
        self.ny = cfg.my + 2 * cfg.mbc

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def initialize(self) -> int:
        return lib().orc_initialize(self.h)

    def advance(self, t: float, dt: float) -> float:
        return lib().orc_advance(self.h, t, dt)

    def regrid(self) -> int:
        return lib().orc_regrid(self.h)

    def ghost_update(self, t: float) -> None:
        lib().orc_ghost_update_all(self.h, t)

    def run(self) -> dict:
        """fclaw2d_run outstyle 1 from t = 0; returns the run's counters."""
        st = OrcRunStats()
        lib().orc_run(self.h, ctypes.byref(st))
        return {k: getattr(st, k) for k, _ in OrcRunStats._fields_}

    def save_step(self) -> None:
        lib().orc_save_step(self.h)

    def restore_step(self) -> None:
        lib().orc_restore_step(self.h)

    @property
    def num_patches(self) -> int:
        return lib().orc_num_patches(self.h)

    def patch_info(self) -> np.ndarray:
        n = self.num_patches
        arrs = [np.zeros(n, np.int32) for _ in range(4)]
        lib().orc_patch_info(self.h, *[_iptr(a) for a in arrs])
        return np.stack(arrs, axis=1)   # level, block, gx, gy

    def get_q(self) -> np.ndarray:
        n = self.num_patches
        out = np.zeros((n, self.cfg.meqn, self.ny, self.nx), np.float64)
        lib().orc_get_q(self.h, _dptr(out))
        return out

    def set_q(self, q: np.ndarray) -> None:
        q = np.ascontiguousarray(q, dtype=np.float64)
        lib().orc_set_q(self.h, _dptr(q))

    def get_aux(self) -> np.ndarray:
        n = self.num_patches
        out = np.zeros((n, max(self.cfg.maux, 0), self.ny, self.nx), np.float64)
        lib().orc_get_aux(self.h, _dptr(out))
        return out

    def get_registers(self) -> np.ndarray:
        n = self.num_patches
        sz = lib().orc_registers_size(self.h)
        out = np.zeros((n, sz), np.float64)
        lib().orc_get_registers(self.h, _dptr(out))
        return out

    def mass(self) -> np.ndarray:
        out = np.zeros(self.cfg.meqn, np.float64)
        lib().orc_mass(self.h, _dptr(out))
        return out

    @property
    def cell_updates(self) -> float:
        return lib().orc_cell_updates(self.h)


def patch_step2(cfg: OrcConfig, q: np.ndarray, aux, dx: float, dy: float, dt: float):
    """clawpack46_step2_wrap on one patch (q updated in place); returns cfl, fm, fp, gm, gp."""
    n = q.size
    fm, fp, gm, gp = (np.zeros(n) for _ in range(4))
    a = aux if aux is not None else np.zeros(1)
    cfl = lib().orc_patch_step2(ctypes.byref(cfg), _dptr(q), _dptr(a), dx, dy, dt,
                                _dptr(fm), _dptr(fp), _dptr(gm), _dptr(gp))
    return cfl, fm, fp, gm, gp


def limiter_phi(mthlim: int, r: float) -> float:
    return lib().orc_limiter_phi(mthlim, r)


# ---- exact Euler solver (unit tests) -------------------------------------------
def euler_star(gam, wl, wr, seed=0.0, tol=1e-10):
    """(p*, u*, rho*L, rho*R, a*L, a*R), Newton iterations for primitive states (rho, u, p)."""
    a, b = np.asarray(wl, np.float64), np.asarray(wr, np.float64)
    out = np.zeros(6)
    it = lib().orc_euler_star(gam, _dptr(a), _dptr(b), seed, tol, _dptr(out))
    return out, it


def euler_interface(gam, ql, qr, seed=0.0, tol=1e-10):
    """waves (3, 4), speeds (3,), amdq, apdq, iterations for conserved states (rho, m_n, m_t, E)."""
    a, b = np.ascontiguousarray(ql, np.float64), np.ascontiguousarray(qr, np.float64)
    w, s, am, ap = np.zeros((3, 4)), np.zeros(3), np.zeros(4), np.zeros(4)
    it = lib().orc_euler_interface(gam, tol, _dptr(a), _dptr(b), seed, _dptr(w), _dptr(s), _dptr(am), _dptr(ap))
    return w, s, am, ap, it


def euler_rpt2(gam, ixy, qlo, qhi, asdq):
    """clawpack46_rpt2_euler4 of one interface (Roe averages of qlo | qhi): (bmasdq, bpasdq)."""
    a, b, c = (np.ascontiguousarray(x, np.float64) for x in (qlo, qhi, asdq))
    bm, bp = np.zeros(4), np.zeros(4)
    lib().orc_euler_rpt2_point(gam, int(ixy), _dptr(a), _dptr(b), _dptr(c), _dptr(bm), _dptr(bp))
    return bm, bp


def euler_postshock(gam, mach):
    out = np.zeros(3)
    lib().orc_euler_postshock(gam, mach, _dptr(out))
    return out


def newton_hist(reset=False) -> np.ndarray:
    out = (ctypes.c_long * 32)()
    lib().orc_newton_hist(out, int(reset))
    return np.array(out[:], np.int64)
