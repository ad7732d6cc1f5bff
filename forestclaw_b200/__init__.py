"""forestclaw_b200 -- B200-native (sm_100a) clawpack 4.6 patch update, ghost fill and
conservative time sync for ForestClaw-style forests of patches.

The product is ``libfc2d_b200.so`` (C ABI in ``include/fc2d_b200.h``).  This module
is a thin ctypes mirror of that ABI with the names and option keys of the
reference's ``fc2d_clawpack46`` / ``fclaw`` options, so Python callers (and the
tests) drive the same entry points a ForestClaw C shim would.  There is no CPU
fallback: if the library or a GPU is missing, constructing a :class:`Solver`
raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfc2d_b200.so")

RP_ADVECTION, RP_SW_ROE, RP_SW_FWAVE, RP_EULER_EXACT, RP_ADVECTION_MANIFOLD = 0, 1, 2, 3, 4
RP_USER = 100   # application __device__ solvers (include/fc2d_b200_user.cuh)
APP_NONE, APP_SWIRL, APP_RADIALDAM, APP_TSUNAMI, APP_SHOCKBUBBLE, APP_SPHERE = 0, 1, 2, 3, 4, 5
PREC_FP64, PREC_FP32WAVE = 0, 1
# refinement criteria: FCLAW_REFINE_CRITERIA_* + 1; TAG_APP = the app's built-in one
TAG_APP, TAG_VALUE, TAG_DIFFERENCE, TAG_MINMAX, TAG_GRADIENT, TAG_GRADIENT_DX = 0, 1, 2, 3, 4, 5


class B200Error(RuntimeError):
    """A failed fc2d_b200_* call (status code and library message)."""

    def __init__(self, fn: str, code: int, msg: str):
        super().__init__(f"{fn} failed ({code}): {msg}")
        self.code = code


class _Options(ctypes.Structure):
    _fields_ = [
        ("mx", ctypes.c_int), ("my", ctypes.c_int), ("mbc", ctypes.c_int), ("meqn", ctypes.c_int),
        ("maux", ctypes.c_int), ("mwaves", ctypes.c_int), ("order", ctypes.c_int * 2),
        ("mthlim", ctypes.c_int * 8), ("mthbc", ctypes.c_int * 4), ("mcapa", ctypes.c_int),
        ("use_fwaves", ctypes.c_int), ("rp", ctypes.c_int), ("minlevel", ctypes.c_int),
        ("maxlevel", ctypes.c_int), ("subcycle", ctypes.c_int), ("time_sync", ctypes.c_int),
        ("flux_correction", ctypes.c_int), ("fluctuation_correction", ctypes.c_int),
        ("refine_threshold", ctypes.c_double), ("coarsen_threshold", ctypes.c_double),
        ("ax", ctypes.c_double), ("bx", ctypes.c_double), ("ay", ctypes.c_double), ("by", ctypes.c_double),
        ("mi", ctypes.c_int), ("mj", ctypes.c_int), ("app", ctypes.c_int), ("grav", ctypes.c_double),
        ("tperiod", ctypes.c_double), ("r0", ctypes.c_double), ("hin", ctypes.c_double),
        ("hout", ctypes.c_double), ("x0", ctypes.c_double), ("y0", ctypes.c_double),
        ("pdata", ctypes.c_double * 32),
        ("gamma", ctypes.c_double), ("mach", ctypes.c_double), ("rhob", ctypes.c_double),
        ("newton_tol", ctypes.c_double),
        ("precision", ctypes.c_int), ("device", ctypes.c_int),
        ("smooth_refine", ctypes.c_int), ("smooth_level", ctypes.c_int),
        ("refinement_criteria", ctypes.c_int), ("threshold_variable", ctypes.c_int),
        ("qinit_cellave", ctypes.c_int),
        ("regrid_interval", ctypes.c_int), ("nout", ctypes.c_int), ("use_fixed_dt", ctypes.c_int),
        ("tfinal", ctypes.c_double), ("initial_dt", ctypes.c_double), ("max_cfl", ctypes.c_double),
        ("desired_cfl", ctypes.c_double),
    ]


class _RunStats(ctypes.Structure):
    _fields_ = [("count_amr_advance", ctypes.c_int), ("count_amr_regrid", ctypes.c_int),
                ("count_amr_new_domain", ctypes.c_int), ("global_num_patches", ctypes.c_int),
                ("rejected", ctypes.c_int), ("steps", ctypes.c_int), ("t_final", ctypes.c_double)]


class _Instance(ctypes.Structure):
    _fields_ = [
        ("minlevel", ctypes.c_int), ("maxlevel", ctypes.c_int),
        ("ax", ctypes.c_double), ("bx", ctypes.c_double), ("ay", ctypes.c_double), ("by", ctypes.c_double),
        ("mi", ctypes.c_int), ("mj", ctypes.c_int), ("pdata", ctypes.c_double * 32),
    ]


MAX_INSTANCES = 256


@dataclass
class Options:
    """fc2d_b200_options_t with the reference's option names and defaults."""
    mx: int = 16
    my: int = 16
    mbc: int = 2
    meqn: int = 1
    maux: int = 0
    mwaves: int = 1
    order: Sequence[int] = (2, 2)
    mthlim: Sequence[int] = (4,)
    mthbc: Sequence[int] = (1, 1, 1, 1)
    mcapa: int = 0
    use_fwaves: int = 0
    rp: int = RP_ADVECTION
    minlevel: int = 0
    maxlevel: int = 0
    subcycle: int = 0
    time_sync: int = 0
    flux_correction: int = 1
    fluctuation_correction: int = 1
    refine_threshold: float = 0.5
    coarsen_threshold: float = 0.1
    ax: float = 0.0
    bx: float = 1.0
    ay: float = 0.0
    by: float = 1.0
    mi: int = 1
    mj: int = 1
    app: int = APP_NONE
    grav: float = 1.0
    tperiod: float = 0.0
    r0: float = 0.3
    hin: float = 2.0
    hout: float = 1.0
    x0: float = 0.0
    y0: float = 0.0
    pdata: Sequence[float] = field(default_factory=tuple)
    gamma: float = 1.4
    mach: float = 1.22
    rhob: float = 0.138
    newton_tol: float = 1e-10
    precision: int = PREC_FP64
    device: int = 0
    smooth_refine: int = 0
    smooth_level: int = 0
    refinement_criteria: int = TAG_APP
    threshold_variable: int = 1
    qinit_cellave: int = 0
    regrid_interval: int = 1
    nout: int = 1
    use_fixed_dt: int = 0
    tfinal: float = 0.0
    initial_dt: float = 0.0
    max_cfl: float = 1.0
    desired_cfl: float = 0.9

    def to_c(self) -> _Options:
        o = _Options()
        for k in ("mx", "my", "mbc", "meqn", "maux", "mwaves", "mcapa", "use_fwaves", "rp", "minlevel",
                  "maxlevel", "subcycle", "time_sync", "flux_correction", "fluctuation_correction",
                  "refine_threshold", "coarsen_threshold", "ax", "bx", "ay", "by", "mi", "mj", "app", "grav",
                  "tperiod", "r0", "hin", "hout", "x0", "y0", "gamma", "mach", "rhob", "newton_tol",
                  "precision", "device", "smooth_refine", "smooth_level", "refinement_criteria",
                  "threshold_variable", "qinit_cellave", "regrid_interval", "nout", "use_fixed_dt", "tfinal",
                  "initial_dt", "max_cfl", "desired_cfl"):
            setattr(o, k, getattr(self, k))
        for i, v in enumerate(self.order):
            o.order[i] = v
        for i, v in enumerate(self.mthlim):
            o.mthlim[i] = v
        for i, v in enumerate(self.mthbc):
            o.mthbc[i] = v
        for i, v in enumerate(self.pdata):
            o.pdata[i] = v
        return o


_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the CUDA library (built in-tree by forestclaw_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: run `python -m forestclaw_b200.build` first")
    L = ctypes.CDLL(path)
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    fp = ctypes.POINTER(ctypes.c_float)
    sig = {
        "fc2d_b200_create": [ctypes.POINTER(_Options), ctypes.POINTER(P)],
        "fc2d_b200_destroy": [P],
        "fc2d_b200_set_riemann": [P, I],
        "fc2d_b200_initialize": [P],
        "fc2d_b200_set_forest": [P, I, ip, ip, ip],
        "fc2d_b200_num_patches": [P, ip],
        "fc2d_b200_patch_info": [P, ip, ip, ip, ip],
        "fc2d_b200_get_q": [P, dp],
        "fc2d_b200_set_q": [P, dp],
        "fc2d_b200_get_aux": [P, dp],
        "fc2d_b200_set_aux": [P, dp],
        "fc2d_b200_registers_size": [P, ip],
        "fc2d_b200_get_registers": [P, dp],
        "fc2d_b200_level_update": [P, I, D, D, dp],
        "fc2d_b200_single_step_update": [P, I, I, I, D, D, dp],
        "fc2d_b200_single_step_update_host": [P, I, I, I, dp, dp, I, I, D, D, dp],
        "fc2d_b200_ghost_update": [P, I, I, D, I],
        "fc2d_b200_timeinterp": [P, I, D],
        "fc2d_b200_time_sync": [P, I, I],
        "fc2d_b200_advance": [P, D, D, dp],
        "fc2d_b200_regrid": [P, ip],
        "fc2d_b200_save_step": [P],
        "fc2d_b200_set_user_variants": [P, P, I, I, I, I, I],
        "fc2d_b200_set_partition": [P, P],
        "fc2d_b200_partition_owner": [P, ip],
        "fc2d_b200_sync_replicas": [P],
        "fc2d_b200_partition_plan": [ctypes.POINTER(_Options), I, ip, ip, ip, I, I, ip, ip, ip,
                                     ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(ctypes.c_ulonglong)],
        "fc2d_b200_restore_step": [P],
        "fc2d_b200_run": [P, ctypes.POINTER(_RunStats)],
        "fc2d_b200_mass": [P, dp],
        "fc2d_b200_cell_updates": [P, dp],
        "fc2d_b200_synchronize": [P],
        "fc2d_b200_last_update_stats": [P, dp, dp, ip, ip],
        "fc2d_b200_last_step_timing": [P, dp, dp],
        "fc2d_b200_graph_stats": [P, ip, ip],
        "fc2d_b200_last_regrid_stats": [P, dp],
        "fc2d_b200_set_timing": [P, I],
        "fc2d_b200_event_record": [P, I],
        "fc2d_b200_event_elapsed": [P, I, I, dp],
        "fc2d_b200_get_stream": [P, ctypes.POINTER(P)],
        "fc2d_b200_set_graphs": [P, I],
        "fc2d_b200_set_programmatic_launch": [P, I],
        "fc2d_b200_mass_noalloc": [P, ctypes.POINTER(ctypes.c_double)],
        "fc2d_b200_newton_histogram": [P, ctypes.POINTER(ctypes.c_ulonglong), I],
        "fc2d_b200_mlp_create": [I, ctypes.c_ulonglong, ctypes.POINTER(P)],
        "fc2d_b200_mlp_destroy": [P],
        "fc2d_b200_mlp_set_params": [P, fp],
        "fc2d_b200_mlp_get_params": [P, fp],
        "fc2d_b200_mlp_set_data": [P, dp, I, D, D],
        "fc2d_b200_mlp_get_data": [P, fp, fp],
        "fc2d_b200_mlp_train": [P, I, I, ctypes.c_float, ctypes.c_ulonglong, dp],
        "fc2d_b200_mlp_gradient": [P, fp, fp, I, fp, dp],
        "fc2d_b200_mlp_predict": [P, fp, I, fp],
        "fc2d_b200_mlp_set_tensor_form": [P, I],
        "fc2d_b200_mlp_newton_histogram": [P, I, ctypes.POINTER(ctypes.c_longlong)],
        "fc2d_b200_sample_interfaces": [P, I, ctypes.c_ulonglong, dp],
        "fc2d_b200_set_pstar_seed": [P, P],
        "fc2d_b200_set_instances": [P, I, ctypes.POINTER(_Instance)],
        "fc2d_b200_num_instances": [P, ip],
        "fc2d_b200_patch_instance": [P, ip],
        "fc2d_b200_advance_instances": [P, dp, dp],
        "fc2d_b200_advance_instances_begin": [P, dp],
        "fc2d_b200_advance_instances_end": [P, dp],
        "fc2d_b200_mass_instances": [P, dp],
        "fc2d_b200_num_variants": [P, ip, ip],
        "fc2d_b200_variant_info": [P, I, ip, ip, ip, ip, ip],
        "fc2d_b200_set_variant": [P, I],
        "fc2d_b200_autotune": [P, I, ip, dp],
        "fc2d_b200_level_variants": [P, ip],
        "fc2d_b200_set_level_variants": [P, ip],
        "fc2d_b200_output_ascii": [P, ctypes.c_char_p, I, D],
        "fc2d_b200_output_vtk": [P, ctypes.c_char_p, I],
        "fc2d_b200_write_vtk_file": [ctypes.c_char_p, I, I, I, I, ip, dp, ctypes.POINTER(ctypes.c_float)],
        "fc2d_b200_write_ascii_frame": [ctypes.c_char_p, I, D, I, I, I, I, I, I, ip, ip, dp, dp, dp, dp, dp],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    L.fc2d_b200_last_error.restype = ctypes.c_char_p
    L.fc2d_b200_last_error.argtypes = []
    _lib = L
    return L


def write_ascii_frame(directory: str, iframe: int, time: float, q: np.ndarray, level, block, xlower, ylower, dx, dy,
                      mbc: int = 2, maux: int = 0) -> None:
    """Write caller-supplied patches as a clawpack 4.6 ASCII frame (host only, no device).
    q: (npatch, meqn, my + 2 mbc, mx + 2 mbc) in the FArrayBox layout; per-patch level,
    block, lower corner and spacing; patches are written in the given order."""
    lib = load_library()
    q = np.ascontiguousarray(q, np.float64)
    npatch, meqn, ny, nx = q.shape
    lv = np.ascontiguousarray(level, np.int32)
    bk = np.ascontiguousarray(block, np.int32)
    arr = [np.ascontiguousarray(v, np.float64) for v in (xlower, ylower, dx, dy)]
    rc = lib.fc2d_b200_write_ascii_frame(os.fsencode(directory), iframe, time, meqn, maux, nx - 2 * mbc,
                                         ny - 2 * mbc, mbc, npatch, _ip(lv), _ip(bk), *[_dp(v) for v in arr], _dp(q))
    if rc != 0:
        raise B200Error("fc2d_b200_write_ascii_frame", rc, "cannot write the frame")


def write_vtk_file(path: str, points: np.ndarray, values: np.ndarray, block) -> None:
    """Write caller-supplied patches as a VTK unstructured grid (host only, no device).
    points: (npatch, (my+1)(mx+1), 3) float64 (i fastest), values: (npatch, my, mx, meqn)
    float32, block: per-patch block number; patches are written in the given order."""
    lib = load_library()
    v = np.ascontiguousarray(values, np.float32)
    npatch, my, mx, meqn = v.shape
    pts = np.ascontiguousarray(points, np.float64)
    if pts.shape != (npatch, (mx + 1) * (my + 1), 3):
        raise ValueError("points must be (npatch, (mx+1)(my+1), 3)")
    bk = np.ascontiguousarray(block, np.int32)
    rc = lib.fc2d_b200_write_vtk_file(os.fsencode(path), mx, my, meqn, npatch, _ip(bk), _dp(pts),
                                      v.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    if rc != 0:
        raise B200Error("fc2d_b200_write_vtk_file", rc, "cannot write " + path)


def read_vtu(path: str) -> dict:
    """Parse a file written by write_vtk_file / Solver.output_vtk: the header's
    attributes and every appended array as a numpy array keyed by its Name."""
    import re
    with open(path, "rb") as f:
        raw = f.read()
    start = raw.index(b'<AppendedData encoding="raw">\n  _') + len(b'<AppendedData encoding="raw">\n  _')
    end = raw.rindex(b"\n </AppendedData>")
    head = raw[:start].decode()
    data = raw[start:end]
    piece = re.search(r'NumberOfPoints="(\d+)" NumberOfCells="(\d+)"', head)
    out = {"npoints": int(piece.group(1)), "ncells": int(piece.group(2)), "header": head}
    types = {"Float64": np.float64, "Float32": np.float32, "Int32": np.int32, "Int64": np.int64, "UInt8": np.uint8}
    for m in re.finditer(r'<DataArray type="(\w+)" Name="(\w+)"(?: NumberOfComponents="(\d+)")? '
                         r'format="appended" offset="(\d+)">', head):
        typ, name, ncomp, off = m.group(1), m.group(2), m.group(3), int(m.group(4))
        nbytes = int(np.frombuffer(data[off:off + 8], np.uint64)[0])
        arr = np.frombuffer(data[off + 8:off + 8 + nbytes], types[typ])
        out[name] = arr.reshape(-1, int(ncomp)) if ncomp else arr
    return out


def exported_symbols() -> list[str]:
    """Names of the C ABI entry points declared in include/fc2d_b200.h."""
    hdr = os.path.join(os.path.dirname(_HERE), "include", "fc2d_b200.h")
    import re
    with open(hdr) as f:
        txt = f.read()
    return sorted(set(re.findall(r"\b(fc2d_b200_[a-z_0-9]+)\s*\(", txt)))


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _fp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


MLP_NPARAM = 4673


class PStarMLP:
    """The p*-seed network of the exact Euler solver and its GPU trainer
    (fc2d_b200_mlp_*): parameters W1[64][6] b1 W2[64][64] b2 w3[64] b3."""

    def __init__(self, device: int = 0, seed: int = 0):
        self.lib = load_library()
        h = ctypes.c_void_p()
        self._check("fc2d_b200_mlp_create", self.lib.fc2d_b200_mlp_create(device, seed, ctypes.byref(h)))
        self.h = h
        self.n = 0

    def _check(self, fn: str, rc: int) -> None:
        if rc != 0:
            raise B200Error(fn, rc, (self.lib.fc2d_b200_last_error() or b"").decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.fc2d_b200_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        out = np.zeros(MLP_NPARAM, np.float32)
        self._check("fc2d_b200_mlp_get_params", self.lib.fc2d_b200_mlp_get_params(self.h, _fp(out)))
        return out

    @params.setter
    def params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == MLP_NPARAM
        self._check("fc2d_b200_mlp_set_params", self.lib.fc2d_b200_mlp_set_params(self.h, _fp(p)))

    def set_data(self, prim, gamma: float = 1.4, tol: float = 1e-12) -> None:
        prim = np.ascontiguousarray(prim, np.float64).reshape(-1, 6)
        self._check("fc2d_b200_mlp_set_data", self.lib.fc2d_b200_mlp_set_data(self.h, _dp(prim), len(prim), gamma, tol))
        self.n = len(prim)

    def data(self):
        X = np.zeros((self.n, 6), np.float32)
        Y = np.zeros(self.n, np.float32)
        self._check("fc2d_b200_mlp_get_data", self.lib.fc2d_b200_mlp_get_data(self.h, _fp(X), _fp(Y)))
        return X, Y

    def train(self, epochs: int, batch: int = 4096, lr: float = 2e-3, seed: int = 0) -> float:
        loss = ctypes.c_double()
        self._check("fc2d_b200_mlp_train", self.lib.fc2d_b200_mlp_train(self.h, epochs, batch, lr, seed, ctypes.byref(loss)))
        return loss.value

    def gradient(self, X, Y):
        X = np.ascontiguousarray(X, np.float32).reshape(-1, 6)
        Y = np.ascontiguousarray(Y, np.float32).reshape(-1)
        g = np.zeros(MLP_NPARAM, np.float32)
        loss = ctypes.c_double()
        self._check("fc2d_b200_mlp_gradient", self.lib.fc2d_b200_mlp_gradient(self.h, _fp(X), _fp(Y), len(Y), _fp(g), ctypes.byref(loss)))
        return g, loss.value

    def predict(self, X) -> np.ndarray:
        X = np.ascontiguousarray(X, np.float32).reshape(-1, 6)
        Y = np.zeros(len(X), np.float32)
        self._check("fc2d_b200_mlp_predict", self.lib.fc2d_b200_mlp_predict(self.h, _fp(X), len(X), _fp(Y)))
        return Y

    def set_tensor_form(self, tcgen05: bool) -> None:
        """Batched evaluation on the tcgen05 tensor cores (default) or in the per-warp mma.sync form."""
        self._check("fc2d_b200_mlp_set_tensor_form", self.lib.fc2d_b200_mlp_set_tensor_form(self.h, int(tcgen05)))

    def newton_histogram(self, use_mlp: bool) -> np.ndarray:
        h = (ctypes.c_longlong * 32)()
        self._check("fc2d_b200_mlp_newton_histogram", self.lib.fc2d_b200_mlp_newton_histogram(self.h, int(use_mlp), h))
        return np.array(h[:], np.int64)


class Solver:
    """A device-resident forest of patches advanced by the sm_100a kernels."""

    def __init__(self, opts: Options):
        self.lib = load_library()
        self.opts = opts
        self._c = opts.to_c()
        h = ctypes.c_void_p()
        self._check("fc2d_b200_create", self.lib.fc2d_b200_create(ctypes.byref(self._c), ctypes.byref(h)))
        self.h = h
        self.nx = opts.mx + 2 * opts.mbc
        self.ny = opts.my + 2 * opts.mbc

    def _check(self, fn: str, rc: int) -> None:
        if rc != 0:
            raise B200Error(fn, rc, (self.lib.fc2d_b200_last_error() or b"").decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.fc2d_b200_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- setup -------------------------------------------------------------
    def initialize(self) -> int:
        self._check("fc2d_b200_initialize", self.lib.fc2d_b200_initialize(self.h))
        return self.num_patches

    def set_forest(self, level, gx, gy) -> None:
        lv = np.ascontiguousarray(level, np.int32)
        x = np.ascontiguousarray(gx, np.int32)
        y = np.ascontiguousarray(gy, np.int32)
        self._check("fc2d_b200_set_forest", self.lib.fc2d_b200_set_forest(self.h, len(lv), _ip(lv), _ip(x), _ip(y)))

    @property
    def num_patches(self) -> int:
        n = ctypes.c_int()
        self._check("fc2d_b200_num_patches", self.lib.fc2d_b200_num_patches(self.h, ctypes.byref(n)))
        return n.value

    def patch_info(self) -> np.ndarray:
        n = self.num_patches
        a = [np.zeros(n, np.int32) for _ in range(4)]
        self._check("fc2d_b200_patch_info", self.lib.fc2d_b200_patch_info(self.h, *[_ip(x) for x in a]))
        return np.stack(a, axis=1)

    # -- data ---------------------------------------------------------------
    def get_q(self) -> np.ndarray:
        out = np.zeros((self.num_patches, self.opts.meqn, self.ny, self.nx), np.float64)
        self._check("fc2d_b200_get_q", self.lib.fc2d_b200_get_q(self.h, _dp(out)))
        return out

    def set_q(self, q: np.ndarray) -> None:
        q = np.ascontiguousarray(q, np.float64)
        self._check("fc2d_b200_set_q", self.lib.fc2d_b200_set_q(self.h, _dp(q)))

    def get_aux(self) -> np.ndarray:
        out = np.zeros((self.num_patches, self.opts.maux, self.ny, self.nx), np.float64)
        self._check("fc2d_b200_get_aux", self.lib.fc2d_b200_get_aux(self.h, _dp(out)))
        return out

    def set_aux(self, aux: np.ndarray) -> None:
        aux = np.ascontiguousarray(aux, np.float64)
        self._check("fc2d_b200_set_aux", self.lib.fc2d_b200_set_aux(self.h, _dp(aux)))

    def get_registers(self) -> np.ndarray:
        n = ctypes.c_int()
        self._check("fc2d_b200_registers_size", self.lib.fc2d_b200_registers_size(self.h, ctypes.byref(n)))
        out = np.zeros((self.num_patches, n.value), np.float64)
        self._check("fc2d_b200_get_registers", self.lib.fc2d_b200_get_registers(self.h, _dp(out)))
        return out

    # -- stepping -------------------------------------------------------------
    def advance(self, t: float, dt: float) -> float:
        cfl = ctypes.c_double()
        self._check("fc2d_b200_advance", self.lib.fc2d_b200_advance(self.h, t, dt, ctypes.byref(cfl)))
        return cfl.value

    def level_update(self, level: int, t: float, dt: float) -> float:
        cfl = ctypes.c_double()
        self._check("fc2d_b200_level_update", self.lib.fc2d_b200_level_update(self.h, level, t, dt, ctypes.byref(cfl)))
        return cfl.value

    def single_step_update(self, level: int, it: int, total: int, t: float, dt: float) -> float:
        cfl = ctypes.c_double()
        self._check("fc2d_b200_single_step_update",
                    self.lib.fc2d_b200_single_step_update(self.h, level, it, total, t, dt, ctypes.byref(cfl)))
        return cfl.value

    def ghost_update(self, minlevel: int, maxlevel: int, t: float, time_interp: int = 0) -> None:
        self._check("fc2d_b200_ghost_update", self.lib.fc2d_b200_ghost_update(self.h, minlevel, maxlevel, t, time_interp))

    def time_sync(self, minlevel: int, maxlevel: int) -> None:
        self._check("fc2d_b200_time_sync", self.lib.fc2d_b200_time_sync(self.h, minlevel, maxlevel))

    def regrid(self) -> int:
        c = ctypes.c_int()
        self._check("fc2d_b200_regrid", self.lib.fc2d_b200_regrid(self.h, ctypes.byref(c)))
        return c.value

    def save_step(self) -> None:
        self._check("fc2d_b200_save_step", self.lib.fc2d_b200_save_step(self.h))

    def restore_step(self) -> None:
        self._check("fc2d_b200_restore_step", self.lib.fc2d_b200_restore_step(self.h))

    def run(self) -> dict:
        """fclaw2d_run outstyle 1 from t = 0 (tfinal, nout, initial_dt, max_cfl, desired_cfl,
        regrid_interval of the options); returns the run's counters."""
        st = _RunStats()
        self._check("fc2d_b200_run", self.lib.fc2d_b200_run(self.h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in _RunStats._fields_}

    def partition_owner(self) -> np.ndarray:
        out = np.zeros(self.num_patches, np.int32)
        self._check("fc2d_b200_partition_owner", self.lib.fc2d_b200_partition_owner(self.h, _ip(out)))
        return out

    def sync_replicas(self) -> None:
        """Every rank of a partitioned forest gets every patch's current data."""
        self._check("fc2d_b200_sync_replicas", self.lib.fc2d_b200_sync_replicas(self.h))

    def mass(self) -> np.ndarray:
        out = np.zeros(self.opts.meqn, np.float64)
        self._check("fc2d_b200_mass", self.lib.fc2d_b200_mass(self.h, _dp(out)))
        return out

    def sample_interfaces(self, n: int, seed: int = 0) -> np.ndarray:
        """n normal-direction interface states (rhoL, uL, pL, rhoR, uR, pR), uniform over the forest."""
        out = np.zeros((n, 6), np.float64)
        self._check("fc2d_b200_sample_interfaces", self.lib.fc2d_b200_sample_interfaces(self.h, n, seed, _dp(out)))
        return out

    def set_pstar_seed(self, mlp) -> None:
        """Start the exact solver's Newton iterations from the network (None: PVRS)."""
        self._check("fc2d_b200_set_pstar_seed",
                    self.lib.fc2d_b200_set_pstar_seed(self.h, mlp.h if mlp is not None else None))

    def newton_histogram(self, reset: bool = False) -> np.ndarray:
        """Interfaces solved in k Newton iterations (k = 0..31) by the exact Euler solver."""
        out = (ctypes.c_ulonglong * 32)()
        self._check("fc2d_b200_newton_histogram", self.lib.fc2d_b200_newton_histogram(self.h, out, int(reset)))
        return np.array(out[:], np.int64)

    # -- output ----------------------------------------------------------------
    def output_ascii(self, directory: str, iframe: int, time: float) -> None:
        """fort.tNNNN / fort.qNNNN of the current forest (clawpack 4.6 ASCII, VisClaw-readable)."""
        self._check("fc2d_b200_output_ascii",
                    self.lib.fc2d_b200_output_ascii(self.h, os.fsencode(directory), iframe, time))

    def output_vtk(self, prefix: str, iframe: int) -> str:
        """<prefix>_frame_NNNN.vtu of the current forest (VTK unstructured grid; points and
        values packed on the device).  Returns the file name."""
        self._check("fc2d_b200_output_vtk", self.lib.fc2d_b200_output_vtk(self.h, os.fsencode(prefix), iframe))
        return f"{prefix}_frame_{iframe:04d}.vtu"

    # -- patch-to-CTA variants and the autotuner -------------------------------
    def variants(self) -> list:
        """Compiled patch-to-CTA variants of this solver's shape (0 = default)."""
        n, cur = ctypes.c_int(), ctypes.c_int()
        self._check("fc2d_b200_num_variants", self.lib.fc2d_b200_num_variants(self.h, ctypes.byref(n), ctypes.byref(cur)))
        out = []
        for v in range(n.value):
            a = [ctypes.c_int() for _ in range(5)]
            self._check("fc2d_b200_variant_info", self.lib.fc2d_b200_variant_info(self.h, v, *[ctypes.byref(x) for x in a]))
            out.append(dict(threads=a[0].value, min_blocks=a[1].value, reg=a[2].value, smem=a[3].value,
                            persistent=a[4].value))
        return out

    @property
    def variant(self) -> int:
        n, cur = ctypes.c_int(), ctypes.c_int()
        self._check("fc2d_b200_num_variants", self.lib.fc2d_b200_num_variants(self.h, ctypes.byref(n), ctypes.byref(cur)))
        return cur.value

    def set_variant(self, v: int) -> None:
        self._check("fc2d_b200_set_variant", self.lib.fc2d_b200_set_variant(self.h, v))

    def level_variants(self) -> np.ndarray:
        """The variant each level 0..32 uses (per-level choice of the autotuner)."""
        out = np.zeros(33, np.int32)
        self._check("fc2d_b200_level_variants", self.lib.fc2d_b200_level_variants(self.h, _ip(out)))
        return out

    def set_level_variants(self, variants) -> None:
        """Each level's variant (33 entries), e.g. another solver's level_variants()."""
        v = np.ascontiguousarray(variants, dtype=np.int32)
        if v.shape != (33,):
            raise ValueError("33 per-level variants expected")
        self._check("fc2d_b200_set_level_variants", self.lib.fc2d_b200_set_level_variants(self.h, _ip(v)))

    def autotune(self, reps: int = 3):
        """Time every variant on the current forest (q unchanged), keep the fastest,
        then keep per level the variant fastest on that level (level_variants()).
        Returns (best variant, ms per pass over all levels for each variant)."""
        n = len(self.variants())
        ms = np.zeros(n, np.float64)
        best = ctypes.c_int()
        self._check("fc2d_b200_autotune", self.lib.fc2d_b200_autotune(self.h, reps, ctypes.byref(best), _dp(ms)))
        return best.value, ms

    # -- batches of independent forests ---------------------------------------
    def set_instances(self, instances) -> None:
        """Hold len(instances) independent forests; each is a dict with minlevel, maxlevel,
        ax, bx, ay, by, mi, mj and pdata (up to 32 app parameters).  Before initialize()."""
        n = len(instances)
        arr = (_Instance * n)()
        for i, d in enumerate(instances):
            for k in ("minlevel", "maxlevel", "ax", "bx", "ay", "by", "mi", "mj"):
                setattr(arr[i], k, d.get(k, getattr(self.opts, k)))
            pd = d.get("pdata", self.opts.pdata)
            for k, v in enumerate(pd):
                arr[i].pdata[k] = v
        self._check("fc2d_b200_set_instances", self.lib.fc2d_b200_set_instances(self.h, n, arr))
        self.ninst = n

    def patch_instance(self) -> np.ndarray:
        out = np.zeros(self.num_patches, np.int32)
        self._check("fc2d_b200_patch_instance", self.lib.fc2d_b200_patch_instance(self.h, _ip(out)))
        return out

    def advance_instances(self, dt) -> np.ndarray:
        """One coarse step of every instance with its own dt; returns the CFL of each."""
        dt = np.ascontiguousarray(dt, np.float64)
        cfl = np.zeros(self.ninst, np.float64)
        self._check("fc2d_b200_advance_instances", self.lib.fc2d_b200_advance_instances(self.h, _dp(dt), _dp(cfl)))
        return cfl

    def advance_instances_begin(self, dt) -> None:
        """Launch one coarse step of every instance; returns without waiting."""
        self._dt_keep = np.ascontiguousarray(dt, np.float64)
        self._check("fc2d_b200_advance_instances_begin",
                    self.lib.fc2d_b200_advance_instances_begin(self.h, _dp(self._dt_keep)))

    def advance_instances_end(self) -> np.ndarray:
        """Wait for the step launched by advance_instances_begin; the CFL of each instance."""
        cfl = np.zeros(self.ninst, np.float64)
        self._check("fc2d_b200_advance_instances_end", self.lib.fc2d_b200_advance_instances_end(self.h, _dp(cfl)))
        return cfl

    def mass_instances(self) -> np.ndarray:
        out = np.zeros((self.ninst, self.opts.meqn), np.float64)
        self._check("fc2d_b200_mass_instances", self.lib.fc2d_b200_mass_instances(self.h, _dp(out)))
        return out

    def mass_noalloc(self) -> np.ndarray:
        """mass() through the allocation-free entry point (static device scratch)."""
        out = np.zeros(self.opts.meqn, np.float64)
        self._check("fc2d_b200_mass_noalloc", self.lib.fc2d_b200_mass_noalloc(self.h, _dp(out)))
        return out

    @property
    def cell_updates(self) -> float:
        v = ctypes.c_double()
        self._check("fc2d_b200_cell_updates", self.lib.fc2d_b200_cell_updates(self.h, ctypes.byref(v)))
        return v.value

    def synchronize(self) -> None:
        self._check("fc2d_b200_synchronize", self.lib.fc2d_b200_synchronize(self.h))

    def set_graphs(self, on: bool) -> None:
        self._check("fc2d_b200_set_graphs", self.lib.fc2d_b200_set_graphs(self.h, int(on)))

    def set_programmatic_launch(self, on: bool) -> None:
        """Programmatic dependent launch of the advance's kernels (default on)."""
        self._check("fc2d_b200_set_programmatic_launch", self.lib.fc2d_b200_set_programmatic_launch(self.h, int(on)))

    def set_timing(self, on: bool) -> None:
        self._check("fc2d_b200_set_timing", self.lib.fc2d_b200_set_timing(self.h, int(on)))

    def event_record(self, slot: int) -> None:
        self._check("fc2d_b200_event_record", self.lib.fc2d_b200_event_record(self.h, slot))

    def event_elapsed(self, a: int, b: int) -> float:
        ms = ctypes.c_double()
        self._check("fc2d_b200_event_elapsed", self.lib.fc2d_b200_event_elapsed(self.h, a, b, ctypes.byref(ms)))
        return ms.value

    def stream_handle(self) -> int:
        p = ctypes.c_void_p()
        self._check("fc2d_b200_get_stream", self.lib.fc2d_b200_get_stream(self.h, ctypes.byref(p)))
        return p.value or 0

    def set_q_ptr(self, ptr: int) -> None:
        """set_q from a raw host pointer (e.g. pinned memory)."""
        self._check("fc2d_b200_set_q", self.lib.fc2d_b200_set_q(self.h, ctypes.cast(ptr, ctypes.POINTER(ctypes.c_double))))

    def get_q_ptr(self, ptr: int) -> None:
        self._check("fc2d_b200_get_q", self.lib.fc2d_b200_get_q(self.h, ctypes.cast(ptr, ctypes.POINTER(ctypes.c_double))))

    def last_regrid_stats(self) -> dict:
        """Wall-clock milliseconds of the last regrid by phase (fc2d_b200_last_regrid_stats)."""
        ms = np.zeros(8, np.float64)
        self._check("fc2d_b200_last_regrid_stats", self.lib.fc2d_b200_last_regrid_stats(self.h, _dp(ms)))
        keys = ("tag", "adapt", "forest", "repopulate", "tables", "upload", "ghost_update", "total")
        return dict(zip(keys, ms.tolist()))

    def last_update_stats(self) -> dict:
        ms, by = ctypes.c_double(), ctypes.c_double()
        ul, tl = ctypes.c_int(), ctypes.c_int()
        self._check("fc2d_b200_last_update_stats",
                    self.lib.fc2d_b200_last_update_stats(self.h, ctypes.byref(ms), ctypes.byref(by),
                                                         ctypes.byref(ul), ctypes.byref(tl)))
        return {"update_ms": ms.value, "update_bytes": by.value, "update_launches": ul.value,
                "total_launches": tl.value}

    def graph_stats(self) -> dict:
        """Advance graphs so far: instantiations and in-place updates (fc2d_b200_graph_stats)."""
        b, u = ctypes.c_int(), ctypes.c_int()
        self._check("fc2d_b200_graph_stats", self.lib.fc2d_b200_graph_stats(self.h, ctypes.byref(b), ctypes.byref(u)))
        return {"builds": b.value, "updates": u.value}

    def last_step_timing(self) -> dict:
        """The most recent advance: host schedule time and the device span of its work (ms)."""
        h, d = ctypes.c_double(), ctypes.c_double()
        self._check("fc2d_b200_last_step_timing",
                    self.lib.fc2d_b200_last_step_timing(self.h, ctypes.byref(h), ctypes.byref(d)))
        return {"host_ms": h.value, "device_ms": d.value}
