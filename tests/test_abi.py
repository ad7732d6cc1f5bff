"""The C-ABI library loads and exports every entry point include/fc2d_b200.h declares (no GPU)."""
import ctypes
import os
import subprocess

import pytest

import forestclaw_b200 as fb


def test_library_built_for_sm100a():
    assert os.path.exists(fb.LIB_PATH), "run python -m forestclaw_b200.build"
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", fb.LIB_PATH], capture_output=True, text=True)
    assert "sm_100a" in out.stdout


def test_exports_every_declared_symbol():
    lib = ctypes.CDLL(fb.LIB_PATH)
    names = fb.exported_symbols()
    assert "fc2d_b200_advance" in names and "fc2d_b200_single_step_update" in names
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/fc2d_b200.h but not exported"


def test_create_reports_errors_without_crashing():
    L = fb.load_library()
    h = ctypes.c_void_p()
    bad = fb.Options(mx=15, my=15).to_c()          # odd patch size is rejected before any CUDA call
    rc = L.fc2d_b200_create(ctypes.byref(bad), ctypes.byref(h))
    assert rc == -1
    assert b"even" in L.fc2d_b200_last_error()
    rc = L.fc2d_b200_create(None, ctypes.byref(h))
    assert rc == -1


def test_unsupported_kernel_shape_rejected():
    L = fb.load_library()
    h = ctypes.c_void_p()
    o = fb.Options(mx=12, my=12, meqn=3, mwaves=3, rp=fb.RP_SW_ROE).to_c()
    rc = L.fc2d_b200_create(ctypes.byref(o), ctypes.byref(h))
    assert rc == -1
    assert b"no compiled update kernel" in L.fc2d_b200_last_error()


def test_c_binding_compiles_against_public_header(tmp_path):
    """The C program that plays ForestClaw's single-step caller builds from the
    public header alone (plain C11, warnings are errors)."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    obj = str(tmp_path / "shim.o")
    r = subprocess.run(["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", "-c", "-I", os.path.join(root, "include"),
                        os.path.join(root, "tests", "c_shim", "shim_protocol.c"), "-o", obj],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_user_solver_modules_register_through_the_abi():
    """The application-solver examples are built and export their registration
    functions; the package exports the entry point they call."""
    from forestclaw_b200 import build
    libs = build.build_user_examples()
    assert any(p.endswith("libacoustics_user.so") for p in libs)
    for p in libs:
        m = ctypes.CDLL(p)
        name = os.path.basename(p)[3:-8]          # lib<app>_user.so -> <app>
        assert hasattr(m, name + "_register_inline")
    assert hasattr(ctypes.CDLL(fb.LIB_PATH), "fc2d_b200_set_user_variants")
