"""The single-step binding of INTEGRATION.md section 1, from C: tests/c_shim/shim_protocol.c
is compiled against include/fc2d_b200.h (no Python in between) and hands host patch
arrays over through fc2d_b200_single_step_update_host, checking the results bit for
bit against a solver whose data stays on the device."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_c_shim_protocol(tmp_path):
    import forestclaw_b200 as fb
    fb.load_library()                                    # built in-tree
    libdir = os.path.join(ROOT, "forestclaw_b200")
    exe = str(tmp_path / "shim_protocol")
    subprocess.run(["gcc", "-std=c11", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_shim", "shim_protocol.c"), "-o", exe, "-L", libdir,
                    "-lfc2d_b200", "-Wl,-rpath," + libdir], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "shim protocol ok" in r.stdout
