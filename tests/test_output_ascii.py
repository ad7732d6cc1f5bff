"""clawpack 4.6 ASCII frames (fort.tNNNN / fort.qNNNN) in the reference's format
(fort_4.6/fclaw2d_clawpatch46_output_ascii.f): I5 integers, E30.20 time, E24.16
patch geometry, E26.16 values (|q| < 1e-99 written as zero, E dropped for
three-digit exponents), a blank line after every row of cells."""
import numpy as np
import pytest


def _frame(tmp_path):
    import forestclaw_b200 as fb
    mbc, mx, my = 2, 2, 1
    q = np.zeros((2, 2, my + 2 * mbc, mx + 2 * mbc))
    # patch 0: cells (1,1), (2,1) of fields 1, 2 (index [p, m, j + mbc - 1, i + mbc - 1])
    q[0, 0, 2, 2], q[0, 1, 2, 2] = 1.0, -2.5e-3
    q[0, 0, 2, 3], q[0, 1, 2, 3] = 1e-120, 1.5e150
    q[1, :, 2, 2:4] = 0.125
    fb.write_ascii_frame(str(tmp_path), 7, 0.5, q, level=[3, 4], block=[0, 1], xlower=[0.25, 0.5],
                         ylower=[0.0, 0.75], dx=[0.125, 0.0625], dy=[0.125, 0.0625], mbc=mbc, maux=1)
    return (tmp_path / "fort.t0007").read_text().splitlines(), (tmp_path / "fort.q0007").read_text().splitlines()


def test_time_header(tmp_path):
    t, _ = _frame(tmp_path)
    assert t == ["    0.50000000000000000000E+00    time",
                 "    2                 meqn",
                 "    2                 ngrids",
                 "    1                 num_aux",
                 "    2                 num_dim"]


def test_patch_blocks(tmp_path):
    _, q = _frame(tmp_path)
    assert q[:11] == ["    0                 grid_number",
                      "    3                 AMR_level",
                      "    0                 block_number",
                      "    0                 mpi_rank",
                      "    2                 mx",
                      "    1                 my",
                      "  0.2500000000000000E+00    xlow",
                      "  0.0000000000000000E+00    ylow",
                      "  0.1250000000000000E+00    dx",
                      "  0.1250000000000000E+00    dy",
                      ""]
    assert q[11] == "    0.1000000000000000E+01   -0.2500000000000000E-02"
    assert q[12] == "    0.0000000000000000E+00    0.1500000000000000+151"
    assert q[13] == "  "
    assert q[14] == "    1                 grid_number"
    assert q[15] == "    4                 AMR_level"
    assert q[25] == "    0.1250000000000000E+00    0.1250000000000000E+00"


def test_values_round_trip(tmp_path):
    import forestclaw_b200 as fb
    rng = np.random.default_rng(1)
    q = rng.standard_normal((3, 1, 12, 12))
    fb.write_ascii_frame(str(tmp_path), 0, 1.0, q, level=[1, 1, 2], block=[0, 0, 0], xlower=[0, 0.5, 0],
                         ylower=[0, 0, 0.5], dx=[1 / 16] * 3, dy=[1 / 16] * 3)
    lines = (tmp_path / "fort.q0000").read_text().splitlines()
    vals = [float(x.replace("D", "E")) for x in lines if x.strip() and "grid_number" not in x and
            not any(k in x for k in ("AMR_level", "block_number", "mpi_rank", "mx", "my", "xlow", "ylow", "dx", "dy"))]
    ref = q[:, 0, 2:-2, 2:-2].reshape(-1)       # rows j, then i within a row
    np.testing.assert_allclose(vals, ref, rtol=1e-15)
