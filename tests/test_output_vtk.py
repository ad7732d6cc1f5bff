"""VTK output (fclaw2d_clawpatch_output_vtk.c): layout of the .vtu file.

CPU tests write caller-supplied patches through the C ABI and parse the file
back: the XML header's offsets, the UInt64 byte count before each appended
array, the quad connectivity over each patch's own points, offsets, types,
the cell fields and the Float32 values.  The GPU test writes a frame from the
device forest and compares it with the solver's q and patch geometry.
"""
import os

import numpy as np
import pytest


def _synthetic(npatch=3, mx=4, my=3, meqn=2, seed=0):
    rng = np.random.default_rng(seed)
    pts = rng.standard_normal((npatch, (mx + 1) * (my + 1), 3))
    vals = rng.standard_normal((npatch, my, mx, meqn)).astype(np.float32)
    block = np.array([0, 1, 1][:npatch], np.int32)
    return pts, vals, block


def test_vtk_file_layout(tmp_path):
    import forestclaw_b200 as fb
    pts, vals, block = _synthetic()
    npatch, my, mx, meqn = vals.shape
    path = str(tmp_path / "t_frame_0000.vtu")
    fb.write_vtk_file(path, pts, vals, block)
    d = fb.read_vtu(path)
    ncell = npatch * mx * my
    assert d["npoints"] == npatch * (mx + 1) * (my + 1) and d["ncells"] == ncell
    assert d["header"].startswith('<?xml version="1.0"?>\n<VTKFile type="UnstructuredGrid" version="0.1" '
                                  'byte_order="LittleEndian" header_type="UInt64" >\n')
    assert 'Name="meqn" NumberOfComponents="2"' in d["header"]
    assert np.array_equal(d["Position"], pts.reshape(-1, 3))
    conn = d["connectivity"].reshape(-1, 4)
    assert conn.dtype == np.int32 and conn.shape == (ncell, 4)
    # cell (i, j) of patch p: points l, l+1, l+mx+2, l+mx+1 with l = p (mx+1)(my+1) + i + j (mx+1)
    p, j, i = 1, 2, 3
    l = p * (mx + 1) * (my + 1) + i + j * (mx + 1)
    assert list(conn[p * mx * my + j * mx + i]) == [l, l + 1, l + mx + 2, l + mx + 1]
    assert np.array_equal(d["offsets"], 4 * np.arange(1, ncell + 1))
    assert np.all(d["types"] == 9)
    assert np.all(d["mpirank"] == 0)
    assert np.array_equal(d["blockno"], np.repeat(block, mx * my))
    assert np.array_equal(d["patchno"], np.repeat(np.arange(npatch), mx * my))
    assert np.array_equal(d["meqn"], vals.reshape(-1, meqn))
    with open(path, "rb") as f:
        assert f.read().endswith(b"\n </AppendedData>\n</VTKFile>\n")


def test_vtk_single_field_has_no_component_count(tmp_path):
    import forestclaw_b200 as fb
    pts, vals, block = _synthetic(meqn=1)
    path = str(tmp_path / "s.vtu")
    fb.write_vtk_file(path, pts, vals, block)
    d = fb.read_vtu(path)
    assert '<DataArray type="Float32" Name="meqn" format="appended"' in d["header"]
    assert np.array_equal(d["meqn"], vals.reshape(-1))


def test_vtk_rejects_bad_arguments(tmp_path):
    import forestclaw_b200 as fb
    pts, vals, block = _synthetic()
    with pytest.raises(ValueError):
        fb.write_vtk_file(str(tmp_path / "x.vtu"), pts[:, :-1], vals, block)
    with pytest.raises(fb.B200Error):
        fb.write_vtk_file(str(tmp_path / "missing_dir" / "x.vtu"), pts, vals, block)


@pytest.mark.gpu
@pytest.mark.parametrize("problem", ["dam", "sphere"])
def test_vtk_from_device_forest(tmp_path, problem):
    import forestclaw_b200 as fb
    from tests.cases import DAM, SPHERE, make
    if problem == "dam":
        _, gc = make(DAM, mx=16, my=16, minlevel=2, maxlevel=4, subcycle=1, time_sync=1)
    else:
        _, gc = make(SPHERE, mx=8, my=8, minlevel=1, maxlevel=3, subcycle=1)
    g = fb.Solver(gc)
    g.initialize()
    g.advance(0.0, 0.002)
    name = g.output_vtk(str(tmp_path / "run"), 3)
    assert os.path.basename(name) == "run_frame_0003.vtu"
    d = fb.read_vtu(name)
    q, info = g.get_q(), g.patch_info()
    np_, meqn = q.shape[0], q.shape[1]
    mx, my, mbc = gc.mx, gc.my, gc.mbc
    assert d["ncells"] == np_ * mx * my
    vals = d["meqn"].reshape(np_, my, mx, meqn) if meqn > 1 else d["meqn"].reshape(np_, my, mx, 1)
    inner = q[:, :, mbc:-mbc, mbc:-mbc].transpose(0, 2, 3, 1).astype(np.float32)
    # every patch written once: the multisets of patch values agree
    assert sorted(v.tobytes() for v in vals) == sorted(v.tobytes() for v in inner)
    pos = d["Position"].reshape(np_, my + 1, mx + 1, 3)
    blocks = d["blockno"].reshape(np_, -1)[:, 0]
    assert np.all(np.diff(blocks) >= 0)                  # block by block
    if problem == "dam":
        # patch_info columns: level, block, gx, gy; corners of the brick's patches
        lev, gx, gy = info[:, 0], info[:, 2], info[:, 3]
        w = (gc.bx - gc.ax) / (gc.mi * 2.0 ** lev)
        h = (gc.by - gc.ay) / (gc.mj * 2.0 ** lev)
        corner = {(round(gc.ax + gx[k] * w[k], 12), round(gc.ay + gy[k] * h[k], 12), round(w[k], 12)): k
                  for k in range(np_)}
        for b in range(np_):
            x0, y0 = pos[b, 0, 0, 0], pos[b, 0, 0, 1]
            k = corner[(round(x0, 12), round(y0, 12), round(pos[b, 0, -1, 0] - x0, 12))]
            assert np.array_equal(vals[b], inner[k])
            dxk = w[k] / mx
            xl = pos[b, 0, 0, 0]
            assert np.array_equal(pos[b, 0, :, 0], xl + np.arange(mx + 1) * dxk) or \
                np.allclose(pos[b, 0, :, 0], xl + np.arange(mx + 1) * dxk, rtol=0, atol=1e-15)
        assert np.all(pos[..., 2] == 0.0)
    else:
        r = np.sqrt((pos ** 2).sum(-1))
        assert np.allclose(r, 1.0, atol=1e-12)
        assert set(blocks.tolist()) == set(range(6))
    g.close()
