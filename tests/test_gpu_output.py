"""fc2d_b200_output_ascii on a device forest: every patch written once, in the
reference's order (block, then along the curve), with its absolute level and the
interior values of q."""
import numpy as np
import pytest

from tests.cases import DAM, make

pytestmark = pytest.mark.gpu


def _parse(path):
    lines = path.read_text().splitlines()
    patches, k = [], 0
    while k < len(lines):
        if "grid_number" not in lines[k]:
            k += 1
            continue
        head = [int(lines[k + i].split()[0]) for i in range(6)]
        geo = [float(lines[k + 6 + i].split()[0]) for i in range(4)]
        mx, my = head[4], head[5]
        k += 11
        rows = []
        while len(rows) < mx * my:
            if lines[k].strip():
                rows.append([float(v) for v in lines[k].split()])
            k += 1
        patches.append((head, geo, np.array(rows)))
    return patches


def test_output_ascii_frame(tmp_path):
    import forestclaw_b200 as fb
    _, gc = make(DAM, mx=8, my=8, minlevel=2, maxlevel=4, subcycle=1)
    g = fb.Solver(gc)
    g.initialize()
    g.advance(0.0, 0.01)
    g.output_ascii(str(tmp_path), 3, 0.01)
    t = (tmp_path / "fort.t0003").read_text().splitlines()
    assert t[1].split()[0] == "3" and int(t[2].split()[0]) == g.num_patches
    patches = _parse(tmp_path / "fort.q0003")
    assert len(patches) == g.num_patches
    q, info = g.get_q(), g.patch_info()
    by_pos = {(int(l), int(x), int(y)): p for p, (l, b, x, y) in enumerate(info)}
    seen = set()
    for num, (head, geo, rows) in enumerate(patches):
        assert head[0] == num
        level = head[1]
        ix, iy = int(round(geo[0] / geo[2] / 8 + 1e-9 + (1 << level) / 2)), int(round(geo[1] / geo[3] / 8 + (1 << level) / 2))
        p = by_pos[(level, ix, iy)]
        seen.add(p)
        ref = q[p][:, 2:-2, 2:-2].transpose(1, 2, 0).reshape(-1, 3)
        ref = np.where(np.abs(ref) < 1e-99, 0.0, ref)
        np.testing.assert_allclose(rows, ref, rtol=1e-15, atol=0)
    assert len(seen) == g.num_patches
