"""MeshSolid's host restatement of the voxeliser (b200lbm.mesh), without a
GPU: the ray-parity test finds the cells of an axis-aligned box exactly --
including boxes whose faces pass through cell centres, where the top-left
rule must count a shared edge once -- and a sphere's cells agree with the
analytic test except within a cell of the surface."""
import numpy as np

from b200lbm.mesh import MeshSolid, box_mesh, icosphere, torus


def _mask(solid, n):
    return np.array([[[solid.contains(x, y, z) for x in range(n)] for y in range(n)] for z in range(n)])


def test_box_cells_exact():
    for lo, hi in (((2.0, 3.0, 1.0), (7.0, 6.0, 5.0)), ((2.5, 3.5, 1.5), (6.5, 5.5, 4.5)),
                   ((1.2, 2.7, 3.1), (6.9, 7.4, 5.05))):
        v, t = box_mesh(lo, hi)
        s = MeshSolid(v, t, center=np.mean([lo, hi], axis=0))
        got = _mask(s, 9)
        c = np.arange(9) + 0.5
        want = ((c[None, None, :] > lo[0]) & (c[None, None, :] < hi[0])
                & (c[None, :, None] > lo[1]) & (c[None, :, None] < hi[1])
                & (c[:, None, None] > lo[2]) & (c[:, None, None] < hi[2]))
        # a centre exactly on a face: the top-left rule decides; only those may differ
        on_face = np.zeros_like(want)
        for a, axis_c in enumerate((c[None, None, :], c[None, :, None], c[:, None, None])):
            on_face |= np.broadcast_to((axis_c == lo[a]) | (axis_c == hi[a]), want.shape)
        assert np.array_equal(got[~on_face], want[~on_face])


def test_sphere_and_torus_near_analytic():
    v, t = icosphere((8.0, 8.2, 7.9), 5.0, subdivisions=3)
    s = MeshSolid(v, t, center=(8.0, 8.2, 7.9))
    got = _mask(s, 16)
    c = np.arange(16) + 0.5
    d = np.sqrt((c[None, None, :] - 8.0) ** 2 + (c[None, :, None] - 8.2) ** 2 + (c[:, None, None] - 7.9) ** 2)
    assert np.all(got[d < 4.7]) and not np.any(got[d > 5.01])
    v, t = torus((8.0, 8.0, 8.0), 4.5, 1.6, nu=32, nv=16)
    s = MeshSolid(v, t, center=(8.0, 8.0, 8.0))
    got = _mask(s, 16)
    rho = np.sqrt((c[None, None, :] - 8.0) ** 2 + (c[None, :, None] - 8.0) ** 2)
    dt = np.sqrt((rho - 4.5) ** 2 + (c[:, None, None] - 8.0) ** 2)
    assert np.all(got[dt < 1.3]) and not np.any(got[dt > 1.61])


def test_rigid_motion_and_impulses():
    v, t = box_mesh((2.0, 2.0, 2.0), (4.0, 4.0, 4.0))
    s = MeshSolid(v, t, center=(3.0, 3.0, 3.0), velocity=(0.1, 0.0, 0.0), angular_velocity=(0.0, 0.0, 0.2))
    out = [0.0, 0.0, 0.0]
    s.surfaceVelocity(3, 3, 2, out)
    assert out == [0.1 + (0.0 * -0.5 - 0.2 * 0.5), 0.0 + (0.2 * 0.5 - 0.0 * -0.5), 0.0]
    s.applyImpulseAtCell(4, 3, 3, 1.0, 2.0, 0.0)
    assert (s.Fx, s.Fy, s.Tz) == (1.0, 2.0, 1.5 * 2.0 - 0.5 * 1.0)
    s.step(1.0)
    assert (s.cx, s.Fx) == (3.1, 0.0)
    w = s.world_triangles().reshape(-1, 3)
    assert np.allclose(w.mean(axis=0), (3.1, 3.0, 3.0))
