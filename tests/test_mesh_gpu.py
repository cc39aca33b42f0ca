"""Mesh bodies on the device (b200lbm.MeshSolid, lbm_voxelize_mesh,
lbm_retag_cells_mesh): the device voxeliser decides every cell as the host
restatement of the same ray-parity test does (MeshSolid.contains) and gives
the same float surface velocities (MeshSolid.surfaceVelocity), for boxes with
faces through cell centres, a rotated box, a sphere and a torus; a moving
mesh body steps bit for bit alike whether its cells come from the device
voxeliser or from the host's per-cell calls (the reference's generic route)."""
import ctypes as C

import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import b200lbm
    return b200lbm


def _host(solid, n):
    """mask and float32 velocities from the solid's own calls, over the
    mesh's bounding box grown by one cell (every other cell is outside)."""
    nx, ny, nz = n
    mask = np.zeros(nx * ny * nz, dtype=np.uint8)
    us = np.zeros(3 * nx * ny * nz, dtype=np.float32)
    w = solid.world_triangles().reshape(-1, 3)
    lo = np.maximum(np.floor(w.min(axis=0)) - 1, 0).astype(int)
    hi = np.minimum(np.ceil(w.max(axis=0)) + 1, np.array(n) - 1).astype(int)
    tmp = [0.0, 0.0, 0.0]
    for z in range(lo[2], hi[2] + 1):
        for y in range(lo[1], hi[1] + 1):
            for x in range(lo[0], hi[0] + 1):
                if solid.contains(x, y, z):
                    i = (z * ny + y) * nx + x
                    mask[i] = 1
                    solid.surfaceVelocity(x, y, z, tmp)
                    us[3 * i:3 * i + 3] = tmp
    return mask, us


def _device(gpu, sim, solid):
    from b200lbm import _capi
    tri = np.ascontiguousarray(solid.world_triangles())
    mask = np.zeros(sim.n, dtype=np.uint8)
    us = np.zeros(3 * sim.n, dtype=np.float32)
    m = solid.motion()
    _capi.check(sim.handle, _capi.lib().lbm_voxelize_mesh(sim.handle, tri.ctypes.data_as(C.c_void_p), len(tri),
                                                          C.byref(m), mask.ctypes.data_as(C.c_void_p),
                                                          us.ctypes.data_as(C.c_void_p)))
    return mask, us


def _solids():
    from b200lbm.mesh import MeshSolid, box_mesh, icosphere, torus
    out = []
    for lo, hi in (((4.0, 5.0, 3.0), (15.0, 12.0, 10.0)), ((4.5, 5.5, 3.5), (14.5, 12.5, 9.5))):
        v, t = box_mesh(lo, hi)
        out.append(MeshSolid(v, t, center=np.mean([lo, hi], axis=0), velocity=(0.01, -0.02, 0.005),
                             angular_velocity=(0.0, 0.003, -0.002)))
    v, t = box_mesh((6.0, 6.0, 6.0), (16.0, 13.0, 11.0))
    rot = MeshSolid(v, t, center=(11.0, 9.5, 8.5), angular_velocity=(0.05, 0.08, -0.03))
    for _ in range(5):
        rot.step(1.0)  # turned about an oblique axis
    out.append(rot)
    v, t = icosphere((10.3, 11.1, 9.7), 6.2, subdivisions=3)
    out.append(MeshSolid(v, t, center=(10.3, 11.1, 9.7), velocity=(0.0, -0.01, 0.0)))
    v, t = torus((11.0, 10.0, 10.0), 6.0, 2.2, nu=28, nv=14)
    out.append(MeshSolid(v, t, center=(11.0, 10.0, 10.0), angular_velocity=(0.0, 0.0, 0.01)))
    return out


def test_voxeliser_equals_host_test(gpu):
    n = (24, 22, 21)
    sim = gpu.Sim(*n)
    for k, solid in enumerate(_solids()):
        hm, hu = _host(solid, n)
        dm, du = _device(gpu, sim, solid)
        assert hm.sum() > 50, k
        assert np.array_equal(dm, hm), (k, int(np.count_nonzero(dm != hm)))
        assert np.array_equal(du, hu), k
    sim.close()


def test_mesh_body_device_equals_host_route(gpu):
    from b200lbm.mesh import MeshSolid, box_mesh
    runs = []
    for use_device in (True, False):
        sim = gpu.Sim(26, 24, 22)
        scenes._params(sim, 0.8, 0.7, 0.008, 0.0015)
        sim.initFlat(9.5)
        v, t = box_mesh((8.2, 10.1, 7.3), (15.7, 15.4, 13.9))
        body = MeshSolid(v, t, center=(11.95, 12.75, 10.6), velocity=(0.04, -0.06, 0.02),
                         angular_velocity=(0.0, 0.01, 0.02))
        body.use_device = use_device
        forces = []
        for _ in range(14):
            sim.step(body)
            body.absorbDeadCells(sim)
            forces.append((body.Fx, body.Fy, body.Fz, body.Tx, body.Ty, body.Tz))
            body.step(1.0)
        runs.append(({k: np.array(getattr(sim, k)) for k in ("phi", "rho", "ux", "f", "h", "tag")}, forces))
        sim.close()
    (fa, Fa), (fb, Fb) = runs
    for k in fa:
        assert np.array_equal(fa[k], fb[k]), k
    assert Fa == Fb
    assert any(abs(f[1]) > 0 for f in Fa)
