"""The renderer oracle (oracle/render_oracle.c) on hand-made volumes: rays
that miss the tank see the sky, an empty tank shows no water surface, a full
one does, and the default view is deterministic."""
import numpy as np


def _vol(nx, ny, nz, level):
    v = np.zeros((nz, ny, nx, 2), dtype=np.uint8)
    v[:, int(level):, :, 0] = 255  # liquid where y >= level (the reference's orientation)
    return v.reshape(-1)


def test_empty_and_full_tank(oracle_mod):
    nx = ny = nz = 24
    empty = oracle_mod.render(_vol(nx, ny, nz, ny), nx, ny, nz, None, width=96, height=72)
    half = oracle_mod.render(_vol(nx, ny, nz, ny // 2), nx, ny, nz, None, width=96, height=72)
    assert empty.shape == (72, 96, 4) and (empty[..., 3] == 255).all()
    # corners of the frame miss the tank in both: identical sky
    assert np.array_equal(empty[0, 0], half[0, 0]) and np.array_equal(empty[-1, -1], half[-1, -1])
    # water changes the middle of the frame
    assert np.abs(empty[30:42, 40:56].astype(int) - half[30:42, 40:56].astype(int)).max() > 10
    again = oracle_mod.render(_vol(nx, ny, nz, ny // 2), nx, ny, nz, None, width=96, height=72)
    assert np.array_equal(half, again)


def test_sphere_is_drawn(oracle_mod):
    nx = ny = nz = 24
    v = _vol(nx, ny, nz, ny)  # no water
    a = oracle_mod.render(v, nx, ny, nz, None, width=96, height=72)
    b = oracle_mod.render(v, nx, ny, nz, (12.0, 12.0, 12.0, 5.0), width=96, height=72)
    assert np.abs(a.astype(int) - b.astype(int)).max() > 30
