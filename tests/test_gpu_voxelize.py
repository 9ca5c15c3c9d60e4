"""Solid voxelisation (rso_voxelize) through the C ABI against the numpy
restatement of the reference's voxeliser (oracle/voxel.py): bit-exact voxel
masks on a cube like the reference's sample mesh, a rotated icosphere and a
torus, the padded power-of-two grid of voxelize_mesh, and the volume of a
sphere within a few percent of 4/3 pi r^3."""
import numpy as np
import pytest

import mesh_shapes as M

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,pref", [("cube", 16), ("icosphere", 24), ("torus", 40), ("icosphere", 63)])
def test_voxelize_matches_restatement(cuda, shape, pref):
    from oracle import voxel
    from robustoptspline3d_b200.voxelize import voxelize
    v, f = {"cube": M.cube, "icosphere": lambda: M.icosphere(3, 5.0, rotation_seed=4), "torus": M.torus}[shape]()
    sg, Rg, bg = voxelize(v, f, pref)
    so, Ro, bo = voxel.voxelize(v, f, pref)
    assert Rg == Ro and Rg > pref and Rg & (Rg - 1) == 0
    assert np.array_equal(bg, bo)
    assert np.array_equal(sg, so), int(np.sum(sg != so))
    if shape == "cube":
        # the mesh spans `pref` voxels on every axis, centred in the padded cube
        idx = np.argwhere(sg)
        assert sg.sum() == pref ** 3 and idx.min() == (Rg - pref) // 2 and idx.max() == (Rg + pref) // 2 - 1


def test_voxelize_sphere_volume(cuda):
    from robustoptspline3d_b200.voxelize import voxelize
    v, f = M.icosphere(4, 1.0, rotation_seed=7)
    s, R, box = voxelize(v, f, 48)
    r = 48 / 2  # the sphere spans 48 voxels
    assert abs(s.sum() / (4 / 3 * np.pi * r ** 3) - 1) < 0.03
