"""Boundary-condition inputs on the device (rso_region_mask, rso_region_field,
rso_shell_elements, rso_mesh_normals) through the C ABI against the numpy
restatement in oracle/boundary.py: region masks and shell elements bit-exact
(both sides round every operation separately), normals to 1e-12 and fields
to 1e-13 relative (exp and pow of the radial norm may differ in the last bit
between the device and numpy), and the whole mesh -> HierarchyGrid input
chain on a sphere."""
import numpy as np
import pytest

import mesh_shapes as M

pytestmark = pytest.mark.gpu


def _tuples(regions):
    return [(r.kind, r.p, r.closed, r.complement) for r in regions]


def _regions():
    from robustoptspline3d_b200 import boundary as B
    # node grid origin (-1, -0.5, 0.25), h = 0.125: many nodes lie exactly on the boundaries
    return [
        [B.box((0, 0, 0.5), (0.5, 0.75, 1.0), closed=True)],
        [B.box((0, 0, 0.5), (0.5, 0.75, 1.0))],
        [B.box((0, 0, 0.5), (0.5, 0.75, 1.0), closed=True, complement=True)],
        [B.sphere((0.0, 0.25, 0.75), 0.5, closed=True), B.sphere((-0.5, 0.0, 1.0), 0.25)],
        [B.sphere((0.0, 0.25, 0.75), 0.5, complement=True)],
        [B.halfspace(0, 0, 1, -0.75, closed=True)],
        [B.halfspace(0, 0, 1, -0.75)],
        [B.halfspace_points((0, 0, 0.5), (1, 0, 0.75), (0, 1, 0.5), closed=True)],
        [B.halfspace(1, -2, 0.5, 0.1, complement=True), B.box((-2, -2, -2), (2, 2, 0.6))],
        [B.cylinder((0, 0, 0.25), 0.375, (0, 0, 1.0))],
        [B.cylinder((-0.5, -0.25, 0.5), 0.3, (1.0, 0.5, 0.25))],
        [],
    ]


@pytest.mark.parametrize("case", range(12))
def test_region_mask_matches_restatement(cuda, case):
    from oracle import boundary as OB
    from robustoptspline3d_b200 import boundary as B
    regions = _regions()[case]
    origin, h, dims = (-1.0, -0.5, 0.25), 0.125, (17, 13, 11)
    got = B.region_mask(regions, origin, h, dims)
    want = OB.region_mask(_tuples(regions), origin, h, dims)
    assert got.shape == (11, 13, 17)
    assert np.array_equal(got, want), int(np.sum(got != want))
    if case == 0:  # closed box: 5 x 7 x 5 nodes on and inside its faces
        assert got.sum() == 5 * 7 * 5
    if case == 1:  # open box: the 3 x 5 x 3 strictly inside
        assert got.sum() == 3 * 5 * 3


def test_region_field_matches_restatement(cuda):
    from oracle import boundary as OB
    from robustoptspline3d_b200 import boundary as B
    rng = np.random.default_rng(9)
    P = rng.uniform(-1, 1, size=(4000, 3))
    P[:50] = np.round(P[:50] * 4) / 4  # some points on region boundaries
    fields = [
        B.Field(B.box((-1, -1, -1), (1, 1, 0.2), closed=True), ("constant", 2.5), ("constant", (0, 0, -3))),
        B.Field(B.sphere((0, 0, 0), 0.8), ("radial", (0.1, 0.2, 0.3), 1.5, 0.7), ("constant", (1, 1, 0))),
        B.Field(B.halfspace(0, 1, 0, 0.0), ("constant", 1.0), ("radial", (0.0, 0.5, 0.0))),
        B.Field(B.sphere((0.2, 0, 0), 0.9, complement=True), ("radial", (0, 0, 0)), ("radial", (0.3, -0.2, 0.1))),
        B.Field(B.box((-2, -2, -2), (2, 2, 2)), ("twist", (0, 0, -1), (0, 0, 1), 0.75),
                ("twist", (0, 0, -1), (0, 0, 1))),
    ]
    got = B.region_field(fields, P)
    tup = []
    for f in fields:
        c = f.c()
        tup.append((( f.region.kind, f.region.p, f.region.closed, f.region.complement), c.norm_kind,
                    list(c.norm_p), c.dir_kind, list(c.dir_p)))
    want = OB.region_field(tup, P)
    scale = np.maximum(np.abs(want), 1.0)
    assert np.max(np.abs(got - want) / scale) <= 1e-13
    assert np.count_nonzero(np.any(got != 0, axis=1)) > 3000


@pytest.mark.parametrize("shape,pref,width", [("torus", 40, 2.0), ("icosphere", 24, 1.0), ("icosphere", 24, 3.5),
                                              ("cube", 16, 3.0)])
def test_shell_elements_match_restatement(cuda, shape, pref, width):
    from oracle import boundary as OB
    from robustoptspline3d_b200 import boundary as B
    from robustoptspline3d_b200.voxelize import voxelize
    v, f = {"cube": M.cube, "icosphere": lambda: M.icosphere(3, 5.0, rotation_seed=4), "torus": M.torus}[shape]()
    solid, R, bx = voxelize(v, f, pref)
    got = B.shell_elements(v, f, bx, R, width, solid)
    want = OB.shell_elements(v, f, bx, R, width, solid)
    assert np.array_equal(got, want), int(np.sum(got != want))
    assert 0 < got.sum() < solid.sum() and not np.any(got & ~solid)
    if shape == "cube":
        # the cube spans pref voxels: elements within `width` voxels of a face, centres at half voxels
        k = int(np.ceil(width - 0.5))
        inner = (pref - 2 * k) ** 3
        assert got.sum() == pref ** 3 - inner


def test_mesh_normals_match_restatement(cuda):
    from oracle import boundary as OB
    from robustoptspline3d_b200 import boundary as B
    v, f = M.torus()
    rng = np.random.default_rng(4)
    P = rng.uniform(-3, 3, size=(3000, 3)) * np.array([1, 1, 0.4])
    P[:5] = np.asarray(v, np.float32)[:5]  # points on the mesh take the face normal
    got = B.mesh_normals(v, f, P)
    want = OB.mesh_normals(v, f, P)
    assert np.max(np.abs(got - want)) <= 1e-12
    assert np.allclose(np.linalg.norm(got, axis=1), 1.0)


def test_mesh_problem_chain(cuda):
    """icosphere -> voxels -> fixed (bottom cap) / load (top cap) / normals / shell -> HierarchyGrid."""
    from robustoptspline3d_b200 import Config, HierarchyGrid
    from robustoptspline3d_b200 import boundary as B
    v, f = M.icosphere(3, 5.0)
    fix = [B.halfspace(0, 0, -1, -3.5, closed=True)]   # z <= -3.5
    load = [B.halfspace(0, 0, 1, -3.5)]                # z > 3.5
    force = [B.Field(B.halfspace(0, 0, 1, -3.5), ("constant", 1.0), ("constant", (0, 0, -1)))]
    pr = B.mesh_problem(v, f, 24, fix, load, force, shell_width=2.0)
    R = pr["resolution"]
    surf = B.surface_nodes(pr["emask"])
    lmask = surf & (pr["load"] > 0) & (pr["fixed"] == 0)
    assert lmask.sum() > 20 and (surf & (pr["fixed"] > 0)).sum() > 20
    n = pr["normals"][lmask.reshape(-1)]
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0) and np.min(n[:, 2]) > 0.3  # top cap points up
    fz = pr["force"][lmask.reshape(-1)]
    assert np.all(fz[:, 2] == -1.0)
    assert pr["shell"].sum() > 0 and not np.any(pr["shell"] & ~pr["emask"])
    g = HierarchyGrid(pr["emask"], pr["fixed"], pr["load"], pr["normals"], Config(poisson_ratio=0.3))
    cls = g.node_class().reshape(R + 1, R + 1, R + 1)
    assert np.array_equal((cls & 2) > 0, surf)
    assert np.array_equal((cls & 8) > 0, lmask)
    g.close()


def test_boundary_edge_cases(cuda):
    """Empty region and field lists, zero shell width, no points, a degenerate
    face, points on faces / edges / vertices, and a one-element grid."""
    from oracle import boundary as OB
    from robustoptspline3d_b200 import boundary as B
    from robustoptspline3d_b200.voxelize import voxelize
    # empty unions: no node selected, zero field
    assert B.region_mask([], (0, 0, 0), 1.0, (3, 2, 1)).sum() == 0
    assert np.all(B.region_field([], np.ones((4, 3))) == 0)
    assert B.region_field([B.Field(B.sphere((0, 0, 0), 1), ("constant", 1.0), ("constant", (0, 0, 1)))],
                          np.zeros((0, 3))).shape == (0, 3)
    # a one-node grid
    m = B.region_mask([B.box((0, 0, 0), (0, 0, 0), closed=True)], (0, 0, 0), 1.0, (1, 1, 1))
    assert m.shape == (1, 1, 1) and m[0, 0, 0] == 1
    assert B.region_mask([B.box((0, 0, 0), (0, 0, 0))], (0, 0, 0), 1.0, (1, 1, 1))[0, 0, 0] == 0
    # zero shell width: no shell element and no launch needed
    v, f = M.cube(4.0)
    solid, R, bx = voxelize(v, f, 8)
    assert B.shell_elements(v, f, bx, R, 0.0, solid).sum() == 0
    # a degenerate (zero-area) face added to the cube changes neither shell nor normals
    vd = np.concatenate([np.asarray(v, np.float32), np.array([[4, 4, 4]], np.float32)])
    fd = np.concatenate([np.asarray(f, np.int32), np.array([[len(v), len(v), len(v)]], np.int32)])
    s1 = B.shell_elements(v, f, bx, R, 1.5, solid)
    s2 = B.shell_elements(vd, fd, bx, R, 1.5, solid)
    assert np.array_equal(s1, s2) and np.array_equal(s2, OB.shell_elements(vd, fd, bx, R, 1.5, solid))
    # points on a face, on an edge and at a vertex: the face normal of the lowest-index face
    P = np.array([[0.5, 0.25, 4.0], [4.0, 4.0, 0.0], [4.0, 4.0, 4.0], [0.0, 0.0, 9.0], [1.0, 2.0, 3.0]])
    n = B.mesh_normals(vd, fd, P)
    assert np.max(np.abs(n - OB.mesh_normals(vd, fd, P))) <= 1e-12
    assert np.allclose(n[0], (0, 0, 1)) and np.allclose(n[3], (0, 0, 1))  # top face; above the top face
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0)
    assert B.mesh_normals(v, f, np.zeros((0, 3))).shape == (0, 3)
