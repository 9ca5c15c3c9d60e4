"""Host-side checks of the boundary-condition inputs: the text format of
static_range::rangeUnion::parse (boundary/BoundaryCondition.h:259-334) with
its quirks, the JSON schema, the plane through three points, the C ABI's
argument checks (no device work), and self-checks of the numpy restatement
in oracle/boundary.py against independent formulations."""
import ctypes

import numpy as np

import mesh_shapes as M


def test_parse_ranges_kinds_and_flags():
    from robustoptspline3d_b200 import boundary as B
    text = "box\n0 0 0 1 2 3\nclosed\nsphere\n1 1 1 0.5\nopen\nhalfspace\n0 0 1 -2\nhalfspace\n0 0 0 1 0 0 0 1 0\n" \
           "box\n2 2 2 4 6 8 2\n"
    r = B.parse_ranges(text)
    assert [x.kind for x in r] == [B.BOX, B.SPHERE, B.HALFSPACE, B.HALFSPACE, B.BOX]
    assert r[0].p == [0, 0, 0, 1, 2, 3] and not r[0].closed
    assert r[1].p == [1, 1, 1, 0.5] and r[1].closed
    assert r[2].p == [0, 0, 1, -2] and not r[2].closed
    assert r[3].p == [0.0, 0.0, 1.0, -0.0]  # plane z = 0, positive side +z
    assert r[4].p == [1, 1, 1, 2, 3, 4]  # homogeneous corners divided by hw


def test_parse_ranges_quirks():
    from robustoptspline3d_b200 import boundary as B
    # the collected numbers are kept after a region: a second line of six adds nothing
    assert len(B.parse_ranges("box\n0 0 0 1 1 1\n0 0 0 2 2 2\n")) == 1
    # numbers may span lines; an empty line after a complete region adds it again
    assert len(B.parse_ranges("box\n0 0 0\n1 1 1\n")) == 1
    assert len(B.parse_ranges("box\n0 0 0 1 1 1\n\nsphere\n0 0 0 1")) == 3
    # diagonal corners in any order give the same canonical box
    assert B.parse_ranges("box\n1 1 1 0 0 0")[0].p == [0, 0, 0, 1, 1, 1]
    # "complement" is parsed but the region stays uncomplemented; closed persists
    r = B.parse_ranges("closed\ncomplement\nsphere\n0 0 0 1\n")
    assert len(r) == 1 and not r[0].complement and r[0].closed
    # extraction stops at the first token that is not a number
    assert len(B.parse_ranges("sphere\n0 0 0 x 1\n")) == 0
    assert B.parse_ranges("sphere\n0 0 0 2.5e-1junk 7\n")[0].p == [0, 0, 0, 0.25]
    # a line longer than 511 characters ends the input
    assert len(B.parse_ranges("sphere\n" + " " * 600 + "\n0 0 0 1\n")) == 0


def test_bc_json_schema():
    from robustoptspline3d_b200 import boundary as B
    doc = {
        "fix": [{"type": "halfspace", "plane": [0, 0, -1, 0.5], "closed": True},
                {"type": "text", "text": "sphere\n0 0 0 2\n"}],
        "load": [{"type": "box", "min": [1, 1, 1], "max": [0, 0, 0], "complement": True},
                 {"type": "cylinder", "bottom": [0, 0, 0], "radius": 1, "axis": [0, 0, 2]}],
        "force": [{"region": {"type": "box", "min": [0, 0, 0], "max": [1, 1, 1]}, "norm": ["constant", 2.0],
                   "direction": ["constant", [0, 0, -3]]}],
    }
    import json
    for src in (doc, json.dumps(doc)):
        d = B.load_bc_json(src)
        assert [r.kind for r in d["fix"]] == [B.HALFSPACE, B.SPHERE] and d["fix"][0].closed
        assert d["load"][0].p == [0, 0, 0, 1, 1, 1] and d["load"][0].complement
        f = d["force"][0].c()
        assert f.norm_kind == B.CONSTANT and f.norm_p[0] == 2.0 and list(f.dir_p[:3]) == [0, 0, -3]


def test_plane_through_points_orientation():
    from robustoptspline3d_b200.boundary import plane_through
    a, b, c, d = plane_through((0, 0, 1), (1, 0, 1), (0, 1, 1))  # counterclockwise seen from +z
    assert (a, b, c) == (0.0, 0.0, 1.0) and d == -1.0


def test_entry_points_reject_bad_arguments_without_gpu():
    from robustoptspline3d_b200 import load_library
    from robustoptspline3d_b200.rso import _Field, _Region
    lib = load_library()
    r = (_Region * 1)()
    r[0].kind = 9
    o = np.zeros(3)
    m = np.zeros(8, np.uint8)
    pd, pu8 = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_uint8)
    assert lib.rso_region_mask(r, 1, o.ctypes.data_as(pd), 1.0, 2, 2, 2, m.ctypes.data_as(pu8)) == 1
    assert lib.rso_region_mask(r, 0, o.ctypes.data_as(pd), 1.0, 0, 2, 2, m.ctypes.data_as(pu8)) == 1
    f = (_Field * 1)()
    f[0].norm_kind = 5
    assert lib.rso_region_field(f, 1, o.ctypes.data_as(pd), 1, o.ctypes.data_as(pd)) == 1
    v, fc = M.cube(1.0)
    v = np.ascontiguousarray(v, np.float32)
    bad = np.ascontiguousarray(fc, np.int32).copy()
    bad[0, 0] = len(v)
    box = np.array([-2, -2, -2, 2, 2, 2], np.float32)
    s = np.zeros(8, np.uint8)
    fp, ip = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int)
    assert lib.rso_shell_elements(v.ctypes.data_as(fp), len(v), bad.ctypes.data_as(ip), len(bad),
                                  box.ctypes.data_as(fp), 2, 1.0, s.ctypes.data_as(pu8), s.ctypes.data_as(pu8)) == 1
    assert lib.rso_mesh_normals(v.ctypes.data_as(fp), len(v), bad.ctypes.data_as(ip), len(bad), o.ctypes.data_as(pd),
                                1, o.ctypes.data_as(pd)) == 1


def test_oracle_closest_point_against_sampling():
    from oracle import boundary as OB
    rng = np.random.default_rng(5)
    for _ in range(20):
        a, b, c = rng.normal(size=(3, 3))
        P = rng.normal(size=(200, 3)) * 2
        q = OB.closest_on_triangle(P, a, b, c)
        # q lies on the triangle: barycentric weights of a dense sample bound the distance from above
        u, v = np.meshgrid(np.linspace(0, 1, 81), np.linspace(0, 1, 81))
        keep = u + v <= 1
        S = a + u[keep, None] * (b - a) + v[keep, None] * (c - a)
        dmin = np.min(np.linalg.norm(P[:, None, :] - S[None], axis=2), axis=1)
        dq = np.linalg.norm(P - q, axis=1)
        assert np.all(dq <= dmin + 1e-12)
        assert np.all(dq >= dmin - 0.03 * np.linalg.norm(b - a + c - a))  # the sample is within a grid step
        # and q is on the triangle's plane
        n = np.cross(b - a, c - a)
        assert np.max(np.abs((q - a) @ n)) < 1e-9 * np.linalg.norm(n) * (1 + np.abs(P).max())


def test_oracle_shell_is_the_global_distance_rule():
    """Face-by-face union over index boxes = elements in some face's index box
    whose distance to the whole mesh is below the width (the reference's rule)."""
    from oracle import boundary as OB
    from oracle import voxel
    v, f = M.torus(2.0, 0.7, 24, 12)
    solid, R, bx = voxel.voxelize(v, f, 20)
    w_units = 2.0
    sh = OB.shell_elements(v, f, bx, R, w_units, solid)
    b = np.asarray(bx, np.float32)
    eh = float(np.float32(np.float32(b[3] - b[0]) / np.float32(R)))
    w = w_units * eh
    V = np.asarray(v, np.float32).astype(np.float64)
    inbox = np.zeros(R ** 3, bool)
    for fc in np.asarray(f):
        lo, hi = V[fc].min(0), V[fc].max(0)
        lid = [min(max(int((lo[j] - w * 1.3 - b[j] - 0.5 * eh) / eh), 0), R - 1) for j in range(3)]
        rid = [min(max(int((hi[j] + w * 1.3 - b[j] - 0.5 * eh) / eh + 1), 0), R - 1) for j in range(3)]
        m = np.zeros((R, R, R), bool)
        m[lid[2]:rid[2], lid[1]:rid[1], lid[0]:rid[0]] = True
        inbox |= m.reshape(-1)
    idx = np.flatnonzero(solid.reshape(-1) & inbox)
    x, y, z = idx % R, (idx // R) % R, idx // R ** 2
    P = np.stack([(x + 0.5) * eh + b[0], (y + 0.5) * eh + b[1], (z + 0.5) * eh + b[2]], axis=1)
    d2 = np.full(len(P), np.inf)
    for fc in np.asarray(f):
        d = P - OB.closest_on_triangle(P, V[fc[0]], V[fc[1]], V[fc[2]])
        d2 = np.minimum(d2, OB._dot(d, d))
    ref = np.zeros(R ** 3, np.uint8)
    ref[idx[d2 < w * w]] = 1
    assert np.array_equal(sh.reshape(-1), ref) and 0 < ref.sum() < solid.sum()


def test_oracle_normals_on_a_sphere():
    from oracle import boundary as OB
    v, f = M.icosphere(3, 1.0)
    rng = np.random.default_rng(3)
    d = rng.normal(size=(100, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    for s in (0.9, 1.1):  # inside and outside: the normal points out either way
        n = OB.mesh_normals(v, f, d * s)
        assert np.allclose(np.linalg.norm(n, axis=1), 1.0)
        assert np.min(np.sum(n * d, axis=1)) > 0.95


def test_surface_nodes_against_direct_rule():
    """surface_nodes: a node touching a solid element is a surface node unless
    every axis has a solid element pair across it (the library's node class)."""
    from robustoptspline3d_b200.boundary import surface_nodes
    rng = np.random.default_rng(8)
    em = (rng.uniform(size=(5, 6, 7)) < 0.6).astype(np.uint8)
    got = surface_nodes(em)
    ez, ey, ex = em.shape
    want = np.zeros((ez + 1, ey + 1, ex + 1), bool)
    pad = np.pad(em.astype(bool), 1)
    for z in range(ez + 1):
        for y in range(ey + 1):
            for x in range(ex + 1):
                s = {(dx, dy, dz): pad[z + dz, y + dy, x + dx] for dx in (0, 1) for dy in (0, 1) for dz in (0, 1)}
                if not any(s.values()):
                    continue
                ax0 = any(s[0, a, b] and s[1, a, b] for a in (0, 1) for b in (0, 1))
                ax1 = any(s[a, 0, b] and s[a, 1, b] for a in (0, 1) for b in (0, 1))
                ax2 = any(s[a, b, 0] and s[a, b, 1] for a in (0, 1) for b in (0, 1))
                want[z, y, x] = not (ax0 and ax1 and ax2)
    assert np.array_equal(got, want)


def test_node_grid_uses_fp32_quotient():
    from robustoptspline3d_b200.boundary import node_grid
    box = np.array([-1.1, -2.2, 0.3, 2.9, 1.8, 4.3], np.float32)
    origin, h = node_grid(box, 7)
    assert h == float(np.float32(np.float32(box[3] - box[0]) / np.float32(7)))
    assert np.array_equal(origin, box[:3].astype(np.float64))


def test_bench_torus_mesh_is_closed_and_outward():
    import bench
    v, f = bench.torus_mesh(nu=24, nv=12)
    assert v.shape == (24 * 12, 3) and f.shape == (2 * 24 * 12, 3)
    # every directed edge appears once and its reverse once: closed and consistently wound
    edges = {}
    for a, b, c in f:
        for e in ((a, b), (b, c), (c, a)):
            edges[e] = edges.get(e, 0) + 1
    assert all(n == 1 for n in edges.values()) and all((b, a) in edges for a, b in edges)
    # outward: the signed volume (divergence theorem) is positive
    A, B, C = v[f[:, 0]].astype(np.float64), v[f[:, 1]].astype(np.float64), v[f[:, 2]].astype(np.float64)
    vol = np.einsum("ij,ij->i", A, np.cross(B, C)).sum() / 6
    # an inscribed polygonal torus of 24 x 12 segments holds about 94 % of the smooth volume
    assert vol > 0 and 0.9 < vol / (2 * np.pi ** 2 * 2.0 * 0.7 ** 2) < 1.0
