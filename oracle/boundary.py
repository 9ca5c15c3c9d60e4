"""Boundary-condition inputs restated in numpy FP64, operation by operation.

TEST INFRASTRUCTURE ONLY: the checker of rso_region_mask, rso_region_field,
rso_shell_elements and rso_mesh_normals; the product library never imports
it.  Parity unpinned: the reference ships no fixtures for these and its CGAL /
Eigen host code cannot be built here.

Follows the reference:
  range and field classes      boundary/BoundaryCondition.h:379-741
  setSolidShellElement         grid/Grid.cpp:253-322 (shell elements)
  outwardNormal                grid/Grid.cpp:2838-2854
  node positions               grid/Grid.cpp:2694-2740 (computeProjectionMatrix)
The reference asks CGAL's AABB tree for squared distances and closest points;
here the closest point of a triangle is computed by Voronoi regions (Ericson,
Real-Time Collision Detection, 5.1.5), which can differ from CGAL's in the
last bits, so an element whose distance equals the shell width to within
rounding may be classified differently from the reference.  Products and sums
are evaluated left to right, as the library's kernels do.
"""
import numpy as np

SPHERE, BOX, HALFSPACE, CYLINDER = 0, 1, 2, 3
CONSTANT, RADIAL, TWIST = 0, 1, 2


def _dot(a, b):
    return a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1] + a[..., 2] * b[..., 2]


def _cross(a, b):
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1], a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)


def _unit(v):
    n = _dot(v, v)
    ok = n > 0
    s = np.sqrt(np.where(ok, n, 1.0))
    return np.where(ok[..., None], v / s[..., None], v)


def _qdiv(n, d):
    ok = d != 0
    return np.where(ok, n / np.where(ok, d, 1.0), 0.0)


def contains(kind, p, closed, complement, P):
    """Membership of points P (n, 3) in one region (rso_region semantics)."""
    P = np.asarray(P, np.float64)
    q = [float(v) for v in p]
    x, y, z = P[:, 0], P[:, 1], P[:, 2]
    if kind == SPHERE:
        dx, dy, dz = x - q[0], y - q[1], z - q[2]
        s = dx * dx + dy * dy + dz * dz
        r2 = q[3] * q[3]
        inn = (s < r2) | (bool(closed) & ((s - r2) < 1e-8))
    elif kind == BOX:
        inner = (q[0] < x) & (x < q[3]) & (q[1] < y) & (y < q[4]) & (q[2] < z) & (z < q[5])
        cl = (q[0] <= x) & (x <= q[3]) & (q[1] <= y) & (y <= q[4]) & (q[2] <= z) & (z <= q[5])
        inn = inner | (bool(closed) & cl)
    elif kind == HALFSPACE:
        s = q[0] * x + q[1] * y + q[2] * z + q[3]
        inn = (s > 0) | (bool(closed) & (s == 0))
    elif kind == CYLINDER:
        ax = np.array(q[4:7])
        height = np.sqrt(ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2])
        zz = ax / height
        v = P - np.array(q[0:3])
        proj = _dot(v, zz[None, :])
        cr = _cross(v, np.broadcast_to(zz, v.shape))
        devi = np.sqrt(_dot(cr, cr))
        return ~((proj > height) | (proj < 0)) & ~(devi >= q[3])
    else:
        raise ValueError(kind)
    return inn ^ bool(complement)


def node_positions(origin, h, dims):
    nx, ny, nz = dims
    i = np.arange(nx * ny * nz)
    ix, iy, iz = i % nx, (i // nx) % ny, i // (nx * ny)
    o = np.asarray(origin, np.float64)
    return np.stack([o[0] + ix * h, o[1] + iy * h, o[2] + iz * h], axis=1)


def region_mask(regions, origin, h, dims):
    """Union of regions [(kind, p, closed, complement)] on the node grid; (nz, ny, nx) uint8."""
    P = node_positions(origin, h, dims)
    m = np.zeros(len(P), bool)
    for kind, p, closed, comp in regions:
        m |= contains(kind, p, closed, comp, P)
    nx, ny, nz = dims
    return m.astype(np.uint8).reshape(nz, ny, nx)


def _norm(kind, q, P):
    if kind == CONSTANT:
        return np.full(len(P), q[0])
    if kind == RADIAL:
        d = np.array(q[0:3])[None, :] - P
        radi = np.sqrt(_dot(d, d))
        return q[3] * np.exp(-np.power(radi, q[4] * 2))
    s = np.array(q[0:3])
    ax = _unit(np.array(q[3:6]) - s)
    cr = _cross(P - s, np.broadcast_to(ax, P.shape))
    return np.sqrt(_dot(cr, cr)) * q[6]


def _dir(kind, q, P):
    if kind == CONSTANT:
        return np.broadcast_to(_unit(np.array(q[0:3])), P.shape)
    if kind == RADIAL:
        return _unit(np.array(q[0:3])[None, :] - P)
    s = np.array(q[0:3])
    return _unit(_cross(P - s, np.broadcast_to(np.array(q[3:6]) - s, P.shape)))


def region_field(fields, P):
    """Sum of fields [((kind, p, closed, complement), norm_kind, norm_p, dir_kind, dir_p)] at P (n, 3)."""
    P = np.asarray(P, np.float64).reshape(-1, 3)
    s = np.zeros_like(P)
    for (kind, p, closed, comp), nk, npar, dk, dpar in fields:
        inside = contains(kind, p, closed, comp, P)
        m = _norm(nk, [float(v) for v in npar], P)
        d = _dir(dk, [float(v) for v in dpar], P)
        s = np.where(inside[:, None], s + m[:, None] * d, s)
    return s


def closest_on_triangle(P, a, b, c):
    """Closest points of triangle (a, b, c) to points P (n, 3), branch by branch
    as the library's device function."""
    P = np.asarray(P, np.float64)
    a, b, c = (np.asarray(t, np.float64)[None, :] for t in (a, b, c))
    ab, ac, ap = b - a, c - a, P - a
    d1, d2 = _dot(ab, ap), _dot(ac, ap)
    bp = P - b
    d3, d4 = _dot(ab, bp), _dot(ac, bp)
    vc = d1 * d4 - d3 * d2
    cp = P - c
    d5, d6 = _dot(ab, cp), _dot(ac, cp)
    vb = d5 * d2 - d1 * d6
    va = d3 * d6 - d5 * d4
    e43, e56 = d4 - d3, d5 - d6
    with np.errstate(invalid="ignore", divide="ignore", over="ignore"):
        den = va + vb + vc
        v, w = _qdiv(vb, den), _qdiv(vc, den)
        inner = (a + v[:, None] * ab) + w[:, None] * ac
        out = inner
        out = np.where(((va <= 0) & (e43 >= 0) & (e56 >= 0))[:, None], b + _qdiv(e43, e43 + e56)[:, None] * (c - b), out)
        out = np.where(((vb <= 0) & (d2 >= 0) & (d6 <= 0))[:, None], a + _qdiv(d2, d2 - d6)[:, None] * ac, out)
        out = np.where(((d6 >= 0) & (d5 <= d6))[:, None], np.broadcast_to(c, P.shape), out)
        out = np.where(((vc <= 0) & (d1 >= 0) & (d3 <= 0))[:, None], a + _qdiv(d1, d1 - d3)[:, None] * ab, out)
        out = np.where(((d3 >= 0) & (d4 <= d3))[:, None], np.broadcast_to(b, P.shape), out)
        out = np.where(((d1 <= 0) & (d2 <= 0))[:, None], np.broadcast_to(a, P.shape), out)
    return out


def _sat_int(q):
    return int(np.trunc(min(max(q, -2147483648.0), 2147483647.0)))


def shell_elements(vertices, faces, box, R, shell_width, solid):
    """Shell elements (R, R, R) uint8, face by face over each face's index box."""
    V = np.asarray(vertices, np.float32).reshape(-1, 3).astype(np.float64)
    F = np.asarray(faces, np.int64).reshape(-1, 3)
    b = np.asarray(box, np.float32)
    eh = float(np.float32(np.float32(b[3] - b[0]) / np.float32(R)))
    w = float(shell_width) * eh
    b0 = [float(b[0]), float(b[1]), float(b[2])]
    sol = np.asarray(solid, np.uint8).reshape(-1)
    shell = np.zeros(R ** 3, np.uint8)
    if not w > 0:
        return shell.reshape(R, R, R)
    sh2 = w * w
    for f in F:
        A, B, C = V[f[0]], V[f[1]], V[f[2]]
        lid, rid = [], []
        for j in range(3):
            lo = min(min(A[j], B[j]), C[j])
            hi = max(max(A[j], B[j]), C[j])
            ql = (lo - w * 1.3 - b0[j] - 0.5 * eh) / eh
            qr = (hi + w * 1.3 - b0[j] - 0.5 * eh) / eh + 1
            lid.append(min(max(_sat_int(ql), 0), R - 1))
            rid.append(min(max(_sat_int(qr), 0), R - 1))
        if any(rid[j] - lid[j] <= 0 for j in range(3)):
            continue
        zz, yy, xx = np.meshgrid(np.arange(lid[2], rid[2]), np.arange(lid[1], rid[1]), np.arange(lid[0], rid[0]),
                                 indexing="ij")
        xx, yy, zz = xx.ravel(), yy.ravel(), zz.ravel()
        e = xx + R * (yy + R * zz)
        keep = sol[e] != 0
        xx, yy, zz, e = xx[keep], yy[keep], zz[keep], e[keep]
        if e.size == 0:
            continue
        P = np.stack([(xx + 0.5) * eh + b0[0], (yy + 0.5) * eh + b0[1], (zz + 0.5) * eh + b0[2]], axis=1)
        d = P - closest_on_triangle(P, A, B, C)
        shell[e[_dot(d, d) < sh2]] = 1
    return shell.reshape(R, R, R)


def mesh_normals(vertices, faces, points):
    """Outward normals at points (n, 3): closest face (lowest index on a tie), then outwardNormal's rule."""
    V = np.asarray(vertices, np.float32).reshape(-1, 3).astype(np.float64)
    F = np.asarray(faces, np.int64).reshape(-1, 3)
    P = np.asarray(points, np.float64).reshape(-1, 3)
    best = np.full(len(P), np.inf)
    bq = P.copy()
    bf = np.zeros(len(P), np.int64)
    for k, f in enumerate(F):
        q = closest_on_triangle(P, V[f[0]], V[f[1]], V[f[2]])
        d = q - P
        d2 = _dot(d, d)
        upd = d2 < best
        best = np.where(upd, d2, best)
        bq = np.where(upd[:, None], q, bq)
        bf = np.where(upd, k, bf)
    A, B, C = V[F[bf, 0]], V[F[bf, 1]], V[F[bf, 2]]
    tn = _cross(A - C, B - C)
    pq = bq - P
    ln = np.sqrt(_dot(pq, pq))
    near = ln < 1e-6
    ln = np.where(_dot(pq, tn) < 0, -ln, ln)
    with np.errstate(invalid="ignore", divide="ignore"):
        n = pq / np.where(near, 1.0, ln)[:, None]
    return np.where(near[:, None], _unit(tn), n)
