"""Seeded synthetic problems in the shapes of the benchmark configurations.

Every problem is a box of unit voxels; masks are (ez, ey, ex) element arrays
and (nz, ny, nx) node arrays, x fastest.  No external data is used.
"""
import numpy as np


def box_filter3(rho, mask):
    """One 3x3x3 box-mean pass over in-box active neighbours."""
    ez, ey, ex = rho.shape
    acc = np.zeros_like(rho)
    cnt = np.zeros_like(rho)
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                src = np.zeros_like(rho)
                m = np.zeros_like(rho)
                zs = slice(max(dz, 0), ez + min(dz, 0))
                zd = slice(max(-dz, 0), ez + min(-dz, 0))
                ys = slice(max(dy, 0), ey + min(dy, 0))
                yd = slice(max(-dy, 0), ey + min(-dy, 0))
                xs = slice(max(dx, 0), ex + min(dx, 0))
                xd = slice(max(-dx, 0), ex + min(-dx, 0))
                src[zd, yd, xd] = (rho * mask)[zs, ys, xs]
                m[zd, yd, xd] = mask[zs, ys, xs]
                acc += src
                cnt += m
    return np.where(cnt > 0, acc / np.maximum(cnt, 1), 0.0)


def cantilever(ex=64, ey=32, ez=32, seed=0):
    """Config 0: all voxels active, x=0 face clamped, unit -z tip line load
    on the x=ex face's mid-height line; density U[0.2,1] then one box pass."""
    rng = np.random.default_rng(seed)
    em = np.ones((ez, ey, ex), np.uint8)
    nx, ny, nz = ex + 1, ey + 1, ez + 1
    fa = np.zeros((nz, ny, nx), np.uint8)
    fa[:, :, 0] = 1
    la = np.zeros((nz, ny, nx), np.uint8)
    la[ez // 2, :, ex] = 1
    rho = box_filter3(rng.uniform(0.2, 1.0, size=em.shape), em.astype(float))
    nn = nx * ny * nz
    f = np.zeros(3 * nn)
    for y in range(ny):
        f[2 * nn + ex + nx * (y + ny * (ez // 2))] = -1.0 / ny
    return dict(emask=em, fixed=fa, load=la, normals=None, rho=rho, f=f)


def ellipsoid(ex=32, ey=16, ez=16, seed=1, shell=3, axes=None):
    """Config 1 shape: voxels whose centres lie in the ellipsoid with
    semi-axes `axes` (default (ex/2-2, ey/2-2, ez/2-2)) centred in the box;
    lowest active node layer clamped; load area = nodes within `shell` voxels
    of the boundary (only surface nodes become load nodes); analytic outward
    normals; rho 0.4 +- 0.05."""
    rng = np.random.default_rng(seed)
    a, b, c = axes if axes is not None else (ex / 2 - 2, ey / 2 - 2, ez / 2 - 2)
    zc, yc, xc = np.meshgrid(np.arange(ez) + 0.5, np.arange(ey) + 0.5, np.arange(ex) + 0.5, indexing="ij")
    em = (((xc - ex / 2) / a) ** 2 + ((yc - ey / 2) / b) ** 2 + ((zc - ez / 2) / c) ** 2 <= 1).astype(np.uint8)
    nx, ny, nz = ex + 1, ey + 1, ez + 1
    zn, yn, xn = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    # active nodes
    vm = np.zeros((nz, ny, nx), bool)
    for k in range(8):
        dx, dy, dz = k & 1, (k >> 1) & 1, k >> 2
        vm[dz:dz + ez, dy:dy + ey, dx:dx + ex] |= em.astype(bool)
    zlow = np.min(np.where(vm.any(axis=(1, 2)))[0])
    fa = np.zeros((nz, ny, nx), np.uint8)
    fa[zlow] = 1
    r = np.sqrt(((xn - ex / 2) / a) ** 2 + ((yn - ey / 2) / b) ** 2 + ((zn - ez / 2) / c) ** 2)
    la = (r >= 1 - shell / min(a, b, c)).astype(np.uint8)
    g = np.stack([(xn - ex / 2) / a ** 2, (yn - ey / 2) / b ** 2, (zn - ez / 2) / c ** 2])
    g = g / np.maximum(np.linalg.norm(g, axis=0), 1e-12)
    rho = np.where(em > 0, 0.4 + rng.uniform(-0.05, 0.05, size=em.shape), 0.0)
    return dict(emask=em, fixed=fa, load=la, normals=np.ascontiguousarray(g.reshape(3, -1).T), rho=rho)


def top_loaded_cube(n=16, seed=2):
    """Config 4 shape at small size: all active, z=0 clamped, load area the
    top face (free-force worst case)."""
    em = np.ones((n, n, n), np.uint8)
    fa = np.zeros((n + 1, n + 1, n + 1), np.uint8)
    fa[0] = 1
    la = np.zeros_like(fa)
    la[n] = 1
    rng = np.random.default_rng(seed)
    rho = rng.uniform(0.3, 1.0, size=em.shape)
    return dict(emask=em, fixed=fa, load=la, normals=None, rho=rho)


def voids_box(ex=48, ey=24, ez=24, nvoids=6, seed=3):
    """Config 2 shape at small size: box with spherical voids, x=0 clamped,
    load area the x=ex face (normal +x)."""
    rng = np.random.default_rng(seed)
    zc, yc, xc = np.meshgrid(np.arange(ez) + 0.5, np.arange(ey) + 0.5, np.arange(ex) + 0.5, indexing="ij")
    em = np.ones((ez, ey, ex), bool)
    for _ in range(nvoids):
        c = rng.uniform([0, 0, 0], [ex, ey, ez])
        r = rng.uniform(2, 5)
        em &= (xc - c[0]) ** 2 + (yc - c[1]) ** 2 + (zc - c[2]) ** 2 > r * r
    em = em.astype(np.uint8)
    nx, ny, nz = ex + 1, ey + 1, ez + 1
    fa = np.zeros((nz, ny, nx), np.uint8)
    fa[:, :, 0] = 1
    la = np.zeros((nz, ny, nx), np.uint8)
    la[:, :, ex] = 1
    nrm = np.zeros((nz * ny * nx, 3))
    nrm[:, 0] = 1.0
    rho = box_filter3(rng.uniform(0.2, 1.0, size=em.shape), em.astype(float))
    return dict(emask=em, fixed=fa, load=la, normals=nrm, rho=rho)
