"""Solid voxelisation restated in numpy FP32, operation by operation.

TEST INFRASTRUCTURE ONLY: the checker of rso_voxelize; the product library
never imports it.  Parity unpinned: the reference ships no voxelisation
fixtures and its voxeliser cannot be built here; the tests add exact counts on
a cube and a sphere's volume.

Restates the solid mode of the cuda_voxelizer the reference vendors
(voxelizer/cpu_voxelizer.cpp:206-330, cpu_voxelize_mesh_solid with
checkCCW, check_point_triangle, TopLeftEdge, get_x_coordinate) and the grid
of voxelize_mesh / padd2SatifyResolution (voxelizer/voxelize_main.cpp:
313-399).  FP32 where the reference computes in float (glm), double where it
promotes (the - 0.5 of the grid indices and the sample points).
"""
import math

import numpy as np

f32 = np.float32
EPS = f32(0.000001)


def grid(vertices, preferred):
    v = np.asarray(vertices, np.float32).reshape(-1, 3)
    R = 1
    for _ in range(32):
        if preferred < R:
            break
        R <<= 1
    lo, hi = v.min(axis=0), v.max(axis=0)
    ln = (hi - lo).astype(f32)
    maxlen = f32(max(ln[0], ln[1], ln[2]))
    pad = f32(f32(maxlen * f32(R)) / f32(preferred))
    bmin = (lo - (pad - ln) / f32(2)).astype(f32)
    bmax = (hi + (pad - ln) / f32(2)).astype(f32)
    return R, bmin, bmax


def _pit(a, b, c, p):
    pa, pb, pc = p - a, p - b, p - c
    t1 = f32(pa[0] * pb[1]) - f32(pa[1] * pb[0])
    if abs(t1) < EPS and pa[0] * pb[0] <= 0 and pa[1] * pb[1] <= 0:
        return 1
    t2 = f32(pb[0] * pc[1]) - f32(pb[1] * pc[0])
    if abs(t2) < EPS and pb[0] * pc[0] <= 0 and pb[1] * pc[1] <= 0:
        return 2
    t3 = f32(pc[0] * pa[1]) - f32(pc[1] * pa[0])
    if abs(t3) < EPS and pc[0] * pa[0] <= 0 and pc[1] * pa[1] <= 0:
        return 3
    return 0 if (t1 * t2 > 0 and t1 * t3 > 0) else -1


def _tl(v0, v1):
    return (v1[1] < v0[1]) or (v1[1] == v0[1] and v0[0] > v1[0])


def voxelize(vertices, faces, preferred):
    """(solid [z][y][x] uint8, R, box) as rso_voxelize computes them."""
    v = np.asarray(vertices, np.float32).reshape(-1, 3)
    F = np.asarray(faces, np.int64).reshape(-1, 3)
    R, bmin, bmax = grid(v, preferred)
    unit = f32(f32(bmax[0] - bmin[0]) / f32(R))
    cross = np.zeros((R, R, R), np.uint8)
    vt = (v - bmin).astype(f32)
    for tri in F:
        v0, v1, v2 = vt[tri[0]], vt[tri[1]], vt[tri[2]]
        e0, e1 = (v1 - v0).astype(f32), (v2 - v1).astype(f32)
        n = np.array([f32(e0[1] * e1[2]) - f32(e0[2] * e1[1]), f32(e0[2] * e1[0]) - f32(e0[0] * e1[2]),
                      f32(e0[0] * e1[1]) - f32(e0[1] * e1[0])], np.float32)
        nd = f32(f32(f32(n[0] * n[0]) + f32(n[1] * n[1])) + f32(n[2] * n[2]))
        if not nd > 0:
            continue
        inv = f32(f32(1) / np.sqrt(nd))
        n = (n * inv).astype(f32)
        if abs(n[0]) < EPS:
            continue
        a, b, c = v0[1:].copy(), v1[1:].copy(), v2[1:].copy()
        d0, d1 = (b - a).astype(f32), (c - a).astype(f32)
        if not (f32(d0[0] * d1[1]) - f32(d1[0] * d0[1])) > 0:
            b, c = c, b
        ymax, zmax = max(a[0], b[0], c[0]), max(a[1], b[1], c[1])
        ymin, zmin = min(a[0], b[0], c[0]), min(a[1], b[1], c[1])
        y1 = max(math.floor(float(f32(ymax / unit)) - 0.5), -1)
        z1 = max(math.floor(float(f32(zmax / unit)) - 0.5), -1)
        y0 = max(math.ceil(float(f32(ymin / unit)) - 0.5), 0)
        z0 = max(math.ceil(float(f32(zmin / unit)) - 0.5), 0)
        for y in range(y0, min(y1, R - 1) + 1):
            for z in range(z0, min(z1, R - 1) + 1):
                p = np.array([f32((y + 0.5) * float(unit)), f32((z + 0.5) * float(unit))], np.float32)
                k = _pit(a, b, c, p)
                if (k == 1 and _tl(a, b)) or (k == 2 and _tl(b, c)) or (k == 3 and _tl(c, a)) or k == 0:
                    num = f32(f32(n[1] * f32(p[0] - v0[1])) + f32(n[2] * f32(p[1] - v0[2])))
                    xi = f32(f32(-num / n[0]) + v0[0])
                    xm = int(float(f32(xi / unit)) - 0.5)
                    if xm < 0:
                        continue
                    cross[z, y, min(xm, R - 1)] ^= 1
    solid = (np.cumsum(cross[:, :, ::-1], axis=2)[:, :, ::-1] & 1).astype(np.uint8)
    return solid, R, np.concatenate([bmin, bmax])
