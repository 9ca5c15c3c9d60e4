"""Mesh input: Wavefront OBJ reading and solid voxelisation (rso_voxelize).

The reference reads a mesh (CGAL / trimesh in its drivers) and voxelises it
with its vendored cuda_voxelizer before building the hierarchy
(voxelizer/voxelize_main.cpp:344-399); voxelize() returns the element mask
HierarchyGrid takes.
"""
import ctypes

import numpy as np

from .rso import RSOError, _np_ptr, _pd, load_library


def read_obj(path):
    """(vertices (n, 3) float32, faces (m, 3) int32) of an OBJ file; polygons are fanned into
    triangles, negative (relative) indices resolved."""
    verts, faces = [], []
    with open(path) as fh:
        for line in fh:
            parts = line.split()
            if not parts:
                continue
            if parts[0] == "v":
                verts.append([float(x) for x in parts[1:4]])
            elif parts[0] == "f":
                idx = []
                for tok in parts[1:]:
                    i = int(tok.split("/")[0])
                    idx.append(i - 1 if i > 0 else len(verts) + i)
                for k in range(1, len(idx) - 1):
                    faces.append([idx[0], idx[k], idx[k + 1]])
    return np.asarray(verts, np.float32).reshape(-1, 3), np.asarray(faces, np.int32).reshape(-1, 3)


def voxelize(vertices, faces, preferred_resolution):
    """(solid mask (R, R, R) uint8 indexed [z][y][x], R, box (6,)) of a closed triangle mesh."""
    lib = load_library()
    v = np.ascontiguousarray(vertices, np.float32).reshape(-1)
    f = np.ascontiguousarray(faces, np.int32).reshape(-1)
    r = ctypes.c_int(0)
    fp = ctypes.POINTER(ctypes.c_float)
    ip = ctypes.POINTER(ctypes.c_int)
    st = lib.rso_voxelize(v.ctypes.data_as(fp), v.size // 3, f.ctypes.data_as(ip), f.size // 3, int(preferred_resolution),
                          None, ctypes.byref(r), None)
    if st:
        raise RSOError(f"rso_voxelize: status {st}")
    R = r.value
    solid = np.zeros(R ** 3, np.uint8)
    box = np.zeros(6, np.float32)
    st = lib.rso_voxelize(v.ctypes.data_as(fp), v.size // 3, f.ctypes.data_as(ip), f.size // 3, int(preferred_resolution),
                          solid.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), ctypes.byref(r), box.ctypes.data_as(fp))
    if st:
        raise RSOError(f"rso_voxelize: status {st}")
    return solid.reshape(R, R, R), R, box
