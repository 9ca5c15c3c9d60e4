"""Boundary conditions of a mesh problem: regions, load fields, shell
elements and outward normals (rso_region_mask, rso_region_field,
rso_shell_elements, rso_mesh_normals).

The reference's driver reads the fixed area, the load area and the load
field into static_range::rangeUnion and dynamic_range::Field_t objects
(config_parser_t, config_parser.h:84-108; boundary/BoundaryCondition.h) and
evaluates them at the surface nodes of the voxel grid in
computeProjectionMatrix (grid/Grid.cpp:2694-2760): a node in the fixed area
becomes a support node, otherwise a node in the load area becomes a load node
carrying the field's force and the mesh's outward normal there
(Grid::outwardNormal, grid/Grid.cpp:2838-2854).  Shell elements are the solid
elements within shell_width voxels of the mesh
(HierarchyGrid::setSolidShellElement, grid/Grid.cpp:253-322).

Regions come from the constructors below, from the text format that
static_range::rangeUnion::parse reads (parse_ranges), or from a JSON document
(load_bc_json).  The reference's JSON reader,
config_parser_t::parse_benchmark_configuration, is declared in config_parser.h
but its body is not among the reference sources, so load_bc_json defines its
own schema over the same region and field kinds.
"""
import ctypes
import json
import re

import numpy as np

from .rso import RSOError, _Field, _Region, load_library
from .voxelize import voxelize

SPHERE, BOX, HALFSPACE, CYLINDER = 0, 1, 2, 3
CONSTANT, RADIAL, TWIST = 0, 1, 2


class Region:
    """One region: kind (SPHERE, BOX, HALFSPACE, CYLINDER), parameters as rso_region.p."""

    def __init__(self, kind, params, closed=False, complement=False):
        self.kind = int(kind)
        self.p = [float(v) for v in params]
        self.closed = bool(closed)
        self.complement = bool(complement)

    def c(self):
        r = _Region()
        r.kind, r.closed, r.complement = self.kind, int(self.closed), int(self.complement)
        for i, v in enumerate(self.p):
            r.p[i] = v
        return r

    def __repr__(self):
        name = {SPHERE: "sphere", BOX: "box", HALFSPACE: "halfspace", CYLINDER: "cylinder"}[self.kind]
        return f"Region({name}, {self.p}, closed={self.closed}, complement={self.complement})"


def sphere(center, radius, closed=False, complement=False):
    """sphereRange_t (boundary/BoundaryCondition.h:401-425)."""
    return Region(SPHERE, list(center) + [radius], closed, complement)


def box(p1, p2, closed=False, complement=False):
    """boxRange_t from two diagonal points: CGAL's Iso_cuboid_3(p, q) keeps the
    coordinate-wise minimum and maximum (boundary/BoundaryCondition.h:443-445)."""
    lo = [min(float(a), float(b)) for a, b in zip(p1, p2)]
    hi = [max(float(a), float(b)) for a, b in zip(p1, p2)]
    return Region(BOX, lo + hi, closed, complement)


def box_h(min_h, max_h, hw=1.0, closed=False, complement=False):
    """boxRange_t from homogeneous corners (min/hw, max/hw), taken as given
    (boundary/BoundaryCondition.h:451-457)."""
    return Region(BOX, [float(v) / hw for v in min_h] + [float(v) / hw for v in max_h], closed, complement)


def halfspace(a, b, c, d, closed=False, complement=False):
    """halfSpaceRange_t(a, b, c, d): CGAL's Plane_3(a, b, c, d) is
    a x + b y + c z + d = 0 and the region its positive side
    (boundary/BoundaryCondition.h:479-483)."""
    return Region(HALFSPACE, [a, b, c, d], closed, complement)


def plane_through(p, q, r):
    """Coefficients (a, b, c, d) of the plane through p, q, r with p, q, r
    counterclockwise seen from its positive side: (p - r) x (q - r), d = -n . r
    (the plane through three points of CGAL's Cartesian kernel)."""
    px, py, pz = (float(v) for v in p)
    qx, qy, qz = (float(v) for v in q)
    rx, ry, rz = (float(v) for v in r)
    rpx, rpy, rpz = px - rx, py - ry, pz - rz
    rqx, rqy, rqz = qx - rx, qy - ry, qz - rz
    a = rpy * rqz - rqy * rpz
    b = rpz * rqx - rqz * rpx
    c = rpx * rqy - rqx * rpy
    d = -a * rx - b * ry - c * rz
    return a, b, c, d


def halfspace_points(p1, p2, p3, closed=False, complement=False):
    """halfSpaceRange_t through three points (boundary/BoundaryCondition.h:491-505)."""
    return Region(HALFSPACE, plane_through(p1, p2, p3), closed, complement)


def cylinder(bottom, radius, axis):
    """cylinderRange_t (boundary/BoundaryCondition.h:509-538); closed and
    complement do not apply to it."""
    return Region(CYLINDER, list(bottom) + [radius] + list(axis))


class Field:
    """rangeField_t: norm(p) * dir(p) inside `region`, zero outside.
    norm: ("constant", value) | ("radial", centre, amplifier=1, damp=1) | ("twist", start, end, amplifier)
    dir:  ("constant", vector) | ("radial", centre) | ("twist", start, end)"""

    def __init__(self, region, norm, direction):
        self.region, self.norm, self.direction = region, tuple(norm), tuple(direction)

    def c(self):
        f = _Field()
        f.region = self.region.c()
        kinds = {"constant": CONSTANT, "radial": RADIAL, "twist": TWIST}
        nk, dk = self.norm[0], self.direction[0]
        f.norm_kind, f.dir_kind = kinds[nk], kinds[dk]
        if nk == "constant":
            npar = [self.norm[1]]
        elif nk == "radial":
            amp = self.norm[2] if len(self.norm) > 2 else 1.0
            damp = self.norm[3] if len(self.norm) > 3 else 1.0
            npar = list(self.norm[1]) + [amp, damp]
        else:
            npar = list(self.norm[1]) + list(self.norm[2]) + [self.norm[3]]
        if dk == "twist":
            dpar = list(self.direction[1]) + list(self.direction[2])
        else:
            dpar = list(self.direction[1])
        for i, v in enumerate(npar):
            f.norm_p[i] = float(v)
        for i, v in enumerate(dpar):
            f.dir_p[i] = float(v)
        return f


# a C++ stream extraction of a double reads this prefix of a token
_NUM = re.compile(r"[+-]?(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?")


def _read_numbers(line):
    """Doubles read from a line as `istringstream >> double` reads them: until the first extraction fails."""
    out = []
    pos = 0
    while True:
        while pos < len(line) and line[pos].isspace():
            pos += 1
        m = _NUM.match(line, pos)
        if not m:
            return out
        out.append(float(m.group(0)))
        pos = m.end()


def parse_ranges(text):
    """Regions of the text format of static_range::rangeUnion::parse
    (boundary/BoundaryCondition.h:259-334), line by line:
      - a line containing "box", "sphere", "halfspace", "closed", "open" or
        "complement" (tested in that order, first match wins) switches the
        parser state and clears the collected numbers;
      - any other line appends its numbers, and a region is added whenever the
        collected count fits the current kind: box 6 (two corners) or 7
        (homogeneous corners), sphere 4 (centre, radius), halfspace 4
        (a, b, c, d) or 9 (three points);
    the numbers are not cleared after a region is added, so each region needs
    its own keyword line, and a line without numbers after a complete region
    adds it once more.  The initial state is box, open.  "complement" is
    recorded but has no effect (the parser adds every region uncomplemented),
    and "nocomplement" matches "complement" first.  Lines longer than 511
    characters end the input (istream::getline into a 512-byte buffer)."""
    regions = []
    kind, closed = BOX, False
    params = []
    lines = text.split("\n")
    if lines and lines[-1] == "":
        lines.pop()  # getline reads no line after a final newline
    for line in lines:
        if len(line) > 511:
            break
        changed = True
        if "box" in line:
            kind = BOX
        elif "sphere" in line:
            kind = SPHERE
        elif "halfspace" in line:
            kind = HALFSPACE
        elif "closed" in line:
            closed = True
        elif "open" in line:
            closed = False
        elif "complement" in line:
            pass
        else:
            changed = False
        if changed:
            params = []
            continue
        params.extend(_read_numbers(line))
        n = len(params)
        if kind == BOX and n == 6:
            regions.append(box(params[0:3], params[3:6], closed))
        elif kind == BOX and n == 7:
            regions.append(box_h(params[0:3], params[3:6], params[6], closed))
        elif kind == SPHERE and n == 4:
            regions.append(sphere(params[0:3], params[3], closed))
        elif kind == HALFSPACE and n == 4:
            regions.append(halfspace(*params, closed=closed))
        elif kind == HALFSPACE and n == 9:
            regions.append(halfspace_points(params[0:3], params[3:6], params[6:9], closed))
    return regions


def _region_from_json(d):
    t = d["type"]
    closed, comp = bool(d.get("closed", False)), bool(d.get("complement", False))
    if t == "sphere":
        return sphere(d["center"], d["radius"], closed, comp)
    if t == "box":
        if "hw" in d:
            return box_h(d["min"], d["max"], d["hw"], closed, comp)
        return box(d["min"], d["max"], closed, comp)
    if t == "halfspace":
        if "points" in d:
            p = d["points"]
            return halfspace_points(p[0], p[1], p[2], closed, comp)
        return halfspace(*d["plane"], closed=closed, complement=comp)
    if t == "cylinder":
        return cylinder(d["bottom"], d["radius"], d["axis"])
    if t == "text":
        raise ValueError("a text entry expands to several regions")
    raise ValueError(f"unknown region type {t!r}")


def _regions_from_json(items):
    out = []
    for d in items:
        if d.get("type") == "text":
            out.extend(parse_ranges(d["text"]))
        else:
            out.append(_region_from_json(d))
    return out


def load_bc_json(src):
    """{"fix": [regions], "load": [regions], "force": [fields]} from a JSON file
    path, a JSON string or a parsed dict.  A region is
      {"type": "sphere", "center": [x, y, z], "radius": r}
      {"type": "box", "min": [...], "max": [...], ("hw": w)}
      {"type": "halfspace", "plane": [a, b, c, d]} | {"type": "halfspace", "points": [p, q, r]}
      {"type": "cylinder", "bottom": [...], "radius": r, "axis": [...]}
      {"type": "text", "text": "<static_range text format>"}
    with optional "closed" and "complement" flags; a field is
      {"region": region, "norm": ["constant", v] | ["radial", centre, amplifier, damp]
                                 | ["twist", start, end, amplifier],
       "direction": ["constant", v] | ["radial", centre] | ["twist", start, end]}."""
    if isinstance(src, dict):
        d = src
    elif isinstance(src, str) and src.lstrip().startswith("{"):
        d = json.loads(src)
    else:
        with open(src) as fh:
            d = json.load(fh)
    out = {"fix": _regions_from_json(d.get("fix", [])), "load": _regions_from_json(d.get("load", []))}
    out["force"] = [Field(_region_from_json(f["region"]), f["norm"], f["direction"]) for f in d.get("force", [])]
    return out


def _check(st, what):
    if st:
        raise RSOError(f"{what}: status {st}")


def region_mask(regions, origin, h, dims):
    """Union of `regions` on the node grid origin + (i, j, k) h, dims = (nx, ny, nz);
    (nz, ny, nx) uint8 array."""
    lib = load_library()
    nx, ny, nz = (int(v) for v in dims)
    arr = (_Region * max(len(regions), 1))(*[r.c() for r in regions])
    o = np.ascontiguousarray(origin, np.float64)
    out = np.zeros(nx * ny * nz, np.uint8)
    _check(lib.rso_region_mask(arr, len(regions), o.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), float(h), nx, ny,
                               nz, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))), "rso_region_mask")
    return out.reshape(nz, ny, nx)


def region_field(fields, points):
    """Sum of the fields at `points` ((n, 3) doubles); (n, 3) array."""
    lib = load_library()
    pts = np.ascontiguousarray(points, np.float64).reshape(-1, 3)
    arr = (_Field * max(len(fields), 1))(*[f.c() for f in fields])
    out = np.zeros_like(pts)
    pd = ctypes.POINTER(ctypes.c_double)
    _check(lib.rso_region_field(arr, len(fields), pts.ctypes.data_as(pd), len(pts), out.ctypes.data_as(pd)),
           "rso_region_field")
    return out


def _mesh_args(vertices, faces):
    v = np.ascontiguousarray(vertices, np.float32).reshape(-1)
    f = np.ascontiguousarray(faces, np.int32).reshape(-1)
    return v, f, v.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), f.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def shell_elements(vertices, faces, box_, resolution, shell_width, solid):
    """Shell elements (R, R, R) uint8 of a mesh voxelised by voxelize()."""
    lib = load_library()
    v, f, vp, fp = _mesh_args(vertices, faces)
    b = np.ascontiguousarray(box_, np.float32)
    s = np.ascontiguousarray(solid, np.uint8).reshape(-1)
    R = int(resolution)
    if s.size != R ** 3:
        raise ValueError("solid must hold R^3 bytes")
    out = np.zeros(R ** 3, np.uint8)
    pu8 = ctypes.POINTER(ctypes.c_uint8)
    _check(lib.rso_shell_elements(vp, v.size // 3, fp, f.size // 3, b.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                  R, float(shell_width), s.ctypes.data_as(pu8), out.ctypes.data_as(pu8)),
           "rso_shell_elements")
    return out.reshape(R, R, R)


def mesh_normals(vertices, faces, points):
    """Outward unit normals of the mesh at `points` ((n, 3)); (n, 3) array."""
    lib = load_library()
    v, f, vp, fp = _mesh_args(vertices, faces)
    pts = np.ascontiguousarray(points, np.float64).reshape(-1, 3)
    out = np.zeros_like(pts)
    pd = ctypes.POINTER(ctypes.c_double)
    _check(lib.rso_mesh_normals(vp, v.size // 3, fp, f.size // 3, pts.ctypes.data_as(pd), len(pts),
                                out.ctypes.data_as(pd)), "rso_mesh_normals")
    return out


def node_grid(box_, resolution):
    """(origin, h) of the node positions origin + (i, j, k) h of the voxel grid:
    h = (box max x - box min x) / R in FP32 as the reference forms it."""
    b = np.asarray(box_, np.float32)
    h = float(np.float32(np.float32(b[3] - b[0]) / np.float32(resolution)))
    return b[:3].astype(np.float64), h


def surface_nodes(emask):
    """Fine-level surface nodes of an element mask (ez, ey, ex): nodes touching a
    solid element for which some axis has no solid element pair across the
    node (mark_surface_nodes_kernel, grid/Grid.cu:2824-2858)."""
    em = np.pad(np.asarray(emask, bool), 1)
    ez, ey, ex = np.asarray(emask).shape
    s = {}
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                s[dx, dy, dz] = em[dz:dz + ez + 1, dy:dy + ey + 1, dx:dx + ex + 1]
    anyn = np.zeros_like(s[0, 0, 0])
    for k in s.values():
        anyn |= k
    ax = [np.zeros_like(anyn) for _ in range(3)]
    for a in (0, 1):
        for b in (0, 1):
            ax[0] |= s[0, a, b] & s[1, a, b]
            ax[1] |= s[a, 0, b] & s[a, 1, b]
            ax[2] |= s[a, b, 0] & s[a, b, 1]
    return anyn & ~(ax[0] & ax[1] & ax[2])


def mesh_problem(vertices, faces, preferred_resolution, fix, load, force=(), shell_width=0.0):
    """Inputs of HierarchyGrid for a mesh: voxelise, then evaluate the fixed and
    load regions on the nodes, the mesh normals and the load field at the load
    nodes (surface nodes in the load area and not in the fixed area) and the
    shell elements.  Returns dict(emask, fixed, load, normals (Nn, 3), force
    (Nn, 3), shell, box, resolution, origin, h)."""
    solid, R, bx = voxelize(vertices, faces, preferred_resolution)
    origin, h = node_grid(bx, R)
    dims = (R + 1, R + 1, R + 1)
    fixed = region_mask(fix, origin, h, dims)
    loadm = region_mask(load, origin, h, dims)
    surf = surface_nodes(solid)
    lnodes = np.flatnonzero(surf & (loadm > 0) & (fixed == 0))
    nn = (R + 1) ** 3
    normals = np.zeros((nn, 3))
    fvec = np.zeros((nn, 3))
    if lnodes.size:
        ix, iy, iz = lnodes % (R + 1), (lnodes // (R + 1)) % (R + 1), lnodes // (R + 1) ** 2
        pts = origin[None, :] + np.stack([ix, iy, iz], axis=1) * h
        normals[lnodes] = mesh_normals(vertices, faces, pts)
        if force:
            fvec[lnodes] = region_field(list(force), pts)
    shell = shell_elements(vertices, faces, bx, R, shell_width, solid) if shell_width > 0 else np.zeros_like(solid)
    return dict(emask=solid, fixed=fixed, load=loadm, normals=normals, force=fvec, shell=shell, box=bx,
                resolution=R, origin=origin, h=h)
