"""ctypes binding of the FP64 CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by the CPU-baseline leg of bench.py, always as the checker.  The product
library (robustoptspline3d_b200) never imports this module.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

_d = ctypes.POINTER(ctypes.c_double)
_u8 = ctypes.POINTER(ctypes.c_uint8)
_i32 = ctypes.POINTER(ctypes.c_int)
_u32 = ctypes.POINTER(ctypes.c_uint32)
_f32 = ctypes.POINTER(ctypes.c_float)
_i64 = ctypes.POINTER(ctypes.c_int64)
_vp = ctypes.c_void_p


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _load():
    if not os.path.exists(_LIB_PATH):
        build()
    lib = ctypes.CDLL(_LIB_PATH)
    sig = {
        "or_k0": (None, [ctypes.c_double, ctypes.c_double, ctypes.c_double, _d]),
        "or_create": (_vp, [ctypes.c_int] * 3 + [_u8, _u8, _u8, _d] + [ctypes.c_double] * 4
                      + [ctypes.c_int, ctypes.c_int]),
        "or_destroy": (None, [_vp]),
        "or_n_levels": (ctypes.c_int, [_vp]),
        "or_level_dims": (None, [_vp, ctypes.c_int, _i32]),
        "or_level_masks": (None, [_vp, ctypes.c_int, _u8, _u8]),
        "or_level_bitwords": (ctypes.c_int, [_vp, ctypes.c_int, _u32, _u32]),
        "or_node_class": (None, [_vp, _u8]),
        "or_ref_numbering": (ctypes.c_int, [_vp, ctypes.c_int, _i32, _i32, _i32, _i32, _i32, _i32]),
        "or_load_nodes": (ctypes.c_int, [_vp, _i32]),
        "or_n_load": (ctypes.c_int, [_vp]),
        "or_set_density": (None, [_vp, _d]),
        "or_apply_K": (None, [_vp, _d, _d]),
        "or_residual": (None, [_vp, _d, _d, _d]),
        "or_update_stencil": (None, [_vp]),
        "or_level_lambda": (ctypes.c_double, [_vp, ctypes.c_int]),
        "or_get_stencil": (None, [_vp, ctypes.c_int, _d]),
        "or_coarse_residual": (None, [_vp, ctypes.c_int, _d, _d, _d]),
        "or_smooth": (None, [_vp, ctypes.c_int, _d, _d, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                             ctypes.c_int]),
        "or_restrict": (None, [_vp, ctypes.c_int, _d, _d]),
        "or_prolong": (None, [_vp, ctypes.c_int, _d, _d]),
        "or_coarsest_solve": (None, [_vp, _d, _d]),
        "or_vcycle": (ctypes.c_double, [_vp, _d, _d, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_double, ctypes.c_int]),
        "or_solve": (ctypes.c_int, [_vp, _d, _d, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_double, _d]),
        "or_sensitivity": (None, [_vp, _d, _d]),
        "or_element_energy": (None, [_vp, _d, _d]),
        "or_heaviside": (None, [ctypes.c_int, _d, ctypes.c_double, ctypes.c_double, _u8, _d]),
        "or_displacement_project": (None, [ctypes.c_void_p, _d]),
        "or_solve_iterations": (ctypes.c_long, [ctypes.c_void_p]),
        "or_ss_funcs": (None, [ctypes.c_int, _d, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                               ctypes.c_double, _d]),
        "or_heaviside_chain": (None, [ctypes.c_int, _d, ctypes.c_double, _d, _d]),
        "or_filter": (None, [_vp, ctypes.c_double, _d, _d]),
        "or_density_filter": (None, [_vp, ctypes.c_double, _d, _d]),
        "or_density_filter_adjoint": (None, [_vp, ctypes.c_double, _d, _d]),
        "or_spline_setup": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
        "or_spline_info": (None, [_vp, _i32, _f32, _f32]),
        "or_spline_axis": (None, [_vp, ctypes.c_int, _i32, _d, _d]),
        "or_coeff2density": (None, [_vp, _d, ctypes.c_double, _u8, _d]),
        "or_density2coeff_adjoint": (None, [_vp, _d, _u8, _d]),
        "or_selfsupport": (ctypes.c_double, [_vp, _d, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                             ctypes.c_double, _d, _d, _d, _d]),
        "or_mc_values": (None, [_vp, _d, ctypes.c_int, _f32, _f32, _f32]),
        "or_equidistant": (ctypes.c_long, [ctypes.c_long, ctypes.c_long, _i64]),
        "or_surface_points": (ctypes.c_int, [_vp, _d, ctypes.c_int, ctypes.c_int, _f32, _f32, _i64]),
        "or_surface_selfsupport": (ctypes.c_double, [_vp, _d, _f32, ctypes.c_long, ctypes.c_double, ctypes.c_int,
                                                     ctypes.c_double, ctypes.c_double, _d, _d, _u8, _d, _d, _d]),
        "or_force_project": (None, [_vp, _d, ctypes.c_int]),
        "or_dense_worst": (ctypes.c_double, [_vp, ctypes.c_int, ctypes.c_double, _d, _d]),
        "or_lanczos": (ctypes.c_double, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_uint64,
                                         _d, _d, _d]),
        "or_modified_pm": (ctypes.c_double, [_vp, ctypes.c_int, ctypes.c_uint64, ctypes.c_int, _d, _d, _i32]),
        "or_mma_create": (_vp, [ctypes.c_int, ctypes.c_int, _d, _d]),
        "or_mma_set_x": (None, [_vp, _d]),
        "or_mma_get": (None, [_vp, _d, _d, _d, _d, _d]),
        "or_mma_update": (ctypes.c_int, [_vp, _d, _d, _d, _d]),
        "or_mma_destroy": (None, [_vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _p(a, t=_d):
    if a is None:
        return None
    return a.ctypes.data_as(t)


def k0(E=1e6, nu=0.3, h=1.0):
    out = np.zeros(576)
    lib().or_k0(E, nu, h, _p(out))
    return out.reshape(24, 24)


def heaviside(rho, beta, rhomin, shell=None):
    rho = np.ascontiguousarray(rho, np.float64)
    out = np.zeros_like(rho)
    sh = None if shell is None else np.ascontiguousarray(shell, np.uint8)
    lib().or_heaviside(rho.size, _p(rho), beta, rhomin, _p(sh, _u8), _p(out))
    return out


def heaviside_chain(rho, beta, g):
    rho = np.ascontiguousarray(rho, np.float64)
    g = np.ascontiguousarray(g, np.float64)
    out = np.zeros_like(rho)
    lib().or_heaviside_chain(rho.size, _p(rho), beta, _p(g), _p(out))
    return out


def ss_funcs(x, beta, a, mid, c):
    """The oracle's Heaviside, Dirac and self-support penalty functions at x:
    rows H, Dirac, h, dh, inner_, dinner_, overhang, doverhang, normal_distri,
    dnormal_distri (grid/Grid.cu:76-190)."""
    x = np.ascontiguousarray(x, np.float64)
    out = np.zeros((10, x.size))
    lib().or_ss_funcs(x.size, _p(x), beta, a, mid, c, _p(out))
    return out


class Problem:
    """One box problem on the CPU oracle (dense-box layout, FP64)."""

    def __init__(self, emask, fixed_area, load_area, load_normals=None, E=1e6, nu=0.3, penal=3.0,
                 rhomin=1e-3, n_levels=0, first_factor=4):
        emask = np.ascontiguousarray(emask, dtype=np.uint8)
        self.ez, self.ey, self.ex = emask.shape
        self.nn = (self.ex + 1) * (self.ey + 1) * (self.ez + 1)
        self.ne = self.ex * self.ey * self.ez
        fa = np.ascontiguousarray(fixed_area, dtype=np.uint8).ravel()
        la = np.ascontiguousarray(load_area, dtype=np.uint8).ravel()
        ln = None if load_normals is None else np.ascontiguousarray(load_normals, dtype=np.float64).ravel()
        self._keep = (emask, fa, la, ln)
        self.emask = emask
        self.h = lib().or_create(self.ex, self.ey, self.ez, _p(emask.ravel(), _u8), _p(fa, _u8), _p(la, _u8),
                                 _p(ln), E, nu, penal, rhomin, n_levels, first_factor)
        self.penal = penal
        self.rhomin = rhomin

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_destroy(self.h)
            self.h = None

    # topology
    def n_levels(self):
        return lib().or_n_levels(self.h)

    def level_dims(self, level):
        d = np.zeros(6, dtype=np.int32)
        lib().or_level_dims(self.h, level, _p(d, _i32))
        return d

    def level_masks(self, level):
        d = self.level_dims(level)
        em = np.zeros(int(d[0] * d[1] * d[2]), dtype=np.uint8)
        vm = np.zeros(int(d[3] * d[4] * d[5]), dtype=np.uint8)
        lib().or_level_masks(self.h, level, _p(em, _u8), _p(vm, _u8))
        return em, vm

    def level_bitwords(self, level):
        d = self.level_dims(level)
        ne = int(d[0] * d[1] * d[2])
        nv = int(d[3] * d[4] * d[5])
        eb = np.zeros((ne + 31) // 32, dtype=np.uint32)
        vb = np.zeros((nv + 31) // 32, dtype=np.uint32)
        lib().or_level_bitwords(self.h, level, _p(eb, _u32), _p(vb, _u32))
        return eb, vb

    def node_class(self):
        out = np.zeros(self.nn, dtype=np.uint8)
        lib().or_node_class(self.h, _p(out, _u8))
        return out

    def ref_numbering(self, level):
        counts = np.zeros(4, dtype=np.int32)
        gs_num = np.zeros(8, dtype=np.int32)
        lib().or_ref_numbering(self.h, level, _p(counts, _i32), _p(gs_num, _i32), None, None, None, None)
        nv, ne, nvgs, negs = [int(c) for c in counts]
        vl = np.zeros(nv, dtype=np.int32)
        el = np.zeros(ne, dtype=np.int32)
        vf = np.zeros(nvgs, dtype=np.int32)
        ef = np.zeros(negs, dtype=np.int32)
        lib().or_ref_numbering(self.h, level, None, None, _p(vl, _i32), _p(el, _i32), _p(vf, _i32), _p(ef, _i32))
        return dict(counts=counts, gs_num=gs_num, vlexi2gs=vl, elexi2gs=el, vflag=vf, eflag=ef)

    def load_nodes(self):
        n = lib().or_n_load(self.h)
        out = np.zeros(max(n, 1), dtype=np.int32)
        lib().or_load_nodes(self.h, _p(out, _i32))
        return out[:n]

    # operator
    def set_density(self, rho):
        self.rho = np.ascontiguousarray(rho, dtype=np.float64).ravel()
        lib().or_set_density(self.h, _p(self.rho))

    def vec(self):
        return np.zeros(3 * self.nn)

    def apply_K(self, u):
        f = self.vec()
        lib().or_apply_K(self.h, _p(np.ascontiguousarray(u, dtype=np.float64)), _p(f))
        return f

    def residual(self, u, f):
        r = self.vec()
        lib().or_residual(self.h, _p(np.ascontiguousarray(u, np.float64)), _p(np.ascontiguousarray(f, np.float64)),
                          _p(r))
        return r

    def update_stencil(self):
        lib().or_update_stencil(self.h)

    def level_lambda(self, level):
        return lib().or_level_lambda(self.h, level)

    def stencil(self, level):
        d = self.level_dims(level)
        nn = int(d[3] * d[4] * d[5])
        out = np.zeros(243 * nn)
        lib().or_get_stencil(self.h, level, _p(out))
        return out.reshape(27, 3, 3, nn)

    def smooth(self, level, u, f, kind=0, omega=1.0, sweeps=1, reverse=0):
        u = np.ascontiguousarray(u, dtype=np.float64).copy()
        lib().or_smooth(self.h, level, _p(u), _p(np.ascontiguousarray(f, np.float64)), kind, omega, sweeps, reverse)
        return u

    def restrict(self, coarse_level, rf):
        d = self.level_dims(coarse_level)
        fc = np.zeros(3 * int(d[3] * d[4] * d[5]))
        lib().or_restrict(self.h, coarse_level, _p(np.ascontiguousarray(rf, np.float64)), _p(fc))
        return fc

    def prolong(self, coarse_level, uc, uf):
        uf = np.ascontiguousarray(uf, dtype=np.float64).copy()
        lib().or_prolong(self.h, coarse_level, _p(np.ascontiguousarray(uc, np.float64)), _p(uf))
        return uf

    def coarse_residual(self, level, u, f):
        d = self.level_dims(level)
        r = np.zeros(3 * int(d[3] * d[4] * d[5]))
        lib().or_coarse_residual(self.h, level, _p(np.ascontiguousarray(u, np.float64)),
                                 _p(np.ascontiguousarray(f, np.float64)), _p(r))
        return r

    def coarsest_solve(self, f):
        d = self.level_dims(self.n_levels() - 1)
        u = np.zeros(3 * int(d[3] * d[4] * d[5]))
        lib().or_coarsest_solve(self.h, _p(np.ascontiguousarray(f, np.float64)), _p(u))
        return u

    def vcycle(self, u, f, pre=1, post=1, kind=0, omega=1.0, symmetric=0):
        u = np.ascontiguousarray(u, dtype=np.float64).copy()
        rr = lib().or_vcycle(self.h, _p(u), _p(np.ascontiguousarray(f, np.float64)), pre, post, kind, omega,
                             symmetric)
        return u, rr

    def solve_iterations(self):
        """Iterations of all solves on this problem so far."""
        return lib().or_solve_iterations(self.h)

    def displacement_project(self, u):
        """u without rigid motion (a no-op for problems with supports)."""
        u = np.ascontiguousarray(u, np.float64).copy()
        lib().or_displacement_project(self.h, _p(u))
        return u

    def solve(self, f, tol=1e-10, max_iter=200, method=1, pre=1, post=1, kind=0, omega=1.0, u0=None):
        u = self.vec() if u0 is None else np.ascontiguousarray(u0, np.float64).copy()
        rr = ctypes.c_double(0)
        it = lib().or_solve(self.h, _p(u), _p(np.ascontiguousarray(f, np.float64)), tol, max_iter, method, pre,
                            post, kind, omega, ctypes.byref(rr))
        return u, it, rr.value

    # design
    def sensitivity(self, u):
        s = np.zeros(self.ne)
        lib().or_sensitivity(self.h, _p(np.ascontiguousarray(u, np.float64)), _p(s))
        return s

    def element_energy(self, u):
        s = np.zeros(self.ne)
        lib().or_element_energy(self.h, _p(np.ascontiguousarray(u, np.float64)), _p(s))
        return s

    def filter(self, radius, g):
        out = np.zeros(self.ne)
        lib().or_filter(self.h, radius, _p(np.ascontiguousarray(g, np.float64)), _p(out))
        return out

    def density_filter(self, radius, g):
        out = np.zeros(self.ne)
        lib().or_density_filter(self.h, radius, _p(np.ascontiguousarray(g, np.float64)), _p(out))
        return out

    def density_filter_adjoint(self, radius, g):
        out = np.zeros(self.ne)
        lib().or_density_filter_adjoint(self.h, radius, _p(np.ascontiguousarray(g, np.float64)), _p(out))
        return out

    def spline_setup(self, order, parts):
        self.n_coeff = lib().or_spline_setup(self.h, order, parts[0], parts[1], parts[2])
        self.order = order
        return self.n_coeff

    def spline_info(self):
        nb = np.zeros(3, dtype=np.int32)
        bmin = np.zeros(3, dtype=np.float32)
        step = np.zeros(3, dtype=np.float32)
        lib().or_spline_info(self.h, _p(nb, _i32), _p(bmin, _f32), _p(step, _f32))
        return nb, bmin, step

    def spline_axis(self, axis):
        n = [self.ex, self.ey, self.ez][axis]
        idx = np.zeros(n, dtype=np.int32)
        N = np.zeros(n * self.order)
        dN = np.zeros(n * self.order)
        lib().or_spline_axis(self.h, axis, _p(idx, _i32), _p(N), _p(dN))
        return idx, N.reshape(n, self.order), dN.reshape(n, self.order)

    def coeff2density(self, c, shell=None):
        out = np.zeros(self.ne)
        sh = None if shell is None else np.ascontiguousarray(shell, np.uint8)
        lib().or_coeff2density(self.h, _p(np.ascontiguousarray(c, np.float64)), self.rhomin, _p(sh, _u8), _p(out))
        return out

    def density2coeff_adjoint(self, g, shell=None):
        out = np.zeros(self.n_coeff)
        sh = None if shell is None else np.ascontiguousarray(shell, np.uint8)
        lib().or_density2coeff_adjoint(self.h, _p(np.ascontiguousarray(g, np.float64)), _p(sh, _u8), _p(out))
        return out

    def selfsupport(self, c, beta, mode=4, opt_angle=0.75 * np.pi, default_angle=0.75 * np.pi):
        per = np.zeros(self.ne)
        dc = np.zeros(self.n_coeff)
        cnt = ctypes.c_double(0)
        dsum = ctypes.c_double(0)
        v = lib().or_selfsupport(self.h, _p(np.ascontiguousarray(c, np.float64)), beta, mode, opt_angle,
                                 default_angle, _p(per), _p(dc), ctypes.byref(cnt), ctypes.byref(dsum))
        return v, per, dc, cnt.value, dsum.value

    # surface-point self-support
    def model_box(self):
        """bounding box of the active elements, {xmin, ymin, zmin, xmax, ymax, zmax}"""
        em = self.emask.reshape(self.ez, self.ey, self.ex)
        lo, hi = [], []
        for ax in (2, 1, 0):
            occ = np.flatnonzero(em.any(axis=tuple(a for a in range(3) if a != ax)))
            lo.append(float(occ[0]))
            hi.append(float(occ[-1] + 1))
        return np.array(lo + hi, np.float32)

    def mc_values(self, c, mc=64, box=None):
        """background values (mc+2)^3 and their coordinates (3, (mc+2)^3)"""
        box = self.model_box() if box is None else np.asarray(box, np.float32)
        out = np.zeros((mc + 2) ** 3, np.float32)
        pos = np.zeros((3, (mc + 2) ** 3), np.float32)
        lib().or_mc_values(self.h, _p(np.ascontiguousarray(c, np.float64)), mc, _p(box, _f32), _p(out, _f32),
                           _p(pos, _f32))
        return out, pos

    def surface_points(self, c, mc=64, n_points=200000, box=None):
        box = self.model_box() if box is None else np.asarray(box, np.float32)
        xyz = np.zeros(3 * max(n_points, 0), np.float32)
        info = np.zeros(4, np.int64)
        lib().or_surface_points(self.h, _p(np.ascontiguousarray(c, np.float64)), mc, n_points, _p(box, _f32),
                                _p(xyz, _f32), _p(info, _i64))
        return xyz.reshape(3, -1), info

    def surface_selfsupport(self, c, xyz, beta, mode=4, opt_angle=0.75 * np.pi, default_angle=0.75 * np.pi):
        xyz = np.ascontiguousarray(xyz, np.float32).reshape(3, -1)
        n = xyz.shape[1]
        nrm = np.zeros(3 * n)
        per = np.zeros(n)
        flags = np.zeros(2 * n, np.uint8)
        dc = np.zeros(self.n_coeff)
        cnt = ctypes.c_double(0)
        dsum = ctypes.c_double(0)
        v = lib().or_surface_selfsupport(self.h, _p(np.ascontiguousarray(c, np.float64)), _p(xyz, _f32), n, beta,
                                         mode, opt_angle, default_angle, _p(nrm), _p(per), _p(flags, _u8), _p(dc),
                                         ctypes.byref(cnt), ctypes.byref(dsum))
        return dict(value=v, normals=nrm.reshape(3, n), per=per, flags=flags.reshape(2, n), dc=dc,
                    count=cnt.value, dirsum=dsum.value)

    # worst case
    def force_project(self, f, cf):
        f = np.ascontiguousarray(f, np.float64).copy()
        lib().or_force_project(self.h, _p(f), cf)
        return f

    def dense_worst(self, cf, tol=1e-12):
        fw, uw = self.vec(), self.vec()
        lam = lib().or_dense_worst(self.h, cf, tol, _p(fw), _p(uw))
        return lam, fw, uw

    def lanczos(self, steps, cf, tol=1e-10, seed=1234):
        fw, uw = self.vec(), self.vec()
        ritz = np.zeros(steps)
        lam = lib().or_lanczos(self.h, steps, cf, tol, seed, _p(fw), _p(uw), _p(ritz))
        return lam, fw, uw, ritz

    def modified_pm(self, cf, seed=1234, max_itn=500):
        fw, uw = self.vec(), self.vec()
        itn = ctypes.c_int(0)
        c = lib().or_modified_pm(self.h, cf, seed, max_itn, _p(fw), _p(uw), ctypes.byref(itn))
        return c, fw, uw, itn.value


class MMA:
    """The reference MMA (mma_t) restated in FP64 on the CPU."""

    def __init__(self, n, m, xmin, xmax):
        self.n, self.m = n, m
        xmin = np.broadcast_to(np.asarray(xmin, np.float64), (n,)).copy()
        xmax = np.broadcast_to(np.asarray(xmax, np.float64), (n,)).copy()
        self.h = lib().or_mma_create(n, m, _p(xmin), _p(xmax))

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_mma_destroy(self.h)
            self.h = None

    def set_x(self, x):
        lib().or_mma_set_x(self.h, _p(np.ascontiguousarray(x, np.float64)))

    def get(self):
        x, L, U, a, b = [np.zeros(self.n) for _ in range(5)]
        lib().or_mma_get(self.h, _p(x), _p(L), _p(U), _p(a), _p(b))
        return x, L, U, a, b

    def update(self, df, dg, g):
        info = np.zeros(4)
        conv = lib().or_mma_update(self.h, _p(np.ascontiguousarray(df, np.float64)),
                                   _p(np.ascontiguousarray(dg, np.float64).ravel()),
                                   _p(np.ascontiguousarray(g, np.float64)), _p(info))
        return bool(conv), info
