"""ctypes binding of librso.so and a Python mirror of the reference's
Grid / optimization / mma_t call surface.

Device arrays are torch CUDA tensors (PyTorch is only the allocator and
stream plumbing here); the arithmetic runs in librso's CUDA kernels.
Names follow the reference:

  HierarchyGrid.genFromMesh      -> rso_create            (grid/Grid.cpp:978)
  HierarchyGrid.update_stencil   -> rso_update_operators  (grid/Grid.cpp:4250)
  Grid.applyK / update_residual  -> rso_apply_K / rso_residual
  HierarchyGrid.v_cycle          -> rso_vcycle            (grid/Grid.cpp:2431)
  computeSensitivity             -> rso_sensitivity       (optimization/optimization.cu:191)
  projectDensities               -> rso_heaviside         (optimization/optimization.cu:350)
  Grid.filterSensitivity         -> rso_filter            (grid/Grid.cu:4298)
  Grid.coeff2density             -> rso_coeff2density     (grid/Grid.cu:3441)
  Grid.ddensity2dcoeff           -> rso_density2coeff_adjoint (grid/Grid.cu:3566)
  deal_background_points         -> rso_selfsupport       (optimization/optimization.cpp:1223)
  deal_surface_points            -> rso_surface_points + rso_surface_selfsupport
                                                          (optimization/optimization.cpp:1185)
  forceProject / modifiedPM      -> rso_force_project / rso_modified_pm / rso_worst_case
  MMA::mma_t::update             -> rso_mma_update        (optimization/mma_t.cpp:18)
"""
import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_NAME = "librso.so"


def library_path():
    return os.path.join(_HERE, _LIB_NAME)


class RSOError(RuntimeError):
    pass


class _Config(ctypes.Structure):
    _fields_ = [("youngs_modulus", ctypes.c_double), ("poisson_ratio", ctypes.c_double),
                ("penal", ctypes.c_double), ("rho_min", ctypes.c_double), ("n_levels", ctypes.c_int),
                ("first_factor", ctypes.c_int), ("smoother", ctypes.c_int), ("omega", ctypes.c_double),
                ("pre", ctypes.c_int), ("post", ctypes.c_int), ("precision", ctypes.c_int), ("mode", ctypes.c_int),
                ("cheb_lower", ctypes.c_double)]


class _SolveInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("rel_res", ctypes.c_double), ("ms", ctypes.c_double)]


class _IterParams(ctypes.Structure):
    _fields_ = [("beta", ctypes.c_double), ("volume_ratio", ctypes.c_double), ("filter_radius", ctypes.c_double),
                ("filter_mode", ctypes.c_int), ("lanczos_steps", ctypes.c_int), ("solve_tol", ctypes.c_double),
                ("constrain_direction", ctypes.c_int), ("ss_mode", ctypes.c_int), ("opt_angle", ctypes.c_double),
                ("default_angle", ctypes.c_double), ("sens_scale", ctypes.c_double), ("vol_scale", ctypes.c_double),
                ("ss_scale", ctypes.c_double), ("seed", ctypes.c_uint64), ("ss_points", ctypes.c_int),
                ("ss_mc_res", ctypes.c_int)]


class _IterInfo(ctypes.Structure):
    _fields_ = [("c_worst", ctypes.c_double), ("lam", ctypes.c_double), ("volume", ctypes.c_double),
                ("ss_value", ctypes.c_double), ("ms_total", ctypes.c_double), ("ms_operators", ctypes.c_double),
                ("ms_worst", ctypes.c_double), ("ms_adjoint", ctypes.c_double), ("ms_selfsupport", ctypes.c_double),
                ("ms_mma", ctypes.c_double), ("solve_iterations", ctypes.c_int), ("mma_converged", ctypes.c_int)]


class _SurfaceInfo(ctypes.Structure):
    _fields_ = [("n_crossings", ctypes.c_longlong), ("n_first_pick", ctypes.c_longlong),
                ("n_in_model", ctypes.c_longlong), ("n_points", ctypes.c_int), ("reserved", ctypes.c_int)]


class _Region(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("closed", ctypes.c_int), ("complement", ctypes.c_int),
                ("reserved", ctypes.c_int), ("p", ctypes.c_double * 8)]


class _Field(ctypes.Structure):
    _fields_ = [("region", _Region), ("norm_kind", ctypes.c_int), ("dir_kind", ctypes.c_int),
                ("norm_p", ctypes.c_double * 7), ("dir_p", ctypes.c_double * 6)]


_vp = ctypes.c_void_p
_ci = ctypes.c_int
_cd = ctypes.c_double
_pd = ctypes.POINTER(ctypes.c_double)
_pi = ctypes.POINTER(ctypes.c_int)
_pu8 = ctypes.POINTER(ctypes.c_uint8)
_pu32 = ctypes.POINTER(ctypes.c_uint32)

# every entry point of include/rso.h with its ctypes signature
SIGNATURES = {
    "rso_default_config": (None, [ctypes.POINTER(_Config)]),
    "rso_create": (_ci, [ctypes.POINTER(_Config), _ci, _ci, _ci, _pu8, _pu8, _pu8, _pd, ctypes.POINTER(_vp)]),
    "rso_destroy": (None, [_vp]),
    "rso_last_error": (ctypes.c_char_p, [_vp]),
    "rso_set_stream": (_ci, [_vp, _vp]),
    "rso_synchronize": (_ci, [_vp]),
    "rso_element_matrix": (_ci, [_cd, _cd, _cd, _pd]),
    "rso_n_levels": (_ci, [_vp]),
    "rso_level_dims": (_ci, [_vp, _ci, _pi]),
    "rso_level_masks": (_ci, [_vp, _ci, _pu8, _pu8]),
    "rso_level_bitwords": (_ci, [_vp, _ci, _pu32, _pu32]),
    "rso_bitsat_rank": (_ci, [_vp, _vp, ctypes.c_int64, _vp]),
    "rso_node_class": (_ci, [_vp, _pu8]),
    "rso_ref_numbering": (_ci, [_vp, _ci, _pi, _pi, _pi, _pi, _pi, _pi]),
    "rso_load_nodes": (_ci, [_vp, _pi, _pi]),
    "rso_set_density": (_ci, [_vp, _vp]),
    "rso_update_operators": (_ci, [_vp]),
    "rso_apply_K": (_ci, [_vp, _vp, _vp]),
    "rso_residual": (_ci, [_vp, _vp, _vp, _vp]),
    "rso_fine_sweep_fp32": (_ci, [_vp, _ci, _vp, _vp, _vp, ctypes.c_double, ctypes.c_double, _vp]),
    "rso_set_vcycle_graphs": (_ci, [_vp, _ci]),
    "rso_set_solve_graphs": (_ci, [_vp, _ci]),
    "rso_set_fine_zchunk": (_ci, [_vp, _ci]),
    "rso_fine_zchunk": (_ci, [_vp]),
    "rso_set_bottom_kernel": (_ci, [_vp, _ci]),
    "rso_bottom_kernel": (_ci, [_vp]),
    "rso_grid_barrier_selftest": (_ci, [_vp, _ci, _cd, _pi]),
    "rso_set_krylov_fp32": (_ci, [_vp, _cd]),
    "rso_set_krylov_fp32_cycles": (_ci, [_vp, _ci]),
    "rso_displacement_project": (_ci, [_vp, _vp]),
    "rso_get_density": (_ci, [_vp, _vp]),
    "rso_set_density_points": (_ci, [_vp, _ci, _pi, ctypes.POINTER(ctypes.c_float)]),
    "rso_voxelize": (_ci, [ctypes.POINTER(ctypes.c_float), _ci, ctypes.POINTER(ctypes.c_int), _ci, _ci, _pu8, _pi,
                           ctypes.POINTER(ctypes.c_float)]),
    "rso_shell_elements": (_ci, [ctypes.POINTER(ctypes.c_float), _ci, ctypes.POINTER(ctypes.c_int), _ci,
                                 ctypes.POINTER(ctypes.c_float), _ci, _cd, _pu8, _pu8]),
    "rso_mesh_normals": (_ci, [ctypes.POINTER(ctypes.c_float), _ci, ctypes.POINTER(ctypes.c_int), _ci, _pd, _ci,
                               _pd]),
    "rso_region_mask": (_ci, [ctypes.POINTER(_Region), _ci, _pd, _cd, _ci, _ci, _ci, _pu8]),
    "rso_region_field": (_ci, [ctypes.POINTER(_Field), _ci, _pd, _ci, _pd]),
    "rso_mma_state_size": (_ci, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    "rso_mma_save": (_ci, [_vp, _pd]),
    "rso_mma_load": (_ci, [_vp, _pd]),
    "rso_oc_update_density": (_ci, [_vp, _ci, _vp, _vp, _vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, _vp,
                                    _pd]),
    "rso_oc_update_coeff": (_ci, [_vp, _vp, _vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, _vp, _pd]),
    "rso_coarse_sweep_fp32": (_ci, [_vp, _ci, _ci, _vp, _vp, _vp, ctypes.c_double, ctypes.c_double, _vp]),
    "rso_prolong_fp32": (_ci, [_vp, _ci, _vp, _vp, _vp]),
    "rso_restrict_fp32": (_ci, [_vp, _ci, _vp, _vp]),
    "rso_autotune": (_ci, [_vp, _pi]),
    "rso_set_launch_shapes": (_ci, [_vp, _pi, _ci]),
    "rso_get_stencil": (_ci, [_vp, _ci, _vp]),
    "rso_coarse_residual": (_ci, [_vp, _ci, _vp, _vp, _vp]),
    "rso_smooth": (_ci, [_vp, _ci, _vp, _vp, _ci, _cd, _ci, _ci]),
    "rso_restrict": (_ci, [_vp, _ci, _vp, _vp]),
    "rso_prolong": (_ci, [_vp, _ci, _vp, _vp]),
    "rso_coarsest_solve": (_ci, [_vp, _vp, _vp]),
    "rso_level_lambda": (_ci, [_vp, _ci, _pd]),
    "rso_vcycle": (_ci, [_vp, _vp, _vp, _ci, _ci, _ci, _pd]),
    "rso_solve": (_ci, [_vp, _vp, _vp, _cd, _ci, _ci, ctypes.POINTER(_SolveInfo)]),
    "rso_solve_batch": (_ci, [_vp, _ci, _vp, _vp, _cd, _ci, ctypes.POINTER(_SolveInfo)]),
    "rso_dot": (_ci, [_vp, _vp, _vp, _pd]),
    "rso_sensitivity": (_ci, [_vp, _vp, _vp]),
    "rso_element_energy": (_ci, [_vp, _vp, _vp]),
    "rso_heaviside": (_ci, [_vp, _vp, _cd, _vp, _vp]),
    "rso_heaviside_chain": (_ci, [_vp, _vp, _cd, _vp, _vp]),
    "rso_filter": (_ci, [_vp, _cd, _vp, _vp]),
    "rso_density_filter": (_ci, [_vp, _cd, _vp, _vp]),
    "rso_density_filter_adjoint": (_ci, [_vp, _cd, _vp, _vp]),
    "rso_filter_noalloc": (_ci, [_vp, _cd, _vp, _vp]),
    "rso_volume": (_ci, [_vp, _vp, _pd]),
    "rso_spline_setup": (_ci, [_vp, _ci, _ci, _ci, _ci, _pi]),
    "rso_spline_axis": (_ci, [_vp, _ci, _pi, _pd, _pd]),
    "rso_coeff2density": (_ci, [_vp, _vp, _vp, _vp]),
    "rso_density2coeff_adjoint": (_ci, [_vp, _vp, _vp, _vp]),
    "rso_selfsupport": (_ci, [_vp, _vp, _cd, _ci, _cd, _cd, _vp, _vp, _pd, _pd, _pd]),
    "rso_surface_points": (_ci, [_vp, _vp, _ci, _ci, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(_SurfaceInfo)]),
    "rso_set_surface_points": (_ci, [_vp, _vp, _ci]),
    "rso_get_surface_points": (_ci, [_vp, _vp, _ci, _pi]),
    "rso_surface_selfsupport": (_ci, [_vp, _vp, _cd, _ci, _cd, _cd, _vp, _vp, _pd, _pd, _pd]),
    "rso_get_surface_normals": (_ci, [_vp, _vp, _vp]),
    "rso_force_project": (_ci, [_vp, _vp, _ci]),
    "rso_worst_case": (_ci, [_vp, _ci, _ci, _cd, ctypes.c_uint64, _vp, _vp, _pd, _pd]),
    "rso_modified_pm": (_ci, [_vp, _ci, ctypes.c_uint64, _ci, _vp, _vp, _pd, _pi]),
    "rso_mma_create": (_ci, [_ci, _ci, _pd, _pd, ctypes.POINTER(_vp)]),
    "rso_mma_set_x": (_ci, [_vp, _pd]),
    "rso_mma_set_x_dev": (_ci, [_vp, _vp]),
    "rso_mma_get": (_ci, [_vp, _pd, _pd, _pd, _pd, _pd]),
    "rso_mma_x_dev": (_vp, [_vp]),
    "rso_mma_update": (_ci, [_vp, _vp, _vp, _pd, _pi, _pd]),
    "rso_mma_destroy": (None, [_vp]),
    "rso_default_iter_params": (None, [ctypes.POINTER(_IterParams)]),
    "rso_design_iteration": (_ci, [_vp, _vp, ctypes.POINTER(_IterParams), ctypes.POINTER(_IterInfo)]),
    "rso_design_iteration_host": (_ci, [_vp, _vp, ctypes.POINTER(_IterParams), _pd, _pd,
                                        ctypes.POINTER(ctypes.c_float), ctypes.POINTER(_IterInfo)]),
    "rso_design_gradient": (_ci, [_vp, _vp, ctypes.POINTER(_IterParams), _pd, _vp, _vp, _vp]),
    "rso_launch_count": (ctypes.c_longlong, []),
    "rso_set_profiling": (_ci, [_vp, _ci]),
    "rso_set_profiling_classes": (_ci, [_vp, ctypes.c_uint]),
    "rso_profile_reset": (_ci, [_vp]),
    "rso_profile_class": (_ci, [_vp, _ci, ctypes.c_char_p, _ci, ctypes.POINTER(ctypes.c_longlong), _pd, _pd, _pd]),
    "rso_profile_top": (_ci, [_vp, ctypes.c_char_p, _ci, ctypes.POINTER(ctypes.c_longlong), _pd, _pd, _pd]),
}

_lib = None


class _StreamOrderedLib:
    """The library seen through the torch binding: before every call, torch's
    current CUDA stream is synchronised, so tensors produced there (fresh
    allocations, fills, copies) are complete when the library reads them on
    its own stream."""

    def __init__(self, lib):
        self._lib = lib

    def __getattr__(self, name):
        fn = getattr(self._lib, name)

        def call(*args):
            import torch
            if torch.cuda.is_initialized():
                torch.cuda.current_stream().synchronize()
            return fn(*args)

        return call


def load_library():
    """Load librso.so; raises if it has not been built (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise RSOError(f"{path} is missing: build it with `python -m robustoptspline3d_b200.build` "
                       "(the CUDA library is the only implementation)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


_STATUS = {0: "OK", 1: "INVALID_ARG", 2: "OOM", 3: "CUDA", 4: "DIVERGED", 5: "NONFINITE", 6: "BUDGET_EXCEEDED",
           7: "UNSUPPORTED", 8: "STATE"}

SMOOTH_GS, SMOOTH_JACOBI, SMOOTH_CHEBYSHEV = 0, 1, 2
FP64, MIXED = 0, 1
SOLVE_VCYCLE, SOLVE_PCG = 0, 1
NO_SUPPORT_CF, NO_SUPPORT_FF, WITH_SUPPORT_CF, WITH_SUPPORT_FF = 0, 1, 2, 3


def _np_ptr(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def _dev(t, dtype=None):
    """Device pointer of a contiguous CUDA tensor (None -> NULL)."""
    if t is None:
        return None
    if not t.is_cuda:
        raise RSOError("expected a CUDA tensor")
    if dtype is not None and t.dtype != dtype:
        raise RSOError(f"expected {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise RSOError("expected a contiguous tensor")
    return ctypes.c_void_p(t.data_ptr())


def element_matrix(E=1e6, nu=0.3, h=1.0):
    out = np.zeros(576)
    st = load_library().rso_element_matrix(E, nu, h, _np_ptr(out, _pd))
    if st:
        raise RSOError(f"rso_element_matrix: {_STATUS.get(st, st)}")
    return out.reshape(24, 24)


@dataclass
class Config:
    youngs_modulus: float = 1e6
    poisson_ratio: float = 0.3
    penal: float = 3.0
    rho_min: float = 1e-3
    n_levels: int = 0
    first_factor: int = 4
    smoother: int = SMOOTH_JACOBI
    omega: float = 0.6
    pre: int = 2
    post: int = 2
    precision: int = MIXED
    mode: int = WITH_SUPPORT_FF
    cheb_lower: float = 0.25

    def _c(self):
        c = _Config()
        for f in _Config._fields_:
            setattr(c, f[0], getattr(self, f[0]))
        return c


@dataclass
class IterParams:
    beta: float = 8.0
    volume_ratio: float = 0.3
    filter_radius: float = 2.0
    filter_mode: int = 0
    lanczos_steps: int = 20
    solve_tol: float = 1e-6
    constrain_direction: int = 0
    ss_mode: int = 4
    opt_angle: float = 0.75 * np.pi
    default_angle: float = 0.75 * np.pi
    sens_scale: float = 1e6
    vol_scale: float = 1e3
    ss_scale: float = 1e3
    seed: int = 1234
    ss_points: int = 0       # > 0: the self-support constraint on that many surface points
    ss_mc_res: int = 64

    def _c(self):
        c = _IterParams()
        for f in _IterParams._fields_:
            setattr(c, f[0], getattr(self, f[0]))
        return c


class HierarchyGrid:
    """The multigrid hierarchy and fine-level design state of one voxel box.

    Arrays: nodal vectors are float64 CUDA tensors of shape (3, nz+1, ny+1, nx+1)
    (or flat 3*Nn); element fields float32 of shape (ez, ey, ex) or flat.
    """

    def __init__(self, emask, fixed_area, load_area, load_normals=None, config=None):
        import torch  # noqa: F401  (CUDA context / allocator)
        self.lib = _StreamOrderedLib(load_library())
        self.cfg = config or Config()
        emask = np.ascontiguousarray(emask, dtype=np.uint8)
        self.ez, self.ey, self.ex = emask.shape
        self.nx, self.ny, self.nz = self.ex + 1, self.ey + 1, self.ez + 1
        self.nn = self.nx * self.ny * self.nz
        self.ne = self.ex * self.ey * self.ez
        self._emask = emask
        fa = np.ascontiguousarray(fixed_area, dtype=np.uint8).ravel()
        la = np.ascontiguousarray(load_area, dtype=np.uint8).ravel()
        ln = None if load_normals is None else np.ascontiguousarray(load_normals, dtype=np.float64).ravel()
        h = ctypes.c_void_p()
        c = self.cfg._c()
        st = self.lib.rso_create(ctypes.byref(c), self.ex, self.ey, self.ez, _np_ptr(emask.ravel(), _pu8),
                                 _np_ptr(fa, _pu8), _np_ptr(la, _pu8), _np_ptr(ln, _pd), ctypes.byref(h))
        if st:
            raise RSOError(f"rso_create: {_STATUS.get(st, st)}: {self.lib.rso_last_error(None).decode()}")
        self.h = h
        self.n_coeff = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.rso_destroy(self.h)
            self.h = None

    def __del__(self):
        # at interpreter shutdown the stream-ordering wrapper may no longer
        # import what it needs; the process exit releases the device memory
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, st, what):
        if st:
            raise RSOError(f"{what}: {_STATUS.get(st, st)}: {self.lib.rso_last_error(self.h).decode()}")

    # ------------------------------------------------------------ topology
    def n_levels(self):
        return self.lib.rso_n_levels(self.h)

    def level_dims(self, level):
        d = np.zeros(6, dtype=np.int32)
        self._chk(self.lib.rso_level_dims(self.h, level, _np_ptr(d, _pi)), "rso_level_dims")
        return d

    def level_masks(self, level):
        d = self.level_dims(level)
        em = np.zeros(int(d[0] * d[1] * d[2]), np.uint8)
        vm = np.zeros(int(d[3] * d[4] * d[5]), np.uint8)
        self._chk(self.lib.rso_level_masks(self.h, level, _np_ptr(em, _pu8), _np_ptr(vm, _pu8)), "rso_level_masks")
        return em, vm

    def level_bitwords(self, level):
        d = self.level_dims(level)
        eb = np.zeros((int(d[0] * d[1] * d[2]) + 31) // 32, np.uint32)
        vb = np.zeros((int(d[3] * d[4] * d[5]) + 31) // 32, np.uint32)
        self._chk(self.lib.rso_level_bitwords(self.h, level, _np_ptr(eb, _pu32), _np_ptr(vb, _pu32)), "bitwords")
        return eb, vb

    def bitsat_rank(self, words, nbits):
        import torch
        w = torch.as_tensor(np.asarray(words, np.uint32).view(np.int32), device="cuda")
        out = torch.empty(nbits, dtype=torch.int32, device="cuda")
        self._chk(self.lib.rso_bitsat_rank(self.h, _dev(w), nbits, _dev(out)), "rso_bitsat_rank")
        return out.cpu().numpy()

    def node_class(self):
        out = np.zeros(self.nn, np.uint8)
        self._chk(self.lib.rso_node_class(self.h, _np_ptr(out, _pu8)), "rso_node_class")
        return out

    def ref_numbering(self, level):
        counts = np.zeros(4, np.int32)
        gs = np.zeros(8, np.int32)
        self._chk(self.lib.rso_ref_numbering(self.h, level, _np_ptr(counts, _pi), _np_ptr(gs, _pi), None, None, None,
                                             None), "rso_ref_numbering")
        nv, ne, nvgs, negs = [int(v) for v in counts]
        vl, el = np.zeros(nv, np.int32), np.zeros(ne, np.int32)
        vf, ef = np.zeros(nvgs, np.int32), np.zeros(negs, np.int32)
        self._chk(self.lib.rso_ref_numbering(self.h, level, None, None, _np_ptr(vl, _pi), _np_ptr(el, _pi),
                                             _np_ptr(vf, _pi), _np_ptr(ef, _pi)), "rso_ref_numbering")
        return dict(counts=counts, gs_num=gs, vlexi2gs=vl, elexi2gs=el, vflag=vf, eflag=ef)

    def load_nodes(self):
        n = ctypes.c_int(0)
        self._chk(self.lib.rso_load_nodes(self.h, None, ctypes.byref(n)), "rso_load_nodes")
        out = np.zeros(max(n.value, 1), np.int32)
        self._chk(self.lib.rso_load_nodes(self.h, _np_ptr(out, _pi), ctypes.byref(n)), "rso_load_nodes")
        return out[:n.value]

    # ------------------------------------------------------------ operator
    def set_density(self, rho):
        import torch
        r = rho if isinstance(rho, torch.Tensor) else torch.as_tensor(np.asarray(rho, np.float32), device="cuda")
        r = r.to(device="cuda", dtype=torch.float32).contiguous()
        self._chk(self.lib.rso_set_density(self.h, _dev(r)), "rso_set_density")

    def get_density(self):
        """The current element densities (float32 CUDA tensor, ez x ey x ex flattened)."""
        import torch
        out = torch.empty(self.ne, dtype=torch.float32, device="cuda")
        self._chk(self.lib.rso_get_density(self.h, _dev(out)), "rso_get_density")
        return out

    def writeDensity(self, prefix):
        """Save the densities of the active elements as HierarchyGrid::writeDensity does
        (grid/Grid.cpp:1267-1300), as raw records instead of OpenVDB: see records.write_density."""
        from . import records
        records.write_density(prefix, self._emask, self.get_density().cpu().numpy())

    def readDensity(self, prefix):
        """Restart from densities saved by writeDensity (HierarchyGrid::readDensity,
        grid/Grid.cpp:1914-1945); call update_stencil next."""
        from . import records
        pos, val = records.read_density(prefix)
        pos = np.ascontiguousarray(pos, np.int32)
        val = np.ascontiguousarray(val, np.float32)
        self._chk(self.lib.rso_set_density_points(self.h, len(val), _np_ptr(pos, _pi),
                                                  val.ctypes.data_as(ctypes.POINTER(ctypes.c_float))),
                  "rso_set_density_points")

    def update_stencil(self):
        self._chk(self.lib.rso_update_operators(self.h), "rso_update_operators")

    def _vec(self, level=0):
        import torch
        d = self.level_dims(level)
        return torch.zeros(3 * int(d[3] * d[4] * d[5]), dtype=torch.float64, device="cuda")

    def applyK(self, u):
        import torch
        f = torch.empty_like(u)
        self._chk(self.lib.rso_apply_K(self.h, _dev(u, torch.float64), _dev(f)), "rso_apply_K")
        return f

    def update_residual(self, u, f):
        import torch
        r = torch.empty_like(u)
        self._chk(self.lib.rso_residual(self.h, _dev(u, torch.float64), _dev(f, torch.float64), _dev(r)), "rso_residual")
        return r

    def autotune(self):
        """Time the launch-shape alternatives on this hierarchy and keep the fastest
        (rso_autotune); returns the choices."""
        c = np.zeros(2 + self.n_levels(), np.int32)
        self._chk(self.lib.rso_autotune(self.h, _np_ptr(c, _pi)), "rso_autotune")
        self._shapes = {"fine_rows": int(c[0]), "fine_zchunk": self.fine_zchunk(), "bottom_level": int(c[1]),
                        "bottom_kernel": self.bottom_kernel(), "row_split": [int(x) for x in c[2:]]}
        return dict(self._shapes)

    def launch_shapes(self):
        """The launch shapes last chosen by autotune() or set_launch_shapes() (the
        built-in rules' markers when neither ran)."""
        sh = getattr(self, "_shapes", None)
        if sh is None:
            sh = {"fine_rows": 4, "fine_zchunk": self.fine_zchunk(), "bottom_level": -2,
                  "bottom_kernel": self.bottom_kernel(), "row_split": [-1] * self.n_levels()}
        return dict(sh)

    def set_launch_shapes(self, fine_rows=4, bottom_level=-2, row_split=None):
        """Launch shapes in rso_autotune's terms (rso_set_launch_shapes)."""
        rs = list(row_split or [])
        c = np.array([fine_rows, bottom_level] + rs, np.int32)
        self._chk(self.lib.rso_set_launch_shapes(self.h, _np_ptr(c, _pi), len(c)), "rso_set_launch_shapes")
        nl = self.n_levels()
        self._shapes = {"fine_rows": int(fine_rows), "fine_zchunk": self.fine_zchunk(), "bottom_level": int(bottom_level),
                        "bottom_kernel": self.bottom_kernel(),
                        "row_split": [int(x) for x in rs[:nl]] + [-1] * max(0, nl - len(rs))}

    def updateDensities(self, rho, sens, vgoal, step=0.1, damp=0.5, shell=None, variant=0):
        """OC density update (rso_oc_update_density): returns (new rho, info dict)."""
        import torch
        src = self._efield(rho)
        out = torch.empty_like(src)
        info = np.zeros(5)
        sh = None if shell is None else torch.as_tensor(np.asarray(shell, np.uint8).ravel(), device="cuda")
        self._chk(self.lib.rso_oc_update_density(self.h, variant, _dev(src), _dev(self._efield(sens)), _dev(sh), vgoal,
                                                 step, damp, _dev(out), _np_ptr(info, _pd)), "rso_oc_update_density")
        return out, {"g": info[0], "volume": info[1], "trials": int(info[2]), "max_change": info[3],
                     "mean_change": info[4]}

    def updateCoeff(self, coeff, csens, vgoal, step=0.1, damp=0.5, cmin=0.0, cmax=1.0):
        """OC coefficient update (rso_oc_update_coeff): returns (new coefficients, densities, info dict)."""
        import torch
        c = torch.as_tensor(np.asarray(coeff, np.float32) if not isinstance(coeff, torch.Tensor) else coeff,
                            device="cuda").to(torch.float32).contiguous().clone()
        cs = torch.as_tensor(np.asarray(csens, np.float32) if not isinstance(csens, torch.Tensor) else csens,
                             device="cuda").to(torch.float32).contiguous()
        rho = torch.empty(self.ne, dtype=torch.float32, device="cuda")
        info = np.zeros(3)
        self._chk(self.lib.rso_oc_update_coeff(self.h, _dev(c), _dev(cs), vgoal, step, damp, cmin, cmax, _dev(rho),
                                               _np_ptr(info, _pd)), "rso_oc_update_coeff")
        return c, rho, {"g": info[0], "volume": info[1], "trials": int(info[2])}

    def set_krylov_fp32(self, replace_factor=1e-2):
        """Mixed precision: run the PCG recurrence in FP32 with true-residual replacement
        whenever the residual has dropped by replace_factor (0 restores the FP64 recurrence)."""
        self._chk(self.lib.rso_set_krylov_fp32(self.h, float(replace_factor)), "rso_set_krylov_fp32")

    def set_krylov_fp32_cycles(self, max_cycles=0):
        """Mixed precision: hand the solve over to the FP64 recurrence after max_cycles
        residual replacements of the FP32 recurrence (0: only when it stalls)."""
        self._chk(self.lib.rso_set_krylov_fp32_cycles(self.h, int(max_cycles)), "rso_set_krylov_fp32_cycles")

    def set_vcycle_graphs(self, on):
        """Replay captured FP32 V-cycles from CUDA graphs (default) or launch every kernel."""
        self._chk(self.lib.rso_set_vcycle_graphs(self.h, 1 if on else 0), "rso_set_vcycle_graphs")

    def set_fine_zchunk(self, planes=0):
        """Node planes per z chunk of the FP32 fine kernel (4, 8, 16, 32; 0: by size)."""
        self._chk(self.lib.rso_set_fine_zchunk(self.h, int(planes)), "rso_set_fine_zchunk")

    def fine_zchunk(self):
        return int(self.lib.rso_fine_zchunk(self.h))

    def set_bottom_kernel(self, kind):
        """Bottom of the FP32 V-cycle: 1 persistent grid-wide kernel, 0 8-CTA cluster kernel."""
        self._chk(self.lib.rso_set_bottom_kernel(self.h, int(kind)), "rso_set_bottom_kernel")

    def bottom_kernel(self):
        return int(self.lib.rso_bottom_kernel(self.h))

    def grid_barrier_selftest(self, short_by=0, limit_ms=10.0):
        """Bounded-wait self-test of the persistent kernel's grid barrier: 1 if a wait gave up."""
        out = ctypes.c_int(0)
        self._chk(self.lib.rso_grid_barrier_selftest(self.h, int(short_by), float(limit_ms), ctypes.byref(out)),
                  "rso_grid_barrier_selftest")
        return int(out.value)

    def set_solve_graphs(self, on):
        """Run the mixed PCG loop as one device-controlled CUDA graph per solve."""
        self._chk(self.lib.rso_set_solve_graphs(self.h, 1 if on else 0), "rso_set_solve_graphs")

    def fine_sweep_fp32(self, op, u, f=None, uprev=None, omega=1.0, c1=0.0):
        """One FP32 fine-level sweep (op 0 residual, 1 K u, 2 Jacobi/Chebyshev step), FP64 in and out."""
        import torch
        out = torch.empty_like(u)
        self._chk(self.lib.rso_fine_sweep_fp32(self.h, op, _dev(u, torch.float64),
                                               None if f is None else _dev(f, torch.float64),
                                               None if uprev is None else _dev(uprev, torch.float64),
                                               omega, c1, _dev(out)), "rso_fine_sweep_fp32")
        return out

    def coarse_sweep_fp32(self, level, op, u, f, uprev=None, omega=1.0, c1=0.0):
        """One FP32 coarse-level sweep (op 0 residual, 2 Jacobi/Chebyshev step), FP64 in and out."""
        import torch
        out = torch.empty_like(u)
        self._chk(self.lib.rso_coarse_sweep_fp32(self.h, level, op, _dev(u, torch.float64), _dev(f, torch.float64),
                                                 _dev(uprev, torch.float64) if uprev is not None else None,
                                                 omega, c1, _dev(out)), "rso_coarse_sweep_fp32")
        return out

    def prolong_fp32(self, coarse_level, uc, uf):
        """uf + P uc in FP32 (the mixed V-cycle's prolongation), FP64 in and out."""
        import torch
        out = torch.empty_like(uf)
        self._chk(self.lib.rso_prolong_fp32(self.h, coarse_level, _dev(uc, torch.float64), _dev(uf, torch.float64),
                                            _dev(out)), "rso_prolong_fp32")
        return out

    def restrict_fp32(self, coarse_level, rf):
        """R rf in FP32 (the mixed V-cycle's restriction), FP64 in and out."""
        import torch
        d = self.level_dims(coarse_level)
        out = torch.empty(3 * int(d[3] * d[4] * d[5]), dtype=torch.float64, device="cuda")
        self._chk(self.lib.rso_restrict_fp32(self.h, coarse_level, _dev(rf, torch.float64), _dev(out)),
                  "rso_restrict_fp32")
        return out

    def stencil(self, level):
        import torch
        d = self.level_dims(level)
        nn = int(d[3] * d[4] * d[5])
        out = torch.empty(243 * nn, dtype=torch.float64, device="cuda")
        self._chk(self.lib.rso_get_stencil(self.h, level, _dev(out)), "rso_get_stencil")
        return out.view(27, 3, 3, nn)

    def coarse_residual(self, level, u, f):
        import torch
        r = torch.empty_like(u)
        self._chk(self.lib.rso_coarse_residual(self.h, level, _dev(u, torch.float64), _dev(f, torch.float64), _dev(r)),
                  "rso_coarse_residual")
        return r

    def gs_relax(self, level, u, f, kind=SMOOTH_GS, omega=1.0, sweeps=1, reverse=0):
        import torch
        u = u.clone()
        self._chk(self.lib.rso_smooth(self.h, level, _dev(u, torch.float64), _dev(f, torch.float64), kind, omega, sweeps,
                                      reverse), "rso_smooth")
        return u

    def restrict_residual(self, coarse_level, rf):
        import torch
        fc = self._vec(coarse_level)
        self._chk(self.lib.rso_restrict(self.h, coarse_level, _dev(rf, torch.float64), _dev(fc)), "rso_restrict")
        return fc

    def prolongate_correction(self, coarse_level, uc, uf):
        import torch
        uf = uf.clone()
        self._chk(self.lib.rso_prolong(self.h, coarse_level, _dev(uc, torch.float64), _dev(uf)), "rso_prolong")
        return uf

    def solve_coarsest(self, f):
        import torch
        u = torch.empty_like(f)
        self._chk(self.lib.rso_coarsest_solve(self.h, _dev(f, torch.float64), _dev(u)), "rso_coarsest_solve")
        return u

    def level_lambda(self, level):
        v = ctypes.c_double(0)
        self._chk(self.lib.rso_level_lambda(self.h, level, ctypes.byref(v)), "rso_level_lambda")
        return v.value

    def v_cycle(self, u, f, pre=1, post=1, symmetric=0):
        import torch
        u = u.clone()
        rr = ctypes.c_double(0)
        self._chk(self.lib.rso_vcycle(self.h, _dev(u, torch.float64), _dev(f, torch.float64), pre, post, symmetric,
                                      ctypes.byref(rr)), "rso_vcycle")
        return u, rr.value

    def solve(self, f, u0=None, tol=1e-10, max_iter=200, method=SOLVE_PCG):
        import torch
        u = torch.zeros_like(f) if u0 is None else u0.clone()
        info = _SolveInfo()
        self._chk(self.lib.rso_solve(self.h, _dev(f, torch.float64), _dev(u), tol, max_iter, method, ctypes.byref(info)),
                  "rso_solve")
        return u, info.iterations, info.rel_res, info.ms

    def solve_batch(self, F, U0=None, tol=1e-10, max_iter=200):
        """k systems at once: F (k, 3*Nn) float64 CUDA tensor; returns U (k, 3*Nn)
        and per-system (iterations, rel_res)."""
        import torch
        F = F.reshape(F.shape[0], -1).contiguous()
        k = F.shape[0]
        U = torch.zeros_like(F) if U0 is None else U0.reshape(k, -1).clone().contiguous()
        infos = (_SolveInfo * k)()
        self._chk(self.lib.rso_solve_batch(self.h, k, _dev(F, torch.float64), _dev(U, torch.float64), tol, max_iter,
                                           infos), "rso_solve_batch")
        return U, [(infos[b].iterations, infos[b].rel_res) for b in range(k)]

    def compliance(self, f, u):
        v = ctypes.c_double(0)
        self._chk(self.lib.rso_dot(self.h, _dev(f), _dev(u), ctypes.byref(v)), "rso_dot")
        return v.value

    # ------------------------------------------------------------ design variables
    def _efield(self, x):
        import torch
        x = x if isinstance(x, torch.Tensor) else torch.as_tensor(np.asarray(x, np.float32))
        return x.to(device="cuda", dtype=torch.float32).contiguous().view(-1)

    def _shell(self, shell):
        import torch
        if shell is None:
            return None
        return torch.as_tensor(np.ascontiguousarray(shell, np.uint8).ravel(), device="cuda")

    def computeSensitivity(self, u):
        import torch
        out = torch.empty(self.ne, dtype=torch.float32, device="cuda")
        self._chk(self.lib.rso_sensitivity(self.h, _dev(u, torch.float64), _dev(out)), "rso_sensitivity")
        return out

    def elementCompliance(self, u):
        import torch
        out = torch.empty(self.ne, dtype=torch.float32, device="cuda")
        self._chk(self.lib.rso_element_energy(self.h, _dev(u, torch.float64), _dev(out)), "rso_element_energy")
        return out

    def projectDensities(self, rho, beta, shell=None):
        import torch
        rho = self._efield(rho)
        sh = self._shell(shell)
        out = torch.empty_like(rho)
        self._chk(self.lib.rso_heaviside(self.h, _dev(rho), beta, _dev(sh), _dev(out)), "rso_heaviside")
        return out

    def projectSensitivity(self, rho, beta, g):
        import torch
        rho, g = self._efield(rho), self._efield(g)
        out = torch.empty_like(g)
        self._chk(self.lib.rso_heaviside_chain(self.h, _dev(rho), beta, _dev(g), _dev(out)), "rso_heaviside_chain")
        return out

    def filterSensitivity(self, radius, g):
        import torch
        g = self._efield(g)
        out = torch.empty_like(g)
        self._chk(self.lib.rso_filter(self.h, radius, _dev(g), _dev(out)), "rso_filter")
        return out

    def densityFilter(self, radius, x, adjoint=False):
        import torch
        x = self._efield(x)
        out = torch.empty_like(x)
        fn = self.lib.rso_density_filter_adjoint if adjoint else self.lib.rso_density_filter
        self._chk(fn(self.h, radius, _dev(x), _dev(out)), "rso_density_filter")
        return out

    def volumeRatio(self, rho):
        v = ctypes.c_double(0)
        self._chk(self.lib.rso_volume(self.h, _dev(self._efield(rho)), ctypes.byref(v)), "rso_volume")
        return v.value

    def set_spline_partition(self, px, py, pz, order):
        n = ctypes.c_int(0)
        self._chk(self.lib.rso_spline_setup(self.h, order, px, py, pz, ctypes.byref(n)), "rso_spline_setup")
        self.n_coeff = n.value
        self.order = order
        return n.value

    def spline_axis(self, axis):
        n = [self.ex, self.ey, self.ez][axis]
        idx = np.zeros(n, np.int32)
        N = np.zeros(n * self.order)
        dN = np.zeros(n * self.order)
        self._chk(self.lib.rso_spline_axis(self.h, axis, _np_ptr(idx, _pi), _np_ptr(N, _pd), _np_ptr(dN, _pd)),
                  "rso_spline_axis")
        return idx, N.reshape(n, self.order), dN.reshape(n, self.order)

    def coeff2density(self, coeff, shell=None):
        import torch
        c = self._efield(coeff)
        out = torch.empty(self.ne, dtype=torch.float32, device="cuda")
        self._chk(self.lib.rso_coeff2density(self.h, _dev(c), _dev(self._shell(shell)), _dev(out)), "rso_coeff2density")
        return out

    def ddensity2dcoeff(self, g, shell=None):
        import torch
        g = self._efield(g)
        out = torch.empty(self.n_coeff, dtype=torch.float32, device="cuda")
        self._chk(self.lib.rso_density2coeff_adjoint(self.h, _dev(g), _dev(self._shell(shell)), _dev(out)),
                  "rso_density2coeff_adjoint")
        return out

    def deal_background_points(self, coeff, beta, mode=4, opt_angle=0.75 * np.pi, default_angle=0.75 * np.pi):
        import torch
        c = self._efield(coeff)
        per = torch.empty(self.ne, dtype=torch.float32, device="cuda")
        dc = torch.empty(self.n_coeff, dtype=torch.float32, device="cuda")
        val, cnt, ds = ctypes.c_double(0), ctypes.c_double(0), ctypes.c_double(0)
        self._chk(self.lib.rso_selfsupport(self.h, _dev(c), beta, mode, opt_angle, default_angle, _dev(per), _dev(dc),
                                           ctypes.byref(val), ctypes.byref(cnt), ctypes.byref(ds)), "rso_selfsupport")
        return val.value, per, dc, cnt.value, ds.value

    # ------------------------------------------------------------ surface-point self-support
    def generate_spline_surface_nodes(self, coeff, mc_res=64, n_points=200000, model_box=None):
        """Sample rho = 0.5 of the spline design (Grid::generate_spline_surface_nodes,
        grid/Grid.cpp:4067-4112); the points stay on the handle.  Returns the
        points, a (3, n) CUDA tensor, and the sampling counts."""
        c = self._efield(coeff)
        box = None
        if model_box is not None:
            box = np.ascontiguousarray(model_box, np.float32)
            if box.size != 6:
                raise RSOError("model_box holds xmin, ymin, zmin, xmax, ymax, zmax")
        info = _SurfaceInfo()
        self._chk(self.lib.rso_surface_points(self.h, _dev(c), int(mc_res), int(n_points),
                                              _np_ptr(box, ctypes.POINTER(ctypes.c_float)), ctypes.byref(info)),
                  "rso_surface_points")
        counts = dict(n_crossings=info.n_crossings, n_first_pick=info.n_first_pick, n_in_model=info.n_in_model,
                      n_points=info.n_points)
        return self.surface_points(), counts

    def uploadSurfacePoints(self, xyz):
        """Use the given points (3, n) for the surface constraint."""
        import torch
        x = xyz if isinstance(xyz, torch.Tensor) else torch.as_tensor(np.asarray(xyz, np.float32))
        x = x.to(device="cuda", dtype=torch.float32).contiguous()
        n = x.numel() // 3
        self._chk(self.lib.rso_set_surface_points(self.h, _dev(x.view(-1)), n), "rso_set_surface_points")

    def surface_points(self):
        import torch
        n = ctypes.c_int(0)
        self._chk(self.lib.rso_get_surface_points(self.h, None, 0, ctypes.byref(n)), "rso_get_surface_points")
        out = torch.empty(3 * n.value, dtype=torch.float32, device="cuda")
        if n.value:
            self._chk(self.lib.rso_get_surface_points(self.h, _dev(out), n.value, ctypes.byref(n)),
                      "rso_get_surface_points")
        return out.view(3, -1)

    def deal_surface_points(self, coeff, beta, mode=4, opt_angle=0.75 * np.pi, default_angle=0.75 * np.pi):
        """The constraint at the handle's surface points (grid/Grid.cu:5709-6505):
        (value, per-point values, dvalue/dcoeff, count, probe sum)."""
        import torch
        c = self._efield(coeff)
        n = ctypes.c_int(0)
        self._chk(self.lib.rso_get_surface_points(self.h, None, 0, ctypes.byref(n)), "rso_get_surface_points")
        per = torch.empty(max(n.value, 1), dtype=torch.float32, device="cuda")
        dc = torch.empty(self.n_coeff, dtype=torch.float32, device="cuda")
        val, cnt, ds = ctypes.c_double(0), ctypes.c_double(0), ctypes.c_double(0)
        self._chk(self.lib.rso_surface_selfsupport(self.h, _dev(c), beta, mode, opt_angle, default_angle, _dev(per),
                                                   _dev(dc), ctypes.byref(val), ctypes.byref(cnt), ctypes.byref(ds)),
                  "rso_surface_selfsupport")
        return val.value, per[:n.value], dc, cnt.value, ds.value

    def surface_normals(self):
        """Outward normals (3, n) float64 and flags (2, n) of the last evaluation."""
        import torch
        n = ctypes.c_int(0)
        self._chk(self.lib.rso_get_surface_points(self.h, None, 0, ctypes.byref(n)), "rso_get_surface_points")
        nrm = torch.empty(3 * max(n.value, 1), dtype=torch.float64, device="cuda")
        fl = torch.empty(2 * max(n.value, 1), dtype=torch.uint8, device="cuda")
        self._chk(self.lib.rso_get_surface_normals(self.h, _dev(nrm), _dev(fl)), "rso_get_surface_normals")
        return nrm[:3 * n.value].view(3, -1), fl[:2 * n.value].view(2, -1)

    # ------------------------------------------------------------ worst case
    def forceProject(self, f, constrain_direction):
        import torch
        f = f.clone()
        self._chk(self.lib.rso_force_project(self.h, _dev(f, torch.float64), int(constrain_direction)), "rso_force_project")
        return f

    def displacementProject(self, u):
        """u without the rigid motion of the active nodes (support-free modes; a copy)."""
        import torch
        u = u.clone()
        self._chk(self.lib.rso_displacement_project(self.h, _dev(u, torch.float64)), "rso_displacement_project")
        return u

    def worst_case(self, steps=20, constrain_direction=0, tol=1e-6, seed=1234):
        import torch
        fw = self._vec()
        uw = self._vec()
        lam = ctypes.c_double(0)
        ritz = np.zeros(steps)
        self._chk(self.lib.rso_worst_case(self.h, steps, int(constrain_direction), tol, seed, _dev(fw), _dev(uw),
                                          ctypes.byref(lam), _np_ptr(ritz, _pd)), "rso_worst_case")
        return lam.value, fw, uw, ritz

    def modifiedPM(self, constrain_direction=0, seed=1234, max_itn=500):
        fw = self._vec()
        uw = self._vec()
        c = ctypes.c_double(0)
        itn = ctypes.c_int(0)
        self._chk(self.lib.rso_modified_pm(self.h, int(constrain_direction), seed, max_itn, _dev(fw), _dev(uw),
                                           ctypes.byref(c), ctypes.byref(itn)), "rso_modified_pm")
        return c.value, fw, uw, itn.value

    # ------------------------------------------------------------ design iteration
    def design_iteration(self, mma, params=None):
        p = (params or IterParams())._c()
        info = _IterInfo()
        self._chk(self.lib.rso_design_iteration(self.h, mma.s, ctypes.byref(p), ctypes.byref(info)),
                  "rso_design_iteration")
        return {f[0]: getattr(info, f[0]) for f in _IterInfo._fields_}

    def design_iteration_host(self, mma, coeff_in, params=None, coeff_out=None, density=True):
        """One design iteration from host coefficients.  coeff_in / coeff_out may be
        numpy arrays or (pinned) CPU torch tensors of float64; density=False skips
        the download of the density field (returned as None)."""
        p = (params or IterParams())._c()
        info = _IterInfo()

        def host_ptr(a):
            if hasattr(a, "data_ptr"):
                if a.is_cuda or a.dtype.itemsize != 8 or not a.is_contiguous():
                    raise RSOError("expected a contiguous float64 CPU tensor")
                return ctypes.cast(ctypes.c_void_p(a.data_ptr()), _pd)
            return _np_ptr(a, _pd)

        cin = coeff_in if hasattr(coeff_in, "data_ptr") else np.ascontiguousarray(coeff_in, np.float64)
        cout = coeff_out if coeff_out is not None else np.zeros(self.n_coeff)
        rho = np.zeros(self.ne, np.float32) if density else None
        rptr = rho.ctypes.data_as(ctypes.POINTER(ctypes.c_float)) if density else None
        self._chk(self.lib.rso_design_iteration_host(self.h, mma.s, ctypes.byref(p), host_ptr(cin), host_ptr(cout),
                                                     rptr, ctypes.byref(info)), "rso_design_iteration_host")
        return cout, rho, {f[0]: getattr(info, f[0]) for f in _IterInfo._fields_}

    def design_gradient(self, coeff, params=None):
        """Objective values {lambda, volume, ss} and their gradients with respect
        to the spline coefficients (float64 CUDA tensors) at `coeff`, with no
        MMA step (rso_design_gradient)."""
        import torch
        p = (params or IterParams())._c()
        c = torch.as_tensor(coeff, dtype=torch.float64, device="cuda").contiguous()
        gl, gv, gs = (torch.empty_like(c) for _ in range(3))
        vals = np.zeros(3)
        self._chk(self.lib.rso_design_gradient(self.h, _dev(c, torch.float64), ctypes.byref(p), _np_ptr(vals, _pd),
                                               _dev(gl), _dev(gv), _dev(gs)), "rso_design_gradient")
        return {"lambda": vals[0], "volume": vals[1], "ss": vals[2]}, gl, gv, gs


class MMA:
    """MMA::mma_t (optimization/mma_t.h:159) on the device in FP64."""

    def __init__(self, n, m, xmin, xmax):
        self.lib = _StreamOrderedLib(load_library())
        self.n, self.m = n, m
        lo = np.broadcast_to(np.asarray(xmin, np.float64), (n,)).copy()
        hi = np.broadcast_to(np.asarray(xmax, np.float64), (n,)).copy()
        s = ctypes.c_void_p()
        st = self.lib.rso_mma_create(n, m, _np_ptr(lo, _pd), _np_ptr(hi, _pd), ctypes.byref(s))
        if st:
            raise RSOError(f"rso_mma_create: {_STATUS.get(st, st)}")
        self.s = s

    def close(self):
        if getattr(self, "s", None):
            self.lib.rso_mma_destroy(self.s)
            self.s = None

    def __del__(self):
        self.close()

    def set_x(self, x):
        import torch
        if isinstance(x, torch.Tensor) and x.is_cuda:
            st = self.lib.rso_mma_set_x_dev(self.s, _dev(x.contiguous(), torch.float64))
        else:
            st = self.lib.rso_mma_set_x(self.s, _np_ptr(np.ascontiguousarray(x, np.float64), _pd))
        if st:
            raise RSOError(f"rso_mma_set_x: {_STATUS.get(st, st)}")

    def save(self):
        """Checkpoint of the MMA state (rso_mma_save): 6 n + 1 doubles."""
        k = ctypes.c_longlong(0)
        self.lib.rso_mma_state_size(self.s, ctypes.byref(k))
        st = np.zeros(k.value)
        if self.lib.rso_mma_save(self.s, _np_ptr(st, _pd)):
            raise RSOError("rso_mma_save failed")
        return st

    def load(self, state):
        """Resume from a checkpoint made by save() (rso_mma_load)."""
        st = np.ascontiguousarray(state, np.float64)
        if st.size != 6 * self.n + 1:
            raise RSOError("checkpoint size does not match this MMA")
        if self.lib.rso_mma_load(self.s, _np_ptr(st, _pd)):
            raise RSOError("rso_mma_load failed")

    def get(self):
        x, L, U, a, b = [np.zeros(self.n) for _ in range(5)]
        st = self.lib.rso_mma_get(self.s, _np_ptr(x, _pd), _np_ptr(L, _pd), _np_ptr(U, _pd), _np_ptr(a, _pd),
                                  _np_ptr(b, _pd))
        if st:
            raise RSOError(f"rso_mma_get: {_STATUS.get(st, st)}")
        return x, L, U, a, b

    def update(self, df, dg, g):
        import torch
        df = df.to(device="cuda", dtype=torch.float64).contiguous()
        dg = dg.to(device="cuda", dtype=torch.float64).contiguous()
        gv = np.ascontiguousarray(g, np.float64)
        conv = ctypes.c_int(0)
        info = np.zeros(4)
        st = self.lib.rso_mma_update(self.s, _dev(df), _dev(dg), _np_ptr(gv, _pd), ctypes.byref(conv),
                                     _np_ptr(info, _pd))
        if st:
            raise RSOError(f"rso_mma_update: {_STATUS.get(st, st)}")
        return bool(conv.value), info
