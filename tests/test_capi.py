"""CPU checks of the C ABI library: it loads, exports every entry point that
include/rso.h declares, the Python binding covers them, and host-only
entry points validate their arguments without touching a GPU."""
import ctypes
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "rso.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(rso_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from robustoptspline3d_b200 import load_library
    from robustoptspline3d_b200.rso import SIGNATURES
    lib = load_library()
    names = declared()
    assert len(names) > 40
    for n in names:
        assert hasattr(lib, n), n
        assert n in SIGNATURES, n


def test_host_entry_points_without_gpu():
    from robustoptspline3d_b200 import load_library, element_matrix
    lib = load_library()
    K = element_matrix(1e6, 0.4)
    assert K.shape == (24, 24) and np.allclose(K, K.T)
    out = np.zeros(576)
    assert lib.rso_element_matrix(1e6, 0.6, 1.0, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 1
    assert lib.rso_element_matrix(1e6, 0.3, -1.0, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 1
    from robustoptspline3d_b200.rso import _Config
    c = _Config()
    lib.rso_default_config(ctypes.byref(c))
    assert c.youngs_modulus == 1e6 and c.first_factor == 4 and c.precision == 1
    # invalid arguments are rejected before any device work
    h = ctypes.c_void_p()
    assert lib.rso_create(ctypes.byref(c), 0, 4, 4, None, None, None, None, ctypes.byref(h)) == 1
    c.first_factor = 3
    em = np.ones(8, np.uint8)
    assert lib.rso_create(ctypes.byref(c), 2, 2, 2, em.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), None, None,
                          None, ctypes.byref(h)) == 1
    assert lib.rso_mma_create(0, 1, None, None, ctypes.byref(h)) == 1
    assert lib.rso_launch_count() >= 0


def test_oracle_header_mentions_pinning():
    txt = open(os.path.join(ROOT, "oracle", "oracle.h")).read()
    assert "TEST INFRASTRUCTURE ONLY" in txt and "parity unpinned" in txt


def test_binding_arity_matches_header():
    """Every prototype in include/rso.h has as many parameters as its ctypes signature."""
    from robustoptspline3d_b200.rso import SIGNATURES
    src = open(os.path.join(ROOT, "include", "rso.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    protos = re.findall(r"\b(rso_[a-z0-9_]+)\s*\(([^;{)]*)\)\s*;", src)
    assert len(protos) > 40
    for name, params in protos:
        params = " ".join(params.split())
        n = 0 if params in ("", "void") else params.count(",") + 1
        assert name in SIGNATURES, name
        assert len(SIGNATURES[name][1]) == n, (name, n, len(SIGNATURES[name][1]))
