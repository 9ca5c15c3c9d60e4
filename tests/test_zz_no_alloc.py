"""The sensitivity filter without device allocation (rso_filter_noalloc)
against the allocating entry point rso_filter, through the C ABI.

Tolerance: 1e-6 relative (both compute the same FP64 sums over the same taps
and round to FP32).  The file is collected last so that it also runs after
every other GPU test in the same process; it needs nothing those set up.
"""
import ctypes

import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _call(g, fn, radius, x):
    out = x.new_full(x.shape, float("nan"))
    st = fn(g.h, radius, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()))
    return st, out


def _rel(a, b):
    a = a.double().cpu().numpy()
    b = b.double().cpu().numpy()
    assert np.all(np.isfinite(a))
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_filter_noalloc_matches_filter(cuda):
    from robustoptspline3d_b200 import HierarchyGrid
    torch = cuda
    prob = P.ellipsoid(24, 16, 12)
    g = HierarchyGrid(prob["emask"], prob["fixed"], prob["load"], prob["normals"])
    rng = np.random.default_rng(31)
    # the largest reach first, so the later, smaller calls find stale taps of
    # an earlier call in the shared table beyond their own cube
    cases = [(6.4, 3), (3.0, 1), (1.5, 2)]
    xs = [torch.tensor(rng.standard_normal(g.ne).astype(np.float32), device="cuda") for _ in cases]
    refs = []
    for (radius, _), x in zip(cases, xs):
        st, ref = _call(g, g.lib.rso_filter, radius, x)
        assert st == 0, g.lib.rso_last_error(g.h).decode()
        refs.append(ref)
    # consecutive calls of the no-allocation entry point
    outs = []
    for (radius, _), x in zip(cases, xs):
        st, out = _call(g, g.lib.rso_filter_noalloc, radius, x)
        assert st == 0, g.lib.rso_last_error(g.h).decode()
        outs.append(out)
    for (radius, _), out, ref in zip(cases, outs, refs):
        assert _rel(out, ref) < TOL, radius
    # the same call again after a smaller one
    st, again = _call(g, g.lib.rso_filter_noalloc, cases[1][0], xs[1])
    assert st == 0 and _rel(again, refs[1]) < TOL
    # radii beyond the fixed table are refused, with a message, before any work
    st, out = _call(g, g.lib.rso_filter_noalloc, 6.5, xs[0])
    assert st == 1
    assert "rso_filter_noalloc" in g.lib.rso_last_error(g.h).decode()
    assert torch.isnan(out).all()
    g.close()


def test_filter_noalloc_leaves_device_memory_unchanged(cuda):
    """Free device memory (cudaMemGetInfo) is the same before and after calls
    at radii this handle has not used yet: no call allocates, the first one
    on the handle included.  Outputs are allocated before the first reading."""
    from robustoptspline3d_b200 import HierarchyGrid
    torch = cuda
    prob = P.cantilever(24, 12, 12)
    g = HierarchyGrid(prob["emask"], prob["fixed"], prob["load"], prob["normals"])
    x = torch.tensor(np.random.default_rng(5).standard_normal(g.ne).astype(np.float32), device="cuda")
    outs = [torch.empty_like(x) for _ in range(4)]
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for radius, out in zip((1.2, 2.6, 4.4, 6.1), outs):
        st = g.lib.rso_filter_noalloc(g.h, radius, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()))
        assert st == 0, g.lib.rso_last_error(g.h).decode()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    for out in outs:
        assert torch.isfinite(out).all()
    g.close()
