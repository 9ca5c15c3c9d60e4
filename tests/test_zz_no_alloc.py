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
