"""Replay of the mixed-precision V-cycle from CUDA graphs (rso_set_vcycle_graphs)
against plain launches, through the C ABI.  A replay runs the same kernels with
the same arguments as the launches it was captured from, so solutions must be
bitwise equal and iteration counts the same; with profiling on, the kernels
inside replayed graphs are timed like launched ones (same launch counts per
class) and the process-wide launch counter advances by the same amount."""
import ctypes

import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu


def make(prob, graphs, precision=1, smoother=2):
    from robustoptspline3d_b200 import Config, HierarchyGrid
    g = HierarchyGrid(prob["emask"], prob["fixed"], prob["load"], prob["normals"],
                      Config(precision=precision, smoother=smoother, poisson_ratio=0.4, omega=0.6, cheb_lower=0.1))
    g.set_density(prob["rho"].astype(np.float32).ravel())
    g.update_stencil()
    g.set_vcycle_graphs(graphs)
    return g


def loads(g, k, seed):
    rng = np.random.default_rng(seed)
    ln = g.load_nodes()
    F = np.zeros((k, 3 * g.nn))
    for b in range(k):
        for c in range(3):
            F[b, c * g.nn + ln] = rng.standard_normal(len(ln))
    return F


def profile(g, cls):
    n = ctypes.c_longlong(0)
    ms = ctypes.c_double(0)
    b = ctypes.c_double(0)
    fl = ctypes.c_double(0)
    name = ctypes.create_string_buffer(64)
    assert g.lib.rso_profile_class(g.h, cls, name, 64, ctypes.byref(n), ctypes.byref(ms), ctypes.byref(b),
                                   ctypes.byref(fl)) == 0
    return name.value.decode(), n.value, ms.value


@pytest.mark.parametrize("gen,smoother", [(lambda: P.cantilever(48, 24, 24), 2),
                                          (lambda: P.ellipsoid(40, 24, 24), 1)])
def test_graph_solves_equal_plain(cuda, gen, smoother):
    prob = gen()
    F = loads(make(prob, False, smoother=smoother), 3, 21)
    res = {}
    for graphs in (False, True):
        g = make(prob, graphs, smoother=smoother)
        lib = g.lib
        l0 = lib.rso_launch_count()
        out = []
        for b in range(3):  # several solves: later V-cycles replay graphs captured in earlier ones
            u, it, rr, _ = g.solve(cuda.tensor(F[b], dtype=cuda.float64, device="cuda"), tol=1e-8, max_iter=200)
            out.append((u.cpu().numpy(), it, rr))
        res[graphs] = (out, lib.rso_launch_count() - l0)
        g.close()
    (plain, n_plain), (graph, n_graph) = res[False], res[True]
    for (up, ip, rp), (ug, ig, rg) in zip(plain, graph):
        assert ip == ig and ip > 6
        assert rp == rg
        assert np.array_equal(up, ug)
    assert n_plain == n_graph


def test_graph_profiling_and_batch(cuda):
    prob = P.cantilever(48, 24, 24)
    F = loads(make(prob, False), 4, 22)
    res = {}
    for graphs in (False, True):
        g = make(prob, graphs)
        g.lib.rso_set_profiling(g.h, 1)
        g.lib.rso_profile_reset(g.h)
        u, it, _, _ = g.solve(cuda.tensor(F[0], dtype=cuda.float64, device="cuda"), tol=1e-8, max_iter=200)
        prof = [profile(g, c) for c in range(10)]
        U, infos = g.solve_batch(cuda.tensor(F, dtype=cuda.float64, device="cuda"), tol=1e-8, max_iter=200)
        res[graphs] = (u.cpu().numpy(), it, prof, U.cpu().numpy(), infos)
        g.close()
    (u0, i0, p0, U0, f0), (u1, i1, p1, U1, f1) = res[False], res[True]
    assert i0 == i1 and np.array_equal(u0, u1)
    for (name, n0, ms0), (_, n1, ms1) in zip(p0, p1):
        assert n0 == n1, name
        if n0:
            assert ms0 > 0 and ms1 > 0, name
    assert dict((n, k) for n, k, _ in p1)["fine_jacobi_fp32"] > 0
    assert [i for i, _ in f0] == [i for i, _ in f1]
    assert np.array_equal(U0, U1)
