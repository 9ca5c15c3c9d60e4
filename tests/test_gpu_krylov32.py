"""Mixed-precision PCG with the FP32 Krylov recurrence and true-residual
replacement (rso_set_krylov_fp32, the mixed-precision default) against the
FP64 recurrence: the reported
residual is a true FP64 one (checked here with the FP64 operator), the
solutions agree to the tolerance, and the iteration counts stay close.  Also
a worst-case eigen step through it, and the argument checks."""
import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300)


def make(prob, smoother=2):
    from robustoptspline3d_b200 import Config, HierarchyGrid
    g = HierarchyGrid(prob["emask"], prob["fixed"], prob["load"], prob["normals"],
                      Config(precision=1, smoother=smoother, poisson_ratio=0.4, cheb_lower=0.1, pre=2, post=2))
    g.set_density(prob["rho"].astype(np.float32).ravel())
    g.update_stencil()
    return g


def rhs(g, seed=31):
    rng = np.random.default_rng(seed)
    f = np.zeros(3 * g.nn)
    ln = g.load_nodes()
    for c in range(3):
        f[c * g.nn + ln] = rng.standard_normal(len(ln))
    return f


@pytest.mark.parametrize("gen", [lambda: P.cantilever(64, 32, 32), lambda: P.ellipsoid(48, 32, 32)])
@pytest.mark.parametrize("factor", [1e-1, 1e-2, 1e-3])
@pytest.mark.parametrize("tol", [1e-6, 1e-10])
def test_fp32_recurrence_meets_true_tolerance(cuda, gen, factor, tol):
    prob = gen()
    g = make(prob)
    fh = rhs(g)
    f = cuda.tensor(fh, dtype=cuda.float64, device="cuda")
    g.set_krylov_fp32(0.0)
    u_ref, it_ref, rr_ref, _ = g.solve(f, tol=tol, max_iter=400)
    g.set_krylov_fp32(factor)
    u, it, rr, _ = g.solve(f, tol=tol, max_iter=400)
    assert rr < tol
    # the reported residual is the true one: recompute it with the FP64 operator
    r = fh - g.applyK(u).cpu().numpy()
    cls = g.node_class()
    sup = np.tile((cls & 4) > 0, 3)
    r[sup] = 0
    assert abs(np.linalg.norm(r) / np.linalg.norm(fh) - rr) <= 1e-3 * rr + 1e-15
    assert rel(u.cpu().numpy(), u_ref.cpu().numpy()) < 1e3 * tol
    assert it <= it_ref + 3, (it, it_ref)
    # switching back restores the FP64 recurrence exactly
    g.set_krylov_fp32(0.0)
    u2, it2, _, _ = g.solve(f, tol=tol, max_iter=400)
    assert it2 == it_ref and np.array_equal(u2.cpu().numpy(), u_ref.cpu().numpy())
    g.close()


def test_mixed_default_is_fp32_recurrence(cuda):
    prob = P.cantilever(32, 16, 16)
    g = make(prob)
    f = cuda.tensor(rhs(g), dtype=cuda.float64, device="cuda")
    u0, it0, _, _ = g.solve(f, tol=1e-8, max_iter=300)
    g.set_krylov_fp32(1e-2)
    u1, it1, _, _ = g.solve(f, tol=1e-8, max_iter=300)
    assert it0 == it1 and np.array_equal(u0.cpu().numpy(), u1.cpu().numpy())
    g.close()


def test_fp32_recurrence_worst_case(cuda):
    prob = P.ellipsoid(40, 24, 24)
    g = make(prob)
    g.set_krylov_fp32(0.0)
    lam_ref = g.worst_case(steps=20, tol=1e-8)[0]
    g.set_krylov_fp32(1e-2)
    lam = g.worst_case(steps=20, tol=1e-8)[0]
    assert abs(lam - lam_ref) <= 1e-6 * abs(lam_ref)
    g.close()


def test_set_krylov_fp32_arguments(cuda):
    from robustoptspline3d_b200.rso import RSOError
    g = make(P.cantilever(16, 8, 8))
    for bad in (-0.1, 1.0, float("nan")):
        with pytest.raises(RSOError):
            g.set_krylov_fp32(bad)
    g.close()


def applyk64_launches(g):
    import ctypes
    n = ctypes.c_longlong(0)
    ms, b, fl = ctypes.c_double(0), ctypes.c_double(0), ctypes.c_double(0)
    name = ctypes.create_string_buffer(64)
    assert g.lib.rso_profile_class(g.h, 3, name, 64, ctypes.byref(n), ctypes.byref(ms), ctypes.byref(b),
                                   ctypes.byref(fl)) == 0
    assert name.value.decode() == "fine_applyK_fp64"
    return n.value


def true_rel(g, fh, u):
    r = fh - g.applyK(u).cpu().numpy()
    sup = np.tile((g.node_class() & 4) > 0, 3)
    r[sup] = 0
    return np.linalg.norm(r) / np.linalg.norm(fh)


@pytest.mark.parametrize("graphs", [False, True])
def test_forced_handover_to_fp64_recurrence(cuda, graphs):
    """rso_set_krylov_fp32_cycles(1) hands every solve over to the FP64
    recurrence after its first residual replacement: the FP64 K p kernel runs
    (profiled launches), the true residual meets the tolerance, and single and
    batched solves agree with the FP64 recurrence's solutions.  Covers the
    q buffer the FP64 recurrence takes over from the FP32 one."""
    prob = P.cantilever(48, 24, 24)
    g = make(prob)
    g.set_vcycle_graphs(graphs)
    tol = 1e-8
    F = np.stack([rhs(g, s) for s in (41, 42, 43, 44)])
    g.set_krylov_fp32(0.0)
    refs = [g.solve(cuda.tensor(F[b], dtype=cuda.float64, device="cuda"), tol=tol, max_iter=300) for b in range(4)]
    g.set_krylov_fp32(1e-2)
    g.set_krylov_fp32_cycles(1)
    g.lib.rso_set_profiling(g.h, 1)
    g.lib.rso_profile_reset(g.h)
    for b in range(4):
        u, it, rr, _ = g.solve(cuda.tensor(F[b], dtype=cuda.float64, device="cuda"), tol=tol, max_iter=300)
        assert rr < tol and np.isfinite(rr)
        assert abs(true_rel(g, F[b], u) - rr) <= 1e-3 * rr + 1e-15
        assert rel(u.cpu().numpy(), refs[b][0].cpu().numpy()) < 1e3 * tol
        assert it <= refs[b][1] + 4, (it, refs[b][1])
    assert applyk64_launches(g) > 0
    U, infos = g.solve_batch(cuda.tensor(F, dtype=cuda.float64, device="cuda"), tol=tol, max_iter=300)
    for b in range(4):
        it, rr = infos[b]
        assert rr < tol and np.isfinite(rr)
        assert true_rel(g, F[b], U[b]) < 1.01 * tol
        assert rel(U[b].cpu().numpy(), refs[b][0].cpu().numpy()) < 1e3 * tol
        assert it <= refs[b][1] + 4, (it, refs[b][1])
    # without the bound the FP32 recurrence does not stall on this problem
    g.set_krylov_fp32_cycles(0)
    g.lib.rso_profile_reset(g.h)
    for b in range(2):
        g.solve(cuda.tensor(F[b], dtype=cuda.float64, device="cuda"), tol=tol, max_iter=300)
    g.solve_batch(cuda.tensor(F, dtype=cuda.float64, device="cuda"), tol=tol, max_iter=300)
    assert applyk64_launches(g) == 0
    g.lib.rso_set_profiling(g.h, 0)
    with pytest.raises(Exception):
        g.set_krylov_fp32_cycles(-1)
    g.close()
