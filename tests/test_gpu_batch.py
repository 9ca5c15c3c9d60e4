"""Batched solves (rso_solve_batch) against one-at-a-time solves of the same
systems, through the C ABI: k right-hand sides on one operator, FP64 and mixed
precision, damped Jacobi and Chebyshev smoothers.  Tolerance: both solve to a
relative residual of 1e-10, so the solutions agree to 1e-8 relative; a zero
right-hand side returns zero after no iteration."""
import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("precision,smoother,gen", [(0, 1, lambda: P.cantilever(32, 16, 16)),
                                                    (1, 2, lambda: P.cantilever(32, 16, 16)),
                                                    (1, 1, lambda: P.ellipsoid(40, 24, 24))])
def test_batch_matches_single(cuda, precision, smoother, gen):
    from robustoptspline3d_b200 import Config, HierarchyGrid
    prob = gen()
    g = HierarchyGrid(prob["emask"], prob["fixed"], prob["load"], prob["normals"],
                      Config(precision=precision, smoother=smoother, poisson_ratio=0.4, omega=0.6))
    g.set_density(prob["rho"].astype(np.float32).ravel())
    g.update_stencil()
    k = 5
    rng = np.random.default_rng(11)
    ln = g.load_nodes()
    F = np.zeros((k, 3 * g.nn))
    for b in range(k - 1):
        for c in range(3):
            F[b, c * g.nn + ln] = rng.standard_normal(len(ln)) * (10.0 ** b)  # different scales converge apart
    # the last system has a zero right-hand side
    Ft = cuda.tensor(F, dtype=cuda.float64, device="cuda")
    U, infos = g.solve_batch(Ft, tol=1e-10, max_iter=400)
    U = U.cpu().numpy()
    for b in range(k - 1):
        ub, it, rr, _ = g.solve(cuda.tensor(F[b], dtype=cuda.float64, device="cuda"), tol=1e-10, max_iter=400)
        assert infos[b][1] < 1e-10
        assert rel(U[b], ub.cpu().numpy()) < 1e-8, b
        assert abs(infos[b][0] - it) <= 1, (b, infos[b][0], it)
    assert infos[k - 1][0] == 0 and np.all(U[k - 1] == 0)
    # a second call with fewer systems reuses the buffers
    U2, infos2 = g.solve_batch(Ft[:2], tol=1e-10, max_iter=400)
    assert rel(U2.cpu().numpy(), U[:2]) < 1e-12
    g.close()
