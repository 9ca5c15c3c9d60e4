"""Device-controlled solves (rso_set_solve_graphs): the mixed-precision PCG
loop with the FP32 recurrence as one CUDA graph (a conditional WHILE node,
IF nodes for the FP64 residual replacement and the V-cycle), its decisions
taken by one-thread kernels.  The graph runs the host loop's kernels with
the host loop's arguments and decides on the same FP64 scalars with the same
arithmetic, so iterations, residuals and solutions are bit-identical to the
host-driven loop: on a cantilever and an ellipsoid, at two tolerances, with
a forced hand-over to the FP64 recurrence (one FP32 cycle), with the
iteration budget exhausted, and across repeated solves that replay the
cached graph."""
import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu


def make(prob):
    from robustoptspline3d_b200 import Config, HierarchyGrid
    g = HierarchyGrid(prob["emask"], prob["fixed"], prob["load"], prob["normals"],
                      Config(precision=1, smoother=2, poisson_ratio=0.4, cheb_lower=0.1, pre=2, post=2))
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


def both(g, f, **kw):
    from robustoptspline3d_b200.rso import RSOError
    out = []
    for on in (False, True):
        g.set_solve_graphs(on)
        try:
            u, it, rr, _ = g.solve(f, **kw)
            out.append((u.cpu().numpy(), it, rr, None))
        except RSOError as e:
            out.append((None, None, None, str(e)))
    g.set_solve_graphs(False)
    return out


@pytest.mark.parametrize("gen", [lambda: P.cantilever(48, 24, 24), lambda: P.ellipsoid(48, 32, 32)])
@pytest.mark.parametrize("tol", [1e-6, 1e-10])
def test_graph_solve_matches_host_loop(cuda, gen, tol):
    g = make(gen())
    f = cuda.tensor(rhs(g), dtype=cuda.float64, device="cuda")
    for rep in range(3):  # the first graph solve captures, the others replay
        (uh, ih, rh, eh), (ug, ig, rg, eg) = both(g, f, tol=tol, max_iter=400)
        assert eh is None and eg is None
        assert ig == ih and rg == rh, (rep, ig, ih, rg, rh)
        assert np.array_equal(ug, uh)
    g.close()


def test_graph_solve_handover_and_budget(cuda):
    g = make(P.cantilever(48, 24, 24))
    f = cuda.tensor(rhs(g), dtype=cuda.float64, device="cuda")
    # one FP32 cycle, then the FP64 recurrence on the host from the graph's iterate
    g.set_krylov_fp32_cycles(1)
    (uh, ih, rh, eh), (ug, ig, rg, eg) = both(g, f, tol=1e-10, max_iter=400)
    assert eh is None and eg is None and ig == ih and rg == rh and np.array_equal(ug, uh)
    g.set_krylov_fp32_cycles(0)
    # a budget too small for the tolerance: the same error on both paths
    (_, _, _, eh), (_, _, _, eg) = both(g, f, tol=1e-12, max_iter=4)
    assert eh is not None and eg is not None and "max_iter" in eh and "max_iter" in eg
    g.close()


def test_graph_solve_worst_case(cuda):
    """Lanczos worst case through graph solves equals the host-driven run."""
    g = make(P.ellipsoid(40, 24, 24))
    res = []
    for on in (False, True):
        g.set_solve_graphs(on)
        lam, fw, uw, ritz = g.worst_case(steps=8, constrain_direction=1, tol=1e-6)
        res.append((lam, fw.cpu().numpy(), uw.cpu().numpy(), ritz))
    assert res[0][0] == res[1][0] and np.array_equal(res[0][3], res[1][3])
    assert np.array_equal(res[0][1], res[1][1]) and np.array_equal(res[0][2], res[1][2])
    g.close()
