"""Independent handles used from several host threads at once (each handle
has its own CUDA stream): results equal those of the same solves run one
after another, bit for bit."""
import concurrent.futures

import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu


def test_concurrent_handles_match_sequential(cuda):
    from robustoptspline3d_b200 import Config, HierarchyGrid
    probs = [P.cantilever(24, 12, 12, seed=1), P.cantilever(32, 16, 16, seed=2), P.cantilever(40, 20, 12, seed=4),
             P.cantilever(16, 8, 8, seed=3)]
    grids, loads = [], []
    for pr in probs:
        g = HierarchyGrid(pr["emask"], pr["fixed"], pr["load"], pr["normals"], Config(smoother=2, poisson_ratio=0.4))
        g.set_density(pr["rho"].astype(np.float32).ravel())
        g.update_stencil()
        grids.append(g)
        loads.append(cuda.tensor(pr["f"], dtype=cuda.float64, device="cuda"))

    def solve(i):
        u, it, rr, _ = grids[i].solve(loads[i], tol=1e-8, max_iter=400)
        return u.cpu().numpy(), it

    seq = [solve(i) for i in range(len(grids))]
    with concurrent.futures.ThreadPoolExecutor(max_workers=len(grids)) as ex:
        con = list(ex.map(solve, range(len(grids))))
    for (us, its), (uc, itc) in zip(seq, con):
        assert its == itc
        assert np.array_equal(us, uc)
    for g in grids:
        g.close()


def test_live_handles_share_the_material(cuda):
    """The element matrix lives in per-device constant memory: a second live
    handle with another Poisson ratio is refused, and accepted once the first
    is destroyed."""
    from robustoptspline3d_b200 import Config, HierarchyGrid, RSOError
    pr = P.cantilever(16, 8, 8)
    a = HierarchyGrid(pr["emask"], pr["fixed"], pr["load"], None, Config(poisson_ratio=0.3))
    with pytest.raises(RSOError, match="Poisson"):
        HierarchyGrid(pr["emask"], pr["fixed"], pr["load"], None, Config(poisson_ratio=0.4))
    b = HierarchyGrid(pr["emask"], pr["fixed"], pr["load"], None, Config(poisson_ratio=0.3))
    b.close()
    a.close()
    c = HierarchyGrid(pr["emask"], pr["fixed"], pr["load"], None, Config(poisson_ratio=0.4))
    c.close()
