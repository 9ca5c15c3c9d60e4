"""Support-free worst-case modes (nscf, nsff: HierarchyGrid::Mode,
grid/Grid.h:170-175; optimization/optimization.cpp:99-117) through the C ABI
against the FP64 oracle: the coarsest pseudo-inverse, forceProject with the
load set's rigid motions removed, solutions without rigid motion
(displacementProject), the Lanczos worst case against the oracle's dense
aggregated one, and the modified power method.

Tolerances as in the other parity tests: FP64 projections 1e-13, coarsest
solve 1e-9, converged solves 1e-5 in displacement, lambda_max 1e-6."""
import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def free_box(ex=12, ey=8, ez=8, seed=8):
    """A box without supports, load set the x = ex face (normal +x)."""
    em = np.ones((ez, ey, ex), np.uint8)
    fa = np.zeros((ez + 1, ey + 1, ex + 1), np.uint8)
    la = np.zeros_like(fa)
    la[:, :, ex] = 1
    nrm = np.zeros((fa.size, 3))
    nrm[:, 0] = 1.0
    rho = P.box_filter3(np.random.default_rng(seed).uniform(0.2, 1.0, em.shape), em.astype(float))
    return dict(emask=em, fixed=fa, load=la, normals=nrm, rho=rho)


def free_ellipsoid():
    """The config-1 shape at small size, floating: no node clamped."""
    prob = P.ellipsoid(20, 12, 12, shell=2)
    prob["fixed"] = np.zeros_like(prob["fixed"])
    return prob


def make(oracle, prob, mode, precision=0, smoother=1):
    from robustoptspline3d_b200 import Config, HierarchyGrid
    cfg = Config(n_levels=2, first_factor=2, mode=mode, precision=precision, smoother=smoother, pre=2, post=2)
    g = HierarchyGrid(prob["emask"], prob["fixed"], prob["load"], prob["normals"], cfg)
    o = oracle.Problem(prob["emask"], prob["fixed"], prob["load"], prob["normals"], n_levels=2, first_factor=2)
    rho = prob["rho"].astype(np.float32).ravel()
    g.set_density(rho)
    o.set_density(rho.astype(np.float64))
    g.update_stencil()
    o.update_stencil()
    return g, o


def t(x, torch):
    return torch.as_tensor(np.ascontiguousarray(x), device="cuda")


@pytest.mark.parametrize("gen,mode,cf", [(free_box, 1, 0), (free_ellipsoid, 0, 1)])
def test_support_free_projections_and_solves(oracle, cuda, gen, mode, cf):
    prob = gen()
    g, o = make(oracle, prob, mode)
    rng = np.random.default_rng(5)
    # no support node
    assert not np.any(g.node_class() & 4)
    # forceProject with the rigid motions of the load set removed
    f = rng.standard_normal(3 * o.nn)
    fo = o.force_project(f, cf)
    fg = g.forceProject(t(f, cuda), cf).cpu().numpy()
    assert rel(fg, fo) < 1e-13
    # displacementProject
    u = rng.standard_normal(3 * o.nn) * np.tile((g.node_class() & 1) > 0, 3)
    assert rel(g.displacementProject(t(u, cuda)).cpu().numpy(), o.displacement_project(u)) < 1e-12
    # the coarsest pseudo-inverse on an arbitrary right-hand side
    last = o.n_levels() - 1
    d = o.level_dims(last)
    nnc = int(d[3] * d[4] * d[5])
    _, vm = o.level_masks(last)
    fc = rng.standard_normal(3 * nnc) * np.tile(vm, 3)
    assert rel(g.solve_coarsest(t(fc, cuda)).cpu().numpy(), o.coarsest_solve(fc)) < 1e-9
    # solutions of a consistent load, without rigid motion, FP64 and mixed
    uo, _, rro = o.solve(fo, tol=1e-12)
    assert rro < 1e-12
    for precision in (0, 1):
        gp, _ = (g, None) if precision == 0 else make(oracle, prob, mode, precision=1, smoother=2)
        ug, it, rr, _ = gp.solve(t(fo, cuda), tol=1e-10, max_iter=400)
        assert rr < 1e-10
        ugn = ug.cpu().numpy()
        assert rel(ugn, uo) < 1e-5, precision
        assert rel(o.displacement_project(ugn), ugn) < 1e-12
        if gp is not g:
            gp.close()
    g.close()


@pytest.mark.parametrize("gen,mode,cf", [(free_box, 1, 0), (free_ellipsoid, 0, 1)])
def test_support_free_worst_case(oracle, cuda, gen, mode, cf):
    prob = gen()
    g, o = make(oracle, prob, mode, precision=1, smoother=2)
    lam_o, fo, uo = o.dense_worst(cf, tol=1e-12)
    lam_g, fg, ug, _ = g.worst_case(steps=60, constrain_direction=cf, tol=1e-10)
    assert abs(lam_g - lam_o) <= 1e-6 * lam_o
    fg = fg.cpu().numpy()
    # the worst load is admissible: its own projection
    assert rel(o.force_project(fg, cf), fg) < 1e-10
    ugn = ug.cpu().numpy()
    assert abs(fg @ ugn - lam_o) <= 1e-6 * lam_o
    g.close()


def test_support_free_modified_pm(oracle, cuda):
    prob = free_box(8, 6, 6)
    g, o = make(oracle, prob, 1, smoother=0)
    cg, _, _, itg = g.modifiedPM(0, seed=42, max_itn=300)
    co, _, _, ito = o.modified_pm(0, seed=42, max_itn=300)
    assert itg == ito
    assert abs(cg - co) <= 1e-8 * abs(co)
    g.close()
