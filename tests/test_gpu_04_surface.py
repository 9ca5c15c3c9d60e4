"""Surface-point self-support (deal_surface_points,
optimization/optimization.cpp:1185-1221) through the C ABI: the sampling of
rho = 0.5 on the background grid (rso_surface_points) against the oracle's
restatement, and the constraint with its coefficient gradient
(rso_surface_selfsupport) against the golden fixture made by the reference's
own per-point code and against the oracle.

Tolerances: sample counts exact; sample coordinates within 1e-5 element
units (the background values and crossings are FP32 from FP64 spline sums
in the same operation order on both sides); normals, per-point values,
means and gradients within 2e-6 / 1e-5 relative against the reference's FP32
fixture and 1e-9 against the FP64 oracle; flags and the orientation probe
sum exact; the gradient of the odd modes within 1e-5 of central differences
(h = 1e-4) of the mean at fixed points."""
import os

import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


def maxrel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


def pair(oracle, mask, order, parts):
    from robustoptspline3d_b200 import Config, HierarchyGrid
    ez, ey, ex = mask.shape
    fixed = np.zeros((ez + 1, ey + 1, ex + 1), np.uint8)
    fixed[:, :, 0] = 1
    load = np.zeros_like(fixed)
    load[:, :, ex] = 1
    g = HierarchyGrid(mask, fixed, load, None, Config(rho_min=1e-3))
    o = oracle.Problem(mask, fixed, load, rhomin=1e-3)
    nc = g.set_spline_partition(*parts, order)
    assert nc == o.spline_setup(order, parts)
    return g, o


def golden_pair(oracle):
    gd = golden("surface.npz")
    e = int(gd["ereso"])
    g, o = pair(oracle, np.ones((e, e, e), np.uint8), int(gd["order"]), [int(v) for v in gd["parts"]])
    return gd, g, o


def check_points(g, o, c, mc, npts, box=None):
    pts, info = g.generate_spline_surface_nodes(c, mc_res=mc, n_points=npts, model_box=box)
    opts, oinfo = o.surface_points(np.asarray(c, np.float64), mc=mc, n_points=npts, box=box)
    assert [info["n_crossings"], info["n_first_pick"], info["n_in_model"], info["n_points"]] == list(oinfo)
    got = pts.cpu().numpy()
    assert got.shape == opts.shape
    if got.size:
        assert np.abs(got - opts).max() <= 1e-5
    return got, oinfo


def test_surface_points_golden_box(oracle, cuda):
    """16^3 box, the fixture's coefficients, background resolution 16: the
    thinning path (more than 2 crossings per requested point), the padding path
    (fewer crossings than points) and no points at all."""
    gd, g, o = golden_pair(oracle)
    c = gd["coeff"]
    box = np.array([0, 0, 0, 16, 16, 16], np.float32)
    _, info = check_points(g, o, c, 16, 300, box)
    assert info[0] > 2 * 300 and info[1] == 900
    _, info = check_points(g, o, c, 16, 5000, box)
    assert info[1] == info[0] and info[2] < 5000
    check_points(g, o, c, 16, 0, box)
    g.close()


def test_surface_points_masked(oracle, cuda):
    """An ellipsoid (the model box = the active elements' bounding box):
    crossings outside the active elements are dropped; the thinning, padding
    and final-pick paths; a design without crossings gives n points at the
    origin."""
    mask = P.ellipsoid(24, 16, 16, shell=0)["emask"]
    em = mask.astype(bool)
    for order, parts, seed, mc, npts in ((4, (3, 3, 3), 7, 24, 700), (4, (3, 3, 3), 7, 12, 100000),
                                         (3, (4, 3, 3), 11, 24, 700)):
        g, o = pair(oracle, mask, order, parts)
        c = np.random.default_rng(seed).uniform(0, 1, g.n_coeff).astype(np.float32)
        pts, info = check_points(g, o, c, mc, npts)
        assert 0 < info[2] < info[1]
        ix = np.floor(pts).astype(int)
        assert np.all(em[ix[2], ix[1], ix[0]])
        if (order, mc) == (3, 24):
            assert info[2] > npts      # final equal-distance pick
            pts2, _ = g.generate_spline_surface_nodes(c, mc_res=mc, n_points=npts)
            assert np.array_equal(pts2.cpu().numpy(), pts)     # deterministic
        else:
            assert info[2] < npts      # padded with the first point
            assert np.all(pts[:, info[2]:] == pts[:, :1])
        g.close()
    g, o = pair(oracle, mask, 4, (3, 3, 3))
    pts, info = check_points(g, o, np.zeros(g.n_coeff, np.float32), 24, 50)
    assert info[0] == 0 and np.all(pts == 0)
    g.close()


def test_surface_constraint_golden(oracle, cuda):
    """At the fixture's 500 points (order 3, beta 8, 135 degree angles), all six
    modes: GPU against the reference's FP32 per-point code and the FP64 oracle."""
    gd, g, o = golden_pair(oracle)
    c = gd["coeff"]
    cd = c.astype(np.float64)
    g.uploadSurfacePoints(gd["pts"])
    opt = float(np.float32(gd["opt_ratio"] * np.pi))
    dft = float(np.float32(gd["default_ratio"] * np.pi))
    sc = gd["scalars"]
    for mode in range(6):
        val, per, dc, cnt, ds = g.deal_surface_points(c, float(gd["beta"]), mode, opt, dft)
        nrm, flags = g.surface_normals()
        r = o.surface_selfsupport(cd, gd["pts"], float(gd["beta"]), mode, opt, dft)
        assert ds == sc[0] == r["dirsum"]
        assert cnt == sc[1 + 2 * mode] == r["count"]
        nrm = nrm.cpu().numpy()
        assert maxrel(nrm, gd["normals"]) <= 2e-6 and maxrel(nrm, r["normals"]) <= 1e-12
        flags = flags.cpu().numpy()
        assert np.array_equal(flags[0], gd["flag"].astype(np.uint8)) and np.array_equal(flags, r["flags"])
        per = per.cpu().numpy()
        assert maxrel(per, gd["per"][mode]) <= 1e-5 and maxrel(per, r["per"]) <= 1e-6, mode
        assert abs(val - sc[2 + 2 * mode]) <= 1e-5 * max(1.0, abs(sc[2 + 2 * mode])), mode
        assert abs(val - r["value"]) <= 1e-9 * max(1.0, abs(r["value"])), mode
        dc = dc.cpu().numpy()
        assert maxrel(dc, gd["dc"][mode]) <= 1e-5 and maxrel(dc, r["dc"]) <= 1e-6, mode
    g.close()


@pytest.mark.parametrize("order", [3, 4])
def test_surface_constraint_sampled(oracle, cuda, order):
    """Sampled points of a masked design, then the constraint at them: GPU
    against the oracle at the oracle's own points, modes 0..5."""
    mask = P.ellipsoid(24, 16, 16, shell=0)["emask"]
    g, o = pair(oracle, mask, order, (4, 3, 3))
    c = np.random.default_rng(11).uniform(0, 1, g.n_coeff).astype(np.float32)
    pts, _ = check_points(g, o, c, 32, 400)
    opts, _ = o.surface_points(c.astype(np.float64), mc=32, n_points=400)
    g.uploadSurfacePoints(opts)
    for mode in range(6):
        val, per, dc, cnt, ds = g.deal_surface_points(c, 8.0, mode)
        r = o.surface_selfsupport(c.astype(np.float64), opts, 8.0, mode)
        assert ds == r["dirsum"] and cnt == r["count"]
        assert abs(val - r["value"]) <= 1e-9 * max(1.0, abs(r["value"])), mode
        assert maxrel(per.cpu().numpy(), r["per"]) <= 1e-6
        assert maxrel(dc.cpu().numpy(), r["dc"]) <= 1e-6, mode
    g.close()


@pytest.mark.parametrize("mode", [3, 5])
def test_surface_gradient_fd(oracle, cuda, mode):
    """Odd modes average over all points, so at fixed points the gradient is the
    derivative of the mean: central differences on 12 coefficients."""
    gd, g, o = golden_pair(oracle)
    c = gd["coeff"].astype(np.float64)
    g.uploadSurfacePoints(gd["pts"])
    _, _, dc, _, _ = g.deal_surface_points(gd["coeff"], 8.0, mode)
    dc = dc.cpu().numpy().astype(np.float64)
    r0 = o.surface_selfsupport(c, gd["pts"], 8.0, mode)
    rng = np.random.default_rng(3)
    idx = rng.choice(np.flatnonzero(np.abs(r0["dc"]) > 1e-3 * np.abs(r0["dc"]).max()), 12, replace=False)
    h = 1e-4
    for i in idx:
        cp, cm = c.copy(), c.copy()
        cp[i] += h
        cm[i] -= h
        fd = (o.surface_selfsupport(cp, gd["pts"], 8.0, mode)["value"] -
              o.surface_selfsupport(cm, gd["pts"], 8.0, mode)["value"]) / (2 * h)
        assert abs(fd - dc[i]) <= 1e-5 * np.abs(dc).max() + 1e-4 * abs(fd), (i, fd, dc[i])
    g.close()


def test_design_gradient_surface_points(oracle, cuda):
    """The design driver with the surface-point variant (IterParams.ss_points):
    its self-support value and gradient equal those of the sampling and the
    constraint called on their own, and match the oracle at the oracle's
    points (the coefficients are FP32 values, as the C ABI takes them)."""
    import robustoptspline3d_b200 as R
    n = 16
    em = np.ones((n, n, n), np.uint8)
    fa = np.zeros((n + 1,) * 3, np.uint8)
    fa[0] = 1
    la = np.zeros_like(fa)
    la[n] = 1
    g = R.HierarchyGrid(em, fa, la, None, R.Config(precision=R.rso.FP64, smoother=R.rso.SMOOTH_JACOBI, omega=0.6))
    nc = g.set_spline_partition(4, 4, 4, 4)
    c32 = np.random.default_rng(5).uniform(0, 1, nc).astype(np.float32)
    for mode in (4, 5):
        prm = R.IterParams(beta=8.0, filter_mode=1, lanczos_steps=6, solve_tol=1e-8, ss_mode=mode, ss_points=500,
                           ss_mc_res=20)
        vals, _, _, gs = g.design_gradient(c32.astype(np.float64), prm)
        pts, counts = g.generate_spline_surface_nodes(c32, mc_res=20, n_points=500)
        val, _, dc, _, _ = g.deal_surface_points(c32, 8.0, mode)
        assert vals["ss"] == val
        assert maxrel(gs.cpu().numpy(), dc.cpu().numpy()) <= 1e-6
        o = oracle.Problem(em, fa, la, n_levels=1)
        o.spline_setup(4, (4, 4, 4))
        opts, oinfo = o.surface_points(c32.astype(np.float64), mc=20, n_points=500)
        assert counts["n_crossings"] == oinfo[0]
        r = o.surface_selfsupport(c32.astype(np.float64), opts, 8.0, mode)
        assert abs(val - r["value"]) <= 1e-9 * max(1.0, abs(r["value"]))
        assert maxrel(gs.cpu().numpy(), r["dc"]) <= 1e-6
    g.close()
