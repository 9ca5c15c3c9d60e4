"""Parity at the sizes of the benchmark configurations, through the C ABI,
against the FP64 oracle (the reference method in FP64, solves to relative
residual 1e-10 on the library side and 1e-12 on the oracle's).

- Config 0 at full size: the 64x32x32 cantilever, 4 levels (64x32x32 ->
  8x4x4), 2 + 2 damped-Jacobi sweeps (omega 0.6 of 2 / lambda_max(D^-1 K)),
  FP64 and mixed precision, solved by V-cycles alone and by PCG: u within
  1e-5, compliance within 1e-6 and dC/drho within 1e-4 relative.
- Config 1 at full size: the 128x64x64 ellipsoid, constrained-direction
  worst case from 20 Lanczos steps, FP64 and mixed, against the oracle's run
  stored in tests/golden/config1.npz (make_config1.py; the oracle needs
  minutes there): lambda_max and the Ritz values within 1e-6, the sign-
  normalised f_worst and u_worst within 1e-5 and d lambda / d rho within 1e-4
  on seeded samples, and the sensitivity field's sum within 1e-5.
- One design iteration of the config-4 shape at 24^3 (order-4 spline on 4^3
  partitions, Heaviside beta 8, self-support mode 4 at 45 degrees, volume
  0.3, 20 Lanczos steps, solves to 1e-10): lambda_max, volume and the
  self-support value, their coefficient gradients through the adjoint chain,
  and the coefficients after the MMA step.
"""
import os

import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("precision", [0, 1])
def test_config0_cantilever_full_size(oracle, cuda, precision):
    from robustoptspline3d_b200 import Config, HierarchyGrid
    prob = P.cantilever(64, 32, 32)
    g = HierarchyGrid(prob["emask"], prob["fixed"], prob["load"], None,
                      Config(poisson_ratio=0.4, n_levels=4, first_factor=2, smoother=1, omega=0.6, pre=2, post=2,
                             precision=precision))
    o = oracle.Problem(prob["emask"], prob["fixed"], prob["load"], None, nu=0.4, n_levels=4, first_factor=2)
    rho = prob["rho"].astype(np.float32).ravel()
    g.set_density(rho)
    o.set_density(rho.astype(np.float64))
    g.update_stencil()
    o.update_stencil()
    assert g.n_levels() == o.n_levels() == 4
    assert list(g.level_dims(3)[:3]) == [8, 4, 4]
    f = prob["f"]
    uo, _, rro = o.solve(f, tol=1e-12, method=1)
    assert rro < 1e-12
    co = f @ uo
    so = o.sensitivity(uo)
    ft = cuda.as_tensor(f, device="cuda")
    for method, max_iter in ((1, 300), (0, 600)):
        ug, it, rr, _ = g.solve(ft, tol=1e-10, method=method, max_iter=max_iter)
        assert rr < 1e-10, (method, it, rr)
        un = ug.cpu().numpy()
        assert rel(un, uo) < 1e-5, method
        assert abs(f @ un - co) <= 1e-6 * abs(co), method
        assert rel(g.computeSensitivity(ug).cpu().numpy(), so) < 1e-4, method
    g.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_config1_worst_case_full_size(cuda, precision):
    from robustoptspline3d_b200 import Config, HierarchyGrid
    ref = np.load(os.path.join(GOLDEN, "config1.npz"))
    prob = P.ellipsoid(128, 64, 64, seed=1, shell=3, axes=(60.0, 30.0, 30.0))
    assert int(prob["emask"].sum()) == int(ref["active"])
    g = HierarchyGrid(prob["emask"], prob["fixed"], prob["load"], prob["normals"],
                      Config(poisson_ratio=float(ref["nu"]), precision=precision, smoother=2, cheb_lower=0.1))
    g.set_density(prob["rho"].astype(np.float32).ravel())
    g.update_stencil()
    assert g.n_levels() == int(ref["n_levels"])
    lam, fw, uw, ritz = g.worst_case(steps=len(ref["ritz"]), constrain_direction=1, tol=float(ref["tol"]),
                                     seed=int(ref["seed"]))
    assert abs(lam - ref["lam"]) <= 1e-6 * ref["lam"]
    assert np.allclose(ritz, ref["ritz"], rtol=1e-6, atol=0)
    f = fw.cpu().numpy()
    u = uw.cpu().numpy()
    s = np.sign(f[ref["jf"]] @ ref["f"])
    assert abs(np.linalg.norm(f) - ref["f_norm"]) <= 1e-9 * ref["f_norm"]
    assert rel(s * f[ref["jf"]], ref["f"]) < 1e-5
    assert rel(s * u[ref["iu"]], ref["u"]) < 1e-5
    assert abs(np.linalg.norm(u) - ref["u_norm"]) <= 1e-5 * ref["u_norm"]
    sens = g.computeSensitivity(uw).cpu().numpy().astype(np.float64)
    assert rel(sens[ref["ks"]], ref["sens"]) < 1e-4
    assert abs(sens.sum() - ref["sens_sum"]) <= 1e-5 * abs(ref["sens_sum"])
    g.close()


def oracle_design(oracle, em, fa, la, order, parts, coeff, beta, lanczos_steps, tol, radius):
    """The oracle's chain of one design iteration (spline -> Heaviside ->
    operators -> Lanczos worst case -> self-support -> adjoint chain)."""
    p = oracle.Problem(em, fa, la, None, nu=0.3)
    p.spline_setup(order, parts)
    rh = p.coeff2density(coeff)
    rho = oracle.heaviside(rh, beta, 1e-3)
    p.set_density(rho)
    p.update_stencil()
    lam, _, uw, _ = p.lanczos(lanczos_steps, 0, tol=tol)
    ssv, _, dss, _, _ = p.selfsupport(coeff, beta, 4)
    s = oracle.heaviside_chain(rh, beta, p.sensitivity(uw))
    v = oracle.heaviside_chain(rh, beta, np.full(p.ne, 1.0 / p.ne))
    dlam = p.density2coeff_adjoint(p.filter(radius, s))
    dvol = p.density2coeff_adjoint(p.filter(radius, v))
    return lam, rho.mean(), ssv, dlam, dvol, dss


@pytest.mark.parametrize("precision", [0, 1])
def test_design_iteration_matches_oracle(oracle, cuda, precision):
    from robustoptspline3d_b200 import MMA, Config, HierarchyGrid, IterParams
    n, order, parts = 24, 4, (4, 4, 4)
    em = np.ones((n, n, n), np.uint8)
    fa = np.zeros((n + 1,) * 3, np.uint8)
    fa[0] = 1
    la = np.zeros_like(fa)
    la[n] = 1
    g = HierarchyGrid(em, fa, la, None, Config(precision=precision, smoother=2, cheb_lower=0.1))
    nc = g.set_spline_partition(*parts, order)
    coeff = np.clip(np.random.default_rng(2026).normal(0.5, 0.15, nc), 0.0, 1.0)
    prm = IterParams(beta=8.0, volume_ratio=0.3, filter_radius=2.0, lanczos_steps=20, solve_tol=1e-10,
                     constrain_direction=0, ss_mode=4)
    vals, gl, gv, gs = g.design_gradient(coeff, prm)
    lam, vol, ssv, dlam, dvol, dss = oracle_design(oracle, em, fa, la, order, parts, coeff, 8.0, 20, 1e-10, 2.0)
    assert abs(vals["lambda"] - lam) <= 1e-6 * abs(lam)
    assert abs(vals["volume"] - vol) <= 1e-6 * abs(vol)
    assert abs(vals["ss"] - ssv) <= 1e-5 * abs(ssv)
    assert rel(gl.cpu().numpy(), dlam) < 1e-4
    assert rel(gv.cpu().numpy(), dvol) < 1e-5
    assert rel(gs.cpu().numpy(), dss) < 1e-4
    # the MMA step of the iteration on the same objective and constraints
    mma = MMA(nc, 2, 0.0, 1.0)
    mma.set_x(coeff)
    g.design_iteration(mma, prm)
    x_gpu = mma.get()[0]
    m = oracle.MMA(nc, 2, 0.0, 1.0)
    m.set_x(coeff)
    m.update(dlam * prm.sens_scale, np.stack([dvol * prm.vol_scale, dss * prm.ss_scale]),
             np.array([prm.vol_scale * (vol - prm.volume_ratio), prm.ss_scale * ssv]))
    x_or = m.get()[0]
    assert np.abs(x_gpu - x_or).max() <= 1e-5
    assert np.abs(x_gpu - coeff).max() > 1e-3  # the step moved the design
    g.close()
    mma.close()
