"""Hand-written adjoint of the robust spline design against central finite
differences, through the C ABI (rso_design_gradient) and the
torch.autograd.Function wrapper.

Objective: lambda_max of the worst-case load (ff mode, Lanczos over FP64
multigrid solves to 1e-10), plus the volume fraction and the self-support
value, as functions of the tricubic B-spline control coefficients.  The
sensitivity filter is off (filter_mode 1) so the adjoint is the exact
gradient.  Step h = 1e-3: the density field is stored in FP32 (as the
reference's rho_e), so a step of 1e-6 would sit below its resolution; the
central difference error at h = 1e-3 is O(h^2).  Tolerance: 1e-4 relative
(norm over the 50 sampled coefficients) for lambda_max and the volume.
The self-support value is checked in mode 5, a smooth function of the
coefficients.  Mode 4 (the overhang default) counts only elements whose
normal points down and divides by their number; both change in steps as the
coefficients move, so a finite difference across a step disagrees with the
derivative between steps, which is checked against the oracle instead.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_FD = 50
H = 1e-3


def _setup(cuda, n=24, order=4, parts=4, ss_mode=5):
    import robustoptspline3d_b200 as R
    em = np.ones((n, n, n), np.uint8)
    fa = np.zeros((n + 1,) * 3, np.uint8)
    fa[0] = 1                      # z = 0 node layer clamped
    la = np.zeros_like(fa)
    la[n] = 1                      # load set: top-face nodes
    g = R.HierarchyGrid(em, fa, la, None, R.Config(precision=R.rso.FP64, smoother=R.rso.SMOOTH_JACOBI,
                                                   omega=0.6, pre=2, post=2, poisson_ratio=0.3))
    nc = g.set_spline_partition(parts, parts, parts, order)
    rng = np.random.default_rng(4)
    c = cuda.tensor(np.clip(rng.normal(0.5, 0.15, nc), 0.05, 0.95), dtype=cuda.float64, device="cuda")
    prm = R.IterParams(beta=8.0, filter_mode=1, lanczos_steps=30, solve_tol=1e-10, constrain_direction=0, ss_mode=ss_mode,
                       seed=77)
    return g, c, prm


def test_adjoint_matches_central_differences(cuda):
    g, c, prm = _setup(cuda)
    vals, gl, gv, gs = g.design_gradient(c, prm)
    assert vals["lambda"] > 0 and 0 < vals["volume"] < 1
    rng = np.random.default_rng(2026)
    # sample among coefficients whose lambda gradient is not negligible
    big = np.nonzero(np.abs(gl.cpu().numpy()) > 1e-3 * np.abs(gl.cpu().numpy()).max())[0]
    idx = rng.choice(big, size=min(N_FD, len(big)), replace=False)
    fd = np.zeros((3, len(idx)))
    for j, k in enumerate(idx):
        cp = c.clone(); cp[k] += H
        cm = c.clone(); cm[k] -= H
        vp = g.design_gradient(cp, prm)[0]
        vm = g.design_gradient(cm, prm)[0]
        for i, key in enumerate(("lambda", "volume", "ss")):
            fd[i, j] = (vp[key] - vm[key]) / (2 * H)
    ad = np.stack([t.cpu().numpy()[idx] for t in (gl, gv, gs)])
    rel = np.linalg.norm(fd - ad, axis=1) / np.linalg.norm(ad, axis=1)
    assert rel[0] < 1e-4, rel
    assert rel[1] < 1e-4, rel
    assert rel[2] < 1e-3, rel
    g.close()


def test_autograd_function(cuda):
    from robustoptspline3d_b200.autograd import worst_case_objective
    g, c, prm = _setup(cuda, n=16, parts=3, ss_mode=4)
    x = c.clone().requires_grad_(True)
    y = worst_case_objective(x, g, prm)
    w = cuda.tensor([1.0, -2.0, 0.5], dtype=cuda.float64, device="cuda")
    (y * w).sum().backward()
    _, gl, gv, gs = g.design_gradient(c, prm)
    expect = gl - 2.0 * gv + 0.5 * gs
    assert y.shape == (3,) and float(y[0].detach()) > 0
    assert cuda.allclose(x.grad, expect, rtol=1e-12, atol=1e-300)
    g.close()
