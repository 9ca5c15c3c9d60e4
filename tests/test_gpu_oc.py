"""Optimality-criteria updaters (rso_oc_update_density, rso_oc_update_coeff)
through the C ABI against the numpy restatement of the reference's loops in
oracle/oc.py.  The bisection runs in FP32 on both sides; the per-element
update uses powf on the device and numpy's float32 power on the host, so the
densities agree to 1e-5 absolute, the threshold to 1e-5 relative, and the
trial counts exactly (a trial whose volume lands within rounding of the goal
would be the exception)."""
import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu


def make(oracle, prob):
    from robustoptspline3d_b200 import Config, HierarchyGrid
    g = HierarchyGrid(prob["emask"], prob["fixed"], prob["load"], prob["normals"], Config(poisson_ratio=0.3))
    o = oracle.Problem(prob["emask"], prob["fixed"], prob["load"], prob["normals"], nu=0.3)
    return g, o


@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("with_shell", [False, True])
def test_oc_density_matches_oracle(oracle, cuda, variant, with_shell):
    from oracle import oc
    prob = P.ellipsoid(24, 16, 12)
    g, o = make(oracle, prob)
    rng = np.random.default_rng(41)
    ne = o.ne
    active = o.level_masks(0)[0].astype(bool)
    rho = rng.uniform(0.2, 1.0, ne).astype(np.float32)
    sens = (-np.abs(rng.standard_normal(ne)) * 3.0).astype(np.float32)
    sens[rng.uniform(size=ne) < 0.1] = 0.5  # positive sensitivities count as zero
    shell = (rng.uniform(size=ne) < 0.05).astype(np.uint8) if with_shell else None
    vgoal, step, damp = 0.45, 0.2, 0.5
    out, info = g.updateDensities(rho, sens, vgoal, step=step, damp=damp, shell=shell, variant=variant)
    ro, go, vo, to = oc.update_density(rho, sens, active, vgoal, step, damp, 1e-3, shell, variant)
    assert info["trials"] == to
    assert abs(info["g"] - go) <= 1e-5 * go
    assert abs(info["volume"] - vo) <= 1e-6
    assert np.max(np.abs(out.cpu().numpy() - ro)) <= 1e-5
    if shell is None:  # with 5 % of the elements held at 1 the goal is out of reach within the trials
        assert abs(vo - vgoal) < 2e-3
    d = np.abs(ro - rho)
    assert abs(info["max_change"] - d.max()) <= 1e-5 and abs(info["mean_change"] - d.mean()) <= 1e-6
    # in place: rho_out may be rho_src
    g2, _ = make(oracle, prob)
    import torch
    buf = torch.as_tensor(rho, device="cuda").clone()
    from robustoptspline3d_b200.rso import _dev
    sh = None if shell is None else torch.as_tensor(shell, device="cuda")
    ss = torch.as_tensor(sens, device="cuda")
    assert g2.lib.rso_oc_update_density(g2.h, variant, _dev(buf), _dev(ss), _dev(sh), vgoal, step, damp,
                                        _dev(buf), None) == 0
    assert np.max(np.abs(buf.cpu().numpy() - ro)) <= 1e-5
    g.close()
    g2.close()


def test_oc_coeff_matches_oracle(oracle, cuda):
    from oracle import oc
    prob = P.ellipsoid(24, 16, 12)
    g, o = make(oracle, prob)
    order, parts = 3, (4, 4, 3)
    nc = o.spline_setup(order, parts)
    assert g.set_spline_partition(*parts, order) == nc
    rng = np.random.default_rng(42)
    c = np.clip(rng.normal(0.6, 0.15, nc), 0.0, 1.0).astype(np.float32)
    cs = (-np.abs(rng.standard_normal(nc))).astype(np.float32)
    vgoal, step, damp = 0.5, 0.1, 0.5
    cg, rg, info = g.updateCoeff(c, cs, vgoal, step=step, damp=damp, cmin=0.0, cmax=1.0)
    co, ro, go, vo, to = oc.update_coeff(o, c, cs, vgoal, step, damp, 0.0, 1.0)
    assert info["trials"] == to
    assert abs(info["g"] - go) <= 1e-5 * go
    assert abs(info["volume"] - vo) <= 1e-5
    assert np.max(np.abs(cg.cpu().numpy() - co)) <= 1e-5
    em = o.level_masks(0)[0].astype(bool)
    assert np.max(np.abs(rg.cpu().numpy()[em] - ro[em])) <= 1e-5
    g.close()
