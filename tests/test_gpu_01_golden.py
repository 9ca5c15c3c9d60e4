"""The CUDA path, through the C ABI, against golden fixtures produced by the
reference's own code (tests/golden/make_golden.py): the Heaviside projection
and its chain (rso_heaviside, rso_heaviside_chain), the sensitivity filter
(rso_filter) and the spline density map with its knot support test
(rso_spline_setup, rso_spline_axis, rso_coeff2density).  Both sides compute
in FP32 (the library's filter and spline sums in FP64 before rounding), so
the tolerances are a few FP32 ulps of each field's magnitude."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SHELL_BIT = 1 << 12


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


def grid(mask):
    from robustoptspline3d_b200 import Config, HierarchyGrid
    e = mask.shape[0]
    fixed = np.zeros((e + 1,) * 3, np.uint8)
    fixed[:, :, 0] = 1
    load = np.zeros_like(fixed)
    load[:, :, e] = 1
    return HierarchyGrid(mask, fixed, load, None, Config(rho_min=1e-3))


def maxrel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


def test_gpu_heaviside_golden(cuda):
    g = golden("proj.npz")
    n = g["rho"].size  # 4096 = 16^3 elements, one per golden entry
    hg = grid(np.ones((16, 16, 16), np.uint8))
    assert hg.ne == n
    shell = ((g["flag"] & SHELL_BIT) != 0).astype(np.uint8)
    for beta, out_rho, out_sens in zip(g["betas"], g["out_rho"], g["out_sens"]):
        fwd = hg.projectDensities(g["rho"], float(beta), shell).cpu().numpy()
        assert np.abs(fwd - out_rho).max() <= 2e-6, beta
        chain = hg.projectSensitivity(g["rho"], float(beta), g["sens"]).cpu().numpy()
        assert maxrel(chain, out_sens) <= 2e-6, beta
    hg.close()


def test_gpu_filter_golden(cuda):
    g = golden("filter.npz")
    mask = g["mask"]
    hg = grid(mask)
    flat = np.flatnonzero(mask.ravel())
    dense = np.zeros(mask.size, np.float32)
    dense[flat] = g["sens"]
    for r, ref in zip(g["radii"], g["out"]):
        out = hg.filterSensitivity(float(r), dense).cpu().numpy()
        assert maxrel(out[flat], ref) <= 4e-6, r
    hg.close()


@pytest.mark.parametrize("case", [0, 1])
def test_gpu_spline_golden(cuda, case):
    g = golden("spline.npz")
    mask = g["mask"]
    order = int(g["order"])
    parts = [int(v) for v in g[f"parts{case}"]]
    hg = grid(mask)
    nc = hg.set_spline_partition(*parts, order)
    assert nc == np.prod([order + q for q in parts])
    kn = g[f"knots{case}"]
    off = 0
    for a in range(3):
        kmin, kstep = kn[off], kn[off + 2]
        off += 3 + 2 * order + parts[a]
        idx, N, _ = hg.spline_axis(a)
        pos = np.arange(mask.shape[0], dtype=np.float32) + np.float32(0.5)
        span = ((pos - kmin) / kstep).astype(np.int32) + order
        inside = (span >= order) & (span <= order + parts[a])
        assert np.array_equal(idx >= 0, inside) and np.array_equal(idx[inside], span[inside])
        assert np.abs(N[inside] - g[f"axis{case}"][a][inside, :order]).max() <= 1e-6
    flat = np.flatnonzero(mask.ravel())
    shell = np.zeros(mask.size, np.uint8)
    shell[flat] = (g[f"eflag{case}"] & SHELL_BIT) != 0
    rho = hg.coeff2density(g[f"coeff{case}"], shell).cpu().numpy()
    assert np.abs(rho[flat] - g[f"rho{case}"]).max() <= 2e-6
    hg.close()
