"""CPU tests: the FP64 oracle against golden fixtures produced by the
reference's own code (tests/golden/make_golden.py runs definitions extracted
unmodified from the reference's sources and compiled on the host).  These pin
the oracle's Heaviside projection and its chain (a17), the sensitivity filter
(a18), the knot series, basis functions and density map of the spline (a19)
and the self-support penalty functions (a21) to the reference's arithmetic.

The reference computes in FP32 and the oracle in FP64, so values agree to
FP32 rounding: tolerances are stated per test relative to the magnitude of
the compared field.  Integer work (knot indices, support tests) is exact."""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SHELL_BIT = 1 << 12


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


def close(a, b, rtol):
    """|a - b| within rtol of the largest |b| (FP32 against FP64 over a field)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    return np.abs(a - b).max() <= rtol * scale


def box_problem(oracle, mask):
    e = mask.shape[0]
    fixed = np.zeros((e + 1,) * 3, np.uint8)
    fixed[:, :, 0] = 1
    load = np.zeros_like(fixed)
    load[:, :, e] = 1
    return oracle.Problem(mask, fixed, load, rhomin=1e-3)


def test_golden_penalty_functions(oracle):
    """Heaviside, Dirac, h, dh, inner_, dinner_, overhang, doverhang,
    normal_distri, dnormal_distri (grid/Grid.cu:76-190) at 805 points for four
    parameter sets: FP32 reference against the FP64 oracle within 2e-6 of each
    row's largest magnitude."""
    g = golden("funcs.npz")
    x = g["x"].astype(np.float64)
    for (beta, a, mid, c), ref in zip(g["params"], g["out"]):
        ours = oracle.ss_funcs(x, beta, a, mid, c)
        for k in range(10):
            assert close(ours[k], ref[k], 2e-6), (k, beta, a, mid, c)


def test_golden_heaviside_projection(oracle):
    """computeProjection_kernel (forward, clamp to [rho_min, 1], shell
    elements 1) and computeProjectionSensitivity_kernel (chain with
    H'(rho)) at beta 1, 8 and 32."""
    g = golden("proj.npz")
    rho = g["rho"].astype(np.float64)
    shell = (g["flag"] & SHELL_BIT) != 0
    for beta, out_rho, out_sens in zip(g["betas"], g["out_rho"], g["out_sens"]):
        fwd = oracle.heaviside(rho, beta, float(g["rhomin"]), shell.astype(np.uint8))
        assert np.abs(fwd - out_rho).max() <= 2e-6
        assert np.all(fwd[shell] == 1) and np.all(out_rho[shell] == 1)
        chain = oracle.heaviside_chain(rho, beta, g["sens"].astype(np.float64))
        assert close(chain, out_sens, 2e-6), beta


@pytest.mark.parametrize("case", [0, 1])
def test_golden_spline(oracle, case):
    """Knot series, basis values and first derivatives at the element centres
    and the density map on a masked 16^3 grid (order 3, the reference's
    compile-time order): knot bounds and steps bit-identical (same float
    arithmetic), the support test per element coordinate exact, basis values
    within 1e-6, densities within 2e-6."""
    g = golden("spline.npz")
    mask = g["mask"]
    e, order = int(g["ereso"]), int(g["order"])
    parts = [int(v) for v in g[f"parts{case}"]]
    o = box_problem(oracle, mask)
    nc = o.spline_setup(order, parts)
    nb, bmin, step = o.spline_info()
    assert list(nb) == [order + q for q in parts] and nc == np.prod(nb)
    kn = g[f"knots{case}"]
    off = 0
    for a in range(3):
        kmin, kmax, kstep = kn[off:off + 3]
        knots = kn[off + 3:off + 3 + 2 * order + parts[a]]
        off += 3 + 2 * order + parts[a]
        assert bmin[a] == kmin and step[a] == kstep
        assert np.all(knots[:order] == kmin) and np.all(knots[-order:] == kmax)
        idx, N, dN = o.spline_axis(a)
        ref = g[f"axis{case}"][a]
        pos = np.arange(e, dtype=np.float32) + np.float32(0.5)
        span = ((pos - kmin) / kstep).astype(np.int32) + order
        inside = (span >= order) & (span <= nb[a])
        assert np.array_equal(idx >= 0, inside) and np.array_equal(idx[inside], span[inside])
        rb, rv, rd = ref[:, :order + 1], ref[:, order + 1:2 * order + 1], ref[:, 2 * order + 1:]
        assert np.all(rb[inside, order] == 0)
        assert np.abs(N[inside] - rb[inside, :order]).max() <= 1e-6
        assert np.abs(N[inside] - rv[inside]).max() <= 1e-6
        assert close(dN[inside], rd[inside], 1e-6)
    flat = np.flatnonzero(mask.ravel())
    shell = np.zeros(mask.size, np.uint8)
    shell[flat] = (g[f"eflag{case}"] & SHELL_BIT) != 0
    rho = o.coeff2density(g[f"coeff{case}"].astype(np.float64), shell)
    assert np.abs(rho[flat] - g[f"rho{case}"]).max() <= 2e-6


def test_golden_filter(oracle):
    """filterSensitivity_kernel on a masked 16^3 grid with isolated elements,
    radii 1, 1.5, 2 and 2.6 (integer reach int(R + 0.5), neighbours within R,
    inactive ones skipped): within 4e-6 of the largest filtered value (the
    reference sums the weights in FP32)."""
    g = golden("filter.npz")
    mask = g["mask"]
    o = box_problem(oracle, mask)
    flat = np.flatnonzero(mask.ravel())
    dense = np.zeros(mask.size)
    dense[flat] = g["sens"]
    for r, ref in zip(g["radii"], g["out"]):
        out = o.filter(float(r), dense)
        assert close(out[flat], ref, 4e-6), r
