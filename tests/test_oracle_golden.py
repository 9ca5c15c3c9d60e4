"""CPU tests: the FP64 oracle against golden fixtures produced by the
reference's own code (tests/golden/make_golden.py runs definitions extracted
unmodified from the reference's sources and compiled on the host).  These pin
the oracle's Heaviside projection and its chain (a17), the sensitivity filter
(a18), the knot series, basis functions and density map of the spline (a19),
the self-support penalty functions (a21) and the surface-point self-support
pieces (background marching-cubes values, equal-distance picks, normals,
orientation, flags, per-point constraint and coefficient gradient) to the
reference's arithmetic.

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


def surface_problem(oracle, g):
    e = int(g["ereso"])
    o = box_problem(oracle, np.ones((e, e, e), np.uint8))
    o.spline_setup(int(g["order"]), [int(v) for v in g["parts"]])
    return o


def test_golden_surface_background(oracle):
    """Background marching-cubes grid of a 16^3 model box at resolution 16
    (grid/Grid.cu:4109-4160): cell-centre coordinates bit-identical (same float
    arithmetic), values (spline - 0.5, 0 - 0.5 outside the box) within 1e-6;
    equal-distance picks (grid/Grid.cpp:3831-3847) identical except where the
    reference's last pick is one past the list, which the oracle clamps."""
    g = golden("surface.npz")
    o = surface_problem(oracle, g)
    e, mc = int(g["ereso"]), int(g["mc"])
    val, pos = o.mc_values(g["coeff"].astype(np.float64), mc, box=np.array([0, 0, 0, e, e, e], np.float32))
    ref = g["mc_out"]
    assert np.array_equal(pos, ref[:3])
    assert np.abs(val - ref[3]).max() <= 1e-6
    assert np.array_equal(val <= 0, ref[3] <= 0)
    off = 0
    for rng_, m in g["equi_pairs"]:
        ref_idx = g["equi"][off:off + m]
        off += m
        idx = np.zeros(m, np.int64)
        assert oracle.lib().or_equidistant(int(rng_), int(m), idx.ctypes.data_as(oracle._i64)) == m
        assert np.array_equal(idx, np.minimum(ref_idx, rng_ - 1)), (rng_, m)
    assert off == g["equi"].size


def test_golden_surface_constraint(oracle):
    """At 500 seeded points of the 16^3 box (order 3, 4x3x5 partitions, beta 8,
    135 degree angles): the outward normals (spline gradient, flipped by the
    orientation probes of grid/Grid.cu:5800-5943) within 2e-6 of the largest,
    the probe sum and the overhang flags exact, and for each of the six modes
    the per-point values within 1e-5, the count exact, the mean within 1e-5
    and the coefficient gradient within 1e-5 of its largest entry (the
    reference accumulates it in FP32)."""
    g = golden("surface.npz")
    o = surface_problem(oracle, g)
    c = g["coeff"].astype(np.float64)
    opt = float(np.float32(g["opt_ratio"] * np.pi))
    dft = float(np.float32(g["default_ratio"] * np.pi))
    sc = g["scalars"]
    for mode in range(6):
        r = o.surface_selfsupport(c, g["pts"], float(g["beta"]), mode, opt, dft)
        assert r["dirsum"] == sc[0]
        assert close(r["normals"], g["normals"], 2e-6)
        assert np.array_equal(r["flags"][0], g["flag"].astype(np.uint8))
        assert close(r["per"], g["per"][mode], 1e-5), mode
        assert r["count"] == sc[1 + 2 * mode], mode
        assert abs(r["value"] - sc[2 + 2 * mode]) <= 1e-5 * max(1.0, abs(sc[2 + 2 * mode])), mode
        assert close(r["dc"], g["dc"][mode], 1e-5), mode
